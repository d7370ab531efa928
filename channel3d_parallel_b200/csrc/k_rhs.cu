// Right-hand sides and RK3 stage update.
//
// compute_rhs_u/v/w (src/equations.f90:24-423) evaluated point-wise for all
// three components in one kernel, fused with the stage update of
// compute_time_step_RK3 (src/time_integration.f90:105-107, 134-136, 163-168).
//
// Interpolations are the reference's midpoint averages (src/interpolation.f90);
// every metric division is a precomputed reciprocal factor (Metric).  The
// RK3 tableau a21 = a31 = 1/4 is exploited by keeping one accumulator
// G = Uo + dt/4 F1 instead of Uo and F1:
//   stage 1:  U* = U + dt*8/15*F1,   G = U + dt/4*F1
//   stage 2:  U* = G + dt*5/12*F2
//   stage 3:  U* = G + dt*3/4 *F3     (a32 = 0)
// which is the reference's update up to FP64 rounding order.
#include "c3d_internal.cuh"

namespace c3d {

struct RhsArgs {
  Dims d;
  Metric m;
  const double* __restrict__ U;
  const double* __restrict__ V;
  const double* __restrict__ W;
  const double* __restrict__ Gu;   // accumulators in (stages 2,3)
  const double* __restrict__ Gv;
  const double* __restrict__ Gw;
  double* __restrict__ Us;         // stage outputs (interior)
  double* __restrict__ Vs;
  double* __restrict__ Ws;
  double* __restrict__ Gu_out;     // accumulators out (stage 1)
  double* __restrict__ Gv_out;
  double* __restrict__ Gw_out;
  const double* __restrict__ Hu;   // exterior pressure-gradient masks (IB) or null
  const double* __restrict__ Hv;
  const double* __restrict__ Hw;
  const DevScalars* sc;
  double cs;   // coefficient of F for U*
  double cg;   // coefficient of F for G (stage 1)
  int comp_mask;  // rhs-only mode: which components to write (bit0 u, bit1 v, bit2 w)
};

// MODE 0: write F into rhs_u/v/w arrays (fine entries), incl. the duplicated
// periodic planes the reference also computes.  MODE 1: stage 1.  MODE 2: stage 2/3.
template <int MODE>
__global__ void __launch_bounds__(256) k_rhs(RhsArgs a) {
  const Dims& d = a.d;
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.Nx + 1 || j > d.Ny + 1 || k > d.Nz + 1) return;
  const Metric& m = a.m;
  const double* __restrict__ U = a.U;
  const double* __restrict__ V = a.V;
  const double* __restrict__ W = a.W;
#define LU(ii, jj, kk) __ldg(U + idxU(d, ii, jj, kk))
#define LV(ii, jj, kk) __ldg(V + idxV(d, ii, jj, kk))
#define LW(ii, jj, kk) __ldg(W + idxW(d, ii, jj, kk))
  const double dPdx = a.sc->dPdx, dPdy = a.sc->dPdy, dPdz = a.sc->dPdz;

  // ---- shared loads
  const double u0 = LU(i, j, k), uxm = LU(i - 1, j, k), uxp = LU(i + 1, j, k);
  const double uym = LU(i, j - 1, k), uyp = LU(i, j + 1, k);
  const double uzm = LU(i, j, k - 1), uzp = LU(i, j, k + 1);
  const double v0 = LV(i, j, k), vxp = LV(i + 1, j, k), vym = LV(i, j - 1, k);
  const double w0 = LW(i, j, k), wxp = LW(i + 1, j, k), wzm = LW(i, j, k - 1);

  // ---------------- Fu (src/equations.f90:40-151)
  double Fu;
  {
    const double v1m = LV(i + 1, j - 1, k);
    const double w1m = LW(i + 1, j, k - 1);
    const double ap = u0 + uxp, am = uxm + u0;
    double r = (am * am - ap * ap) * (0.25 * m.rdxg[i]);
    r += ((uym + u0) * (vym + v1m) - (u0 + uyp) * (v0 + vxp)) * (0.25 * m.rdy[j]);
    r += ((uzm + u0) * (wzm + w1m) - (u0 + uzp) * (w0 + wxp)) * (0.25 * m.rdz[k]);
    const double visc = m.cxpF[i] * (uxp - u0) - m.cxmF[i] * (u0 - uxm)
                      + m.cypC[j] * (uyp - u0) - m.cymC[j] * (u0 - uym)
                      + m.czpC[k] * (uzp - u0) - m.czmC[k] * (u0 - uzm);
    r += visc;
    r += a.Hu ? dPdx * __ldg(a.Hu + idxU(d, i, j, k)) : dPdx;
    Fu = r;
  }
  // ---------------- Fw (src/equations.f90:309-421)
  double Fw;
  {
    const double wxm = LW(i - 1, j, k), wym = LW(i, j - 1, k), wyp = LW(i, j + 1, k);
    const double wzp = LW(i, j, k + 1);
    const double umzp = LU(i - 1, j, k + 1);
    const double vzp = LV(i, j, k + 1), vymzp = LV(i, j - 1, k + 1);
    const double am = wzm + w0, ap = w0 + wzp;
    double r = (am * am - ap * ap) * (0.25 * m.rdzg[k]);
    r += ((uxm + umzp) * (wxm + w0) - (u0 + uzp) * (w0 + wxp)) * (0.25 * m.rdx[i]);
    r += ((vym + vymzp) * (wym + w0) - (v0 + vzp) * (w0 + wyp)) * (0.25 * m.rdy[j]);
    const double visc = m.cxpC[i] * (wxp - w0) - m.cxmC[i] * (w0 - wxm)
                      + m.cypC[j] * (wyp - w0) - m.cymC[j] * (w0 - wym)
                      + m.czpF[k] * (wzp - w0) - m.czmF[k] * (w0 - wzm);
    r += visc;
    r += a.Hw ? dPdz * __ldg(a.Hw + idxW(d, i, j, k)) : dPdz;
    Fw = r;
  }
  // ---------------- Fv (src/equations.f90:174-286), faces j = 2..ny-1
  const bool hasv = (j <= d.Ny);
  double Fv = 0.0;
  if (hasv) {
    const double vxm = LV(i - 1, j, k), vyp = LV(i, j + 1, k);
    const double vzm = LV(i, j, k - 1), vzp = LV(i, j, k + 1);
    const double um1 = LU(i - 1, j + 1, k);
    const double wyp = LW(i, j + 1, k), wypzm = LW(i, j + 1, k - 1);
    const double am = vym + v0, ap = v0 + vyp;
    double r = (am * am - ap * ap) * (0.25 * m.rdyg[j]);
    r += ((uxm + um1) * (vxm + v0) - (u0 + uyp) * (v0 + vxp)) * (0.25 * m.rdx[i]);
    r += ((vzm + v0) * (wzm + wypzm) - (v0 + vzp) * (w0 + wyp)) * (0.25 * m.rdz[k]);
    const double visc = m.cxpC[i] * (vxp - v0) - m.cxmC[i] * (v0 - vxm)
                      + m.cypF[j] * (vyp - v0) - m.cymF[j] * (v0 - vym)
                      + m.czpC[k] * (vzp - v0) - m.czmC[k] * (v0 - vzm);
    r += visc;
    r += a.Hv ? dPdy * __ldg(a.Hv + idxV(d, i, j, k)) : dPdy;
    Fv = r;
  }
#undef LU
#undef LV
#undef LW

  if (MODE == 0) {
    // rhs_u(2:nx-1, 2:nyg-1, 2:nzg-1): x 2..Nx+1, z 2..Nz+2 (plane Nz+2 duplicates 2)
    const int nu1 = d.nx - 2, nu2 = d.nyg - 2;
    if (a.comp_mask & 1) {
      double* R = a.Us;
      R[(i - 2) + (int64_t)nu1 * ((j - 2) + (int64_t)nu2 * (k - 2))] = Fu;
      if (k == 2) R[(i - 2) + (int64_t)nu1 * ((j - 2) + (int64_t)nu2 * (d.Nz))] = Fu;
    }
    // rhs_v(2:nxg-1, 2:ny-1, 2:nzg-1): x 2..Nx+2
    if ((a.comp_mask & 2) && hasv) {
      double* R = a.Vs;
      const int n1 = d.nxg - 2, n2 = d.ny - 2;
      const int64_t o = (int64_t)n1 * n2;
      R[(i - 2) + (int64_t)n1 * (j - 2) + o * (k - 2)] = Fv;
      if (i == 2) R[(d.Nx) + (int64_t)n1 * (j - 2) + o * (k - 2)] = Fv;
      if (k == 2) {
        R[(i - 2) + (int64_t)n1 * (j - 2) + o * d.Nz] = Fv;
        if (i == 2) R[(d.Nx) + (int64_t)n1 * (j - 2) + o * d.Nz] = Fv;
      }
    }
    // rhs_w(2:nxg-1, 2:nyg-1, 2:nz-1): x 2..Nx+2
    if (a.comp_mask & 4) {
      double* R = a.Ws;
      const int n1 = d.nxg - 2, n2 = d.nyg - 2;
      const int64_t o = (int64_t)n1 * n2;
      R[(i - 2) + (int64_t)n1 * (j - 2) + o * (k - 2)] = Fw;
      if (i == 2) R[(d.Nx) + (int64_t)n1 * (j - 2) + o * (k - 2)] = Fw;
    }
    return;
  }

  const int64_t iu = idxU(d, i, j, k), iw = idxW(d, i, j, k);
  if (MODE == 1) {
    a.Us[iu] = u0 + a.cs * Fu;
    a.Gu_out[iu] = u0 + a.cg * Fu;
    a.Ws[iw] = w0 + a.cs * Fw;
    a.Gw_out[iw] = w0 + a.cg * Fw;
    if (hasv) {
      const int64_t iv = idxV(d, i, j, k);
      a.Vs[iv] = v0 + a.cs * Fv;
      a.Gv_out[iv] = v0 + a.cg * Fv;
    }
  } else {
    a.Us[iu] = __ldg(a.Gu + iu) + a.cs * Fu;
    a.Ws[iw] = __ldg(a.Gw + iw) + a.cs * Fw;
    if (hasv) {
      const int64_t iv = idxV(d, i, j, k);
      a.Vs[iv] = __ldg(a.Gv + iv) + a.cs * Fv;
    }
  }
}

// ---------------------------------------------------------------------------
// Tiled stage kernel: a CTA owns a TX x TY tile of (i, j) columns and marches
// over a run of KC z planes, keeping planes k-1, k, k+1 of U, V and W (tile
// plus a one-cell halo in x and y) in a rolling shared-memory window.  Every
// field value is read from HBM once per CTA (halo overhead (TX+2)(TY+2)/(TX*TY));
// the arithmetic is that of k_rhs.
// ---------------------------------------------------------------------------
constexpr int TX = 32, TY = 8, KC = 64;
constexpr int PX = TX + 2, PY = TY + 2, PN = PX * PY;
constexpr int NSLOT = 8;   // planes k-1, k, k+1 in use, k+2..k+4 in flight
constexpr int AHEAD = 3;   // planes issued beyond k+1

__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  const int n = valid ? 8 : 0;   // src-size 0 zero-fills the destination
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int MODE>
__global__ void __launch_bounds__(TX * TY, 2) k_rhs_tiled(RhsArgs a) {
  extern __shared__ double rhs_smem[];
  double (*sU)[PN] = reinterpret_cast<double (*)[PN]>(rhs_smem);
  double (*sV)[PN] = reinterpret_cast<double (*)[PN]>(rhs_smem + NSLOT * PN);
  double (*sW)[PN] = reinterpret_cast<double (*)[PN]>(rhs_smem + 2 * NSLOT * PN);
  double* sZ = rhs_smem + 3 * NSLOT * PN;     // z factors of planes k0..k1: [6][KC]
  const Dims& d = a.d;
  const Metric& m = a.m;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * TX + tx;
  const int i0 = 2 + blockIdx.x * TX, j0 = 2 + blockIdx.y * TY;
  const int k0 = 2 + blockIdx.z * KC;
  const int k1 = min(k0 + KC - 1, d.Nz + 1);
  const int i = i0 + tx, j = j0 + ty;
  const bool active = (i <= d.Nx + 1) && (j <= d.Ny + 1);
  const bool hasv = active && (j <= d.Ny);

  // halo-tile positions of this thread (at most two: PN <= 2 * TX * TY): the
  // offset of plane 1 and the x/y validity are fixed, plane k adds k-1 planes
  constexpr int kPos = (PN + TX * TY - 1) / (TX * TY);
  int64_t offU[kPos], offV[kPos], offW[kPos];
  bool okU[kPos], okV[kPos], okW[kPos];
#pragma unroll
  for (int q = 0; q < kPos; ++q) {
    const int t = tid + q * TX * TY;
    const int li = t % PX, lj = t / PX;
    const int gi = i0 - 1 + li, gj = j0 - 1 + lj;
    const bool in = t < PN;
    okU[q] = in && gi <= d.nx && gj <= d.nyg;
    okV[q] = in && gi <= d.nxg && gj <= d.ny;
    okW[q] = in && gi <= d.nxg && gj <= d.nyg;
    offU[q] = okU[q] ? idxU(d, gi, gj, 1) : 0;
    offV[q] = okV[q] ? idxV(d, gi, gj, 1) : 0;
    offW[q] = okW[q] ? idxW(d, gi, gj, 1) : 0;
  }
  const int64_t plU = (int64_t)d.nx * d.nyg, plV = (int64_t)d.nxg * d.ny, plW = (int64_t)d.nxg * d.nyg;
  for (int t = tid; t < 6 * KC; t += TX * TY) {
    const int q = t / KC, kk = k0 + (t - q * KC);
    const double* f = q == 0 ? m.rdz : q == 1 ? m.rdzg : q == 2 ? m.czpC : q == 3 ? m.czmC : q == 4 ? m.czpF : m.czmF;
    sZ[t] = kk <= k1 ? f[kk] : 0.0;
  }
  pdl_wait();
  pdl_trigger();
  // asynchronous copy of plane k (tile + halo) of U, V, W into a slot
  auto issue_plane = [&](int k) {
    const int slot = k & (NSLOT - 1);
    const int64_t kk = k - 1;
#pragma unroll
    for (int q = 0; q < kPos; ++q) {
      const int t = tid + q * TX * TY;
      if (t < PN) {
        const bool vu = okU[q] && k <= d.nzg, vv = okV[q] && k <= d.nzg, vw = okW[q] && k <= d.nz;
        cp_async8(&sU[slot][t], vu ? a.U + offU[q] + kk * plU : a.U, vu);
        cp_async8(&sV[slot][t], vv ? a.V + offV[q] + kk * plV : a.V, vv);
        cp_async8(&sW[slot][t], vw ? a.W + offW[q] + kk * plW : a.W, vw);
      }
    }
    cp_async_commit();
  };
  const double dPdx = a.sc->dPdx, dPdy = a.sc->dPdy, dPdz = a.sc->dPdz;
  issue_plane(k0 - 1);
  issue_plane(k0);
  for (int q = 1; q <= AHEAD; ++q) {
    if (k0 + q <= k1 + 1) issue_plane(k0 + q);
    else cp_async_commit();
  }
  const int c = (ty + 1) * PX + (tx + 1);     // own cell in the padded tile
  // x- and y-indexed metric factors of this column, constant over the march
  const int ic = active ? i : 2, jc = active ? j : 2;
  const double rdxg_i = m.rdxg[ic], rdx_i = m.rdx[ic];
  const double cxpF_i = m.cxpF[ic], cxmF_i = m.cxmF[ic], cxpC_i = m.cxpC[ic], cxmC_i = m.cxmC[ic];
  const double rdy_j = m.rdy[jc], rdyg_j = m.rdyg[jc];
  const double cypC_j = m.cypC[jc], cymC_j = m.cymC[jc], cypF_j = m.cypF[jc], cymF_j = m.cymF[jc];
  const int64_t iu0 = idxU(d, ic, jc, 1), iv0 = idxV(d, ic, jc, 1), iw0 = idxW(d, ic, jc, 1);
  // accumulators, loaded one plane ahead of their use
  double gu = 0.0, gv = 0.0, gw = 0.0;
  if (MODE == 2 && active) {
    const int64_t kk = k0 - 1;
    gu = __ldg(a.Gu + iu0 + kk * plU);
    gw = __ldg(a.Gw + iw0 + kk * plW);
    if (hasv) gv = __ldg(a.Gv + iv0 + kk * plV);
  }
  for (int k = k0; k <= k1; ++k) {
    if (k + 1 + AHEAD <= k1 + 1) issue_plane(k + 1 + AHEAD);
    else cp_async_commit();                   // keep the group count uniform
    cp_async_wait<AHEAD>();                   // planes up to k+1 have landed
    __syncthreads();
    const int sm = (k - 1) & (NSLOT - 1), s0 = k & (NSLOT - 1), sp = (k + 1) & (NSLOT - 1);
    const int kz = k - k0;
    const double rdz_k = sZ[kz], rdzg_k = sZ[KC + kz];
    const double czpC_k = sZ[2 * KC + kz], czmC_k = sZ[3 * KC + kz];
    const double czpF_k = sZ[4 * KC + kz], czmF_k = sZ[5 * KC + kz];
    if (active) {
      const int64_t kk = k - 1;
      const int64_t iu = iu0 + kk * plU, iw = iw0 + kk * plW;
      const int64_t iv = iv0 + kk * plV;
      double gu_n = 0.0, gv_n = 0.0, gw_n = 0.0;
      if (MODE == 2 && k < k1) {              // the next plane's accumulators
        gu_n = __ldg(a.Gu + iu + plU);
        gw_n = __ldg(a.Gw + iw + plW);
        if (hasv) gv_n = __ldg(a.Gv + iv + plV);
      }
#define AU(s, di, dj) sU[s][c + (di) + (dj) * PX]
#define AV(s, di, dj) sV[s][c + (di) + (dj) * PX]
#define AW(s, di, dj) sW[s][c + (di) + (dj) * PX]
      const double u0 = AU(s0, 0, 0), uxm = AU(s0, -1, 0), uxp = AU(s0, 1, 0);
      const double uym = AU(s0, 0, -1), uyp = AU(s0, 0, 1);
      const double uzm = AU(sm, 0, 0), uzp = AU(sp, 0, 0);
      const double v0 = AV(s0, 0, 0), vxp = AV(s0, 1, 0), vym = AV(s0, 0, -1);
      const double w0 = AW(s0, 0, 0), wxp = AW(s0, 1, 0), wzm = AW(sm, 0, 0);
      double Fu, Fv = 0.0, Fw;
      {
        const double v1m = AV(s0, 1, -1);
        const double w1m = AW(sm, 1, 0);
        // independent partial sums (short dependency chains)
        const double ap = u0 + uxp, am = uxm + u0;
        const double cx = (am * am - ap * ap) * (0.25 * rdxg_i);
        const double cy = ((uym + u0) * (vym + v1m) - (u0 + uyp) * (v0 + vxp)) * (0.25 * rdy_j);
        const double cz = ((uzm + u0) * (wzm + w1m) - (u0 + uzp) * (w0 + wxp)) * (0.25 * rdz_k);
        const double vx = cxpF_i * (uxp - u0) - cxmF_i * (u0 - uxm);
        const double vy = cypC_j * (uyp - u0) - cymC_j * (u0 - uym);
        const double vz = czpC_k * (uzp - u0) - czmC_k * (u0 - uzm);
        const double f = a.Hu ? dPdx * __ldg(a.Hu + iu) : dPdx;
        Fu = ((cx + cy) + (cz + f)) + ((vx + vy) + vz);
      }
      {
        const double wxm = AW(s0, -1, 0), wym = AW(s0, 0, -1), wyp = AW(s0, 0, 1);
        const double wzp = AW(sp, 0, 0);
        const double umzp = AU(sp, -1, 0);
        const double vzp = AV(sp, 0, 0), vymzp = AV(sp, 0, -1);
        const double am = wzm + w0, ap = w0 + wzp;
        const double cz = (am * am - ap * ap) * (0.25 * rdzg_k);
        const double cx = ((uxm + umzp) * (wxm + w0) - (u0 + uzp) * (w0 + wxp)) * (0.25 * rdx_i);
        const double cy = ((vym + vymzp) * (wym + w0) - (v0 + vzp) * (w0 + wyp)) * (0.25 * rdy_j);
        const double vx = cxpC_i * (wxp - w0) - cxmC_i * (w0 - wxm);
        const double vy = cypC_j * (wyp - w0) - cymC_j * (w0 - wym);
        const double vz = czpF_k * (wzp - w0) - czmF_k * (w0 - wzm);
        const double f = a.Hw ? dPdz * __ldg(a.Hw + iw) : dPdz;
        Fw = ((cz + cx) + (cy + f)) + ((vx + vy) + vz);
      }
      if (hasv) {
        const double vxm = AV(s0, -1, 0), vyp = AV(s0, 0, 1);
        const double vzm = AV(sm, 0, 0), vzp = AV(sp, 0, 0);
        const double um1 = AU(s0, -1, 1);
        const double wyp = AW(s0, 0, 1), wypzm = AW(sm, 0, 1);
        const double am = vym + v0, ap = v0 + vyp;
        const double cy = (am * am - ap * ap) * (0.25 * rdyg_j);
        const double cx = ((uxm + um1) * (vxm + v0) - (u0 + uyp) * (v0 + vxp)) * (0.25 * rdx_i);
        const double cz = ((vzm + v0) * (wzm + wypzm) - (v0 + vzp) * (w0 + wyp)) * (0.25 * rdz_k);
        const double vx = cxpC_i * (vxp - v0) - cxmC_i * (v0 - vxm);
        const double vy = cypF_j * (vyp - v0) - cymF_j * (v0 - vym);
        const double vz = czpC_k * (vzp - v0) - czmC_k * (v0 - vzm);
        const double f = a.Hv ? dPdy * __ldg(a.Hv + iv) : dPdy;
        Fv = ((cy + cx) + (cz + f)) + ((vx + vy) + vz);
      }
#undef AU
#undef AV
#undef AW
      if (MODE == 1) {
        a.Us[iu] = u0 + a.cs * Fu;
        a.Gu_out[iu] = u0 + a.cg * Fu;
        a.Ws[iw] = w0 + a.cs * Fw;
        a.Gw_out[iw] = w0 + a.cg * Fw;
        if (hasv) {
          a.Vs[iv] = v0 + a.cs * Fv;
          a.Gv_out[iv] = v0 + a.cg * Fv;
        }
      } else {
        a.Us[iu] = gu + a.cs * Fu;
        a.Ws[iw] = gw + a.cs * Fw;
        if (hasv) a.Vs[iv] = gv + a.cs * Fv;
        gu = gu_n; gv = gv_n; gw = gw_n;
      }
    }
    // No barrier here: the slot the next iteration refills, (k+5) mod 8, held
    // plane k-3, last read in iteration k-2; every thread finished that
    // iteration before it reached this iteration's barrier.
  }
}

static RhsArgs base_args(Handle* h) {
  RhsArgs a{};
  a.d = h->d;
  a.m = h->m;
  a.U = h->U; a.V = h->V; a.W = h->W;
  a.sc = h->sc;
  if (h->p.exterior_pressure_gradient && h->ib != nullptr) {
    a.Hu = ib_hu(h); a.Hv = ib_hv(h); a.Hw = ib_hw(h);
  }
  return a;
}

static dim3 rhs_block() { return dim3(32, 4, 2); }
static dim3 rhs_grid(const Dims& d) {
  dim3 b = rhs_block();
  return dim3((d.Nx + b.x - 1) / b.x, (d.Ny + b.y - 1) / b.y, (d.Nz + b.z - 1) / b.z);
}

static const int kRhsSmem = (3 * NSLOT * PN + 6 * KC) * (int)sizeof(double);

int rhs_setup(Handle* h) {
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_rhs_tiled<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRhsSmem));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_rhs_tiled<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRhsSmem));
  return 0;
}

// stage = 1, 2, 3; U,V,W (with valid ghosts) -> Us,Vs,Ws interior (+ G at stage 1)
int launch_rhs_stage(Handle* h, int stage, double dt) {
  RhsArgs a = base_args(h);
  a.Us = h->Us; a.Vs = h->Vs; a.Ws = h->Ws;
  const Dims& d = h->d;
  const dim3 tb(TX, TY, 1);
  const dim3 tg((d.Nx + TX - 1) / TX, (d.Ny + TY - 1) / TY, (d.Nz + KC - 1) / KC);
  if (stage == 1) {
    a.Gu_out = h->Gu; a.Gv_out = h->Gv; a.Gw_out = h->Gw;
    a.cs = dt * (8.0 / 15.0);
    a.cg = dt * (1.0 / 4.0);
    if (h->rhs_kernel == 0) C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_rhs_tiled<1>, tg, tb, kRhsSmem, h->stream, a));
    else k_rhs<1><<<rhs_grid(d), rhs_block(), 0, h->stream>>>(a);
  } else {
    a.Gu = h->Gu; a.Gv = h->Gv; a.Gw = h->Gw;
    a.cs = (stage == 2) ? dt * (5.0 / 12.0) : dt * (3.0 / 4.0);
    if (h->rhs_kernel == 0) C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_rhs_tiled<2>, tg, tb, kRhsSmem, h->stream, a));
    else k_rhs<2><<<rhs_grid(d), rhs_block(), 0, h->stream>>>(a);
  }
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// compute_time_step_Euler (src/time_integration.f90:34-52): U* = U + dt*F
// for the three components (the stage-1 kernel with its accumulator output
// sent to the G work fields, which Euler does not read)
int launch_rhs_euler(Handle* h, double dt) {
  RhsArgs a = base_args(h);
  a.Us = h->Us; a.Vs = h->Vs; a.Ws = h->Ws;
  a.Gu_out = h->Gu; a.Gv_out = h->Gv; a.Gw_out = h->Gw;
  a.cs = dt;
  a.cg = dt;
  const Dims& d = h->d;
  const dim3 tb(TX, TY, 1);
  const dim3 tg((d.Nx + TX - 1) / TX, (d.Ny + TY - 1) / TY, (d.Nz + KC - 1) / KC);
  if (h->rhs_kernel == 0) k_rhs_tiled<1><<<tg, tb, kRhsSmem, h->stream>>>(a);
  else k_rhs<1><<<rhs_grid(d), rhs_block(), 0, h->stream>>>(a);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// fine entries: component 1/2/3 -> rhsU/rhsV/rhsW
int launch_rhs_only(Handle* h, int component) {
  RhsArgs a = base_args(h);
  a.Us = h->rhsU; a.Vs = h->rhsV; a.Ws = h->rhsW;
  a.comp_mask = 1 << (component - 1);
  k_rhs<0><<<rhs_grid(h->d), rhs_block(), 0, h->stream>>>(a);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

}  // namespace c3d
