// Constant-mass-flow correction and device reductions.
//
// compute_dP{x,y,z}_for_constant_mass_flow (src/mass_flow.f90:144-267) and
// their use at the end of compute_time_step_RK3 (src/time_integration.f90:187-211);
// for x:
//   Int_U = sum_{k=2}^{nzg-1} sum_{j=3}^{nyg-1} sum_{i=2}^{nx-1}
//              (Hu(j) U(j) + Hu(j-1) U(j-1)) * 0.5*(yg(j)-yg(j-1))
//   norm  = same with U = 1
//   shift = Qflow_x_0 - Int_U/norm;  U(interior) += shift;  BC;
//   dPdx  = 0.5*(dPdx_prev + shift/dt);
// y (V between the walls y(1:ny)) and z (W, yg weights) likewise.
// The z range includes plane nzg-1, the periodic duplicate of plane 2, exactly
// as the reference's last rank does.  Reductions are deterministic: a fixed
// grid writes per-block partials that one block sums in a fixed order.
#include "c3d_internal.cuh"

namespace c3d {

static const int kRedBlocks = 148 * 4;
static const int kRedThreads = 256;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double2 block_sum2(double2 v) {
  __shared__ double sx[32], sy[32];
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sx[wid] = v.x; sy[wid] = v.y; }
  __syncthreads();
  double2 r = make_double2(0.0, 0.0);
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    r.x = lane < nw ? sx[lane] : 0.0;
    r.y = lane < nw ? sy[lane] : 0.0;
    r.x = warp_sum(r.x);
    r.y = warp_sum(r.y);
  }
  __syncthreads();
  return r;
}

// Trapezoid flux of one field: sum over rows (j, k) and i of
//   (H(j) F(j) + H(j-1) F(j-1)) * w(j)      and      (H(j) + H(j-1)) * w(j)
// with F(i,j,k) at Fortran offset (i-1) + f1*((j-1) + f2*(k-1)) and H at the
// same position of its own extents (h1, h2); H null means H = 1.
struct FluxView {
  const double* F;
  int64_t f1, f2;
  const double* H;
  int64_t h1, h2;
  const double* w;                // per-j weight
  int i0, ni, j0, nj, k0, nk;     // i0..i0+ni-1, j0..j0+nj-1 (pairs j, j-1), k0..k0+nk-1
};

// the three fluxes of src/mass_flow.f90 on the handle's fields
//   comp 0: U between yg(2:nyg-1), i = 2..nx-1, k = 2..nzg-1 (:24-53, :144-175)
//   comp 1: V between y(1:ny),     i = 2..nxg-1, k = 2..nzg-1 (:62-91, :190-221)
//   comp 2: W between yg(2:nyg-1), i = 2..nxg-1, k = 2..nz-1  (:100-129, :236-267)
// For comp 2 the correction routine declares its dummy W with the extents of
// U, Dimension(nx,nyg,nzg) (:238), so its W(i,j,k) is the real W's element at
// offset (i-1) + nx*((j-1) + nyg*(k-1)); u_view = true reads that view (every
// offset reached lies inside W), false the true layout (compute_mean_mass_flow_W).
static FluxView flux_view(Handle* h, int comp, const double* F, const double* H, bool u_view) {
  const Dims& d = h->d;
  FluxView v{};
  v.F = F;
  v.H = H;
  if (comp == 0) {
    v.f1 = v.h1 = d.nx; v.f2 = v.h2 = d.nyg;
    v.w = h->m.wq;
    v.i0 = 2; v.ni = d.nx - 2; v.j0 = 3; v.nj = d.nyg - 3; v.k0 = 2; v.nk = d.nzg - 2;
  } else if (comp == 1) {
    v.f1 = v.h1 = d.nxg; v.f2 = v.h2 = d.ny;
    v.w = h->m.wqv;
    v.i0 = 2; v.ni = d.nxg - 2; v.j0 = 2; v.nj = d.ny - 1; v.k0 = 2; v.nk = d.nzg - 2;
  } else {
    v.f1 = u_view ? d.nx : d.nxg; v.f2 = d.nyg;
    v.h1 = d.nxg; v.h2 = d.nyg;
    v.w = h->m.wq;
    v.i0 = 2; v.ni = d.nxg - 2; v.j0 = 3; v.nj = d.nyg - 3; v.k0 = 2; v.nk = d.nz - 2;
  }
  return v;
}

// One warp per x-row (j, k) so that a row's index arithmetic is done once.
// Every block writes its partial sum; the last block to finish (ticket in
// DevScalars) adds the partials in block order and
//   mode 0: stores qflow = flux/norm;
//   mode 1: also the constant-flux correction of component comp
//           (shift = q0 - flux/norm) and dPd{x,y,z} = (dPd_prev + shift/dt)/2
//           (RK3, src/time_integration.f90:187-211);
//   mode 2: the same with dPd{x,y} = shift/dt (Euler, :65-78).
__global__ void __launch_bounds__(kRedThreads) k_flux(FluxView v, double2* __restrict__ part, DevScalars* sc,
                                                     double q0, double dt, int mode, int comp) {
  const int nrows = v.nj * v.nk;
  const int lane = threadIdx.x & 31;
  const int wpb = kRedThreads / 32;
  double2 acc = make_double2(0.0, 0.0);
  for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < nrows; row += gridDim.x * wpb) {
    const int kk = row / v.nj;
    const int j = v.j0 + (row - kk * v.nj);
    const int k = v.k0 + kk;
    const double w = v.w[j];
    const int64_t a0 = (v.i0 - 1) + v.f1 * ((j - 1) + v.f2 * (int64_t)(k - 1)), b0 = a0 - v.f1;
    const int64_t ha0 = (v.i0 - 1) + v.h1 * ((j - 1) + v.h2 * (int64_t)(k - 1)), hb0 = ha0 - v.h1;
    for (int ii = lane; ii < v.ni; ii += 32) {
      const double fa = v.F[a0 + ii], fb = v.F[b0 + ii];
      if (v.H) {
        const double ha = v.H[ha0 + ii], hb = v.H[hb0 + ii];
        acc.x += (ha * fa + hb * fb) * w;
        acc.y += (ha + hb) * w;
      } else {
        acc.x += (fa + fb) * w;
        acc.y += 2.0 * w;
      }
    }
  }
  double2 s = block_sum2(acc);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double2 t = make_double2(0.0, 0.0);
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    const double2 pv = __ldcg(part + b);
    t.x += pv.x;
    t.y += pv.y;
  }
  t = block_sum2(t);
  if (threadIdx.x == 0) {
    const double q = t.x / t.y;
    sc->qflow = q;
    if (mode >= 1) {
      const double shift = q0 - t.x / t.y;
      double* dp = comp == 0 ? &sc->dPdx : (comp == 1 ? &sc->dPdy : &sc->dPdz);
      if (comp == 0) {
        sc->shift = shift;
        sc->dpdx_prev = sc->dPdx;
      } else if (comp == 1) {
        sc->shift_v = shift;
      } else {
        sc->shift_w = shift;
      }
      *dp = mode == 1 ? 0.5 * (*dp + shift / dt) : shift / dt;
    }
    sc->ticket = 0u;
  }
}

// F(interior) += shift followed by the boundary conditions is, entry for
// entry, F += shift on every copy of an interior value, and on the y ghost
// rows (j = 1, n2): -shift for the odd ghosts of U and W, nothing for the
// zero wall values of V (face = 1).  One warp per x-row of the whole array.
__global__ void __launch_bounds__(256) k_shift_field(double* __restrict__ F, int n1, int n2, int n3, int face,
                                                    const double* __restrict__ shift) {
  const double s = *shift;
  const int nrows = n2 * n3;
  const int lane = threadIdx.x & 31;
  for (int row = blockIdx.x * 8 + (threadIdx.x >> 5); row < nrows; row += gridDim.x * 8) {
    const int j = 1 + row % n2;
    const bool wall = (j == 1 || j == n2);
    if (face && wall) continue;
    const double sr = wall ? -s : s;
    double* f = F + (int64_t)row * n1;
    for (int i = lane; i < n1; i += 32) f[i] += sr;
  }
}

static const double* flux_weight(Handle* h, int comp) {
  if (!h->ib) return nullptr;
  return comp == 0 ? ib_hu(h) : (comp == 1 ? ib_hv(h) : ib_hw(h));
}

// constant mass flow at the end of compute_time_step_RK3,
// src/time_integration.f90:187-211: x, then y, then z, each only when
// enabled; euler: that of compute_time_step_Euler (:65-78, x and y only,
// dPd = shift/dt)
int launch_massflow_correction(Handle* h, double dt, bool euler, bool skip_x) {
  const Dims& d = h->d;
  const int on[3] = {skip_x ? 0 : h->p.x_mass_cte, h->p.y_mass_cte, euler ? 0 : h->p.z_mass_cte};
  const double q0[3] = {h->Qflow_x_0, h->Qflow_y_0, h->Qflow_z_0};
  double* F[3] = {h->U, h->V, h->W};
  const int n1[3] = {d.nx, d.nxg, d.nxg}, n2[3] = {d.nyg, d.ny, d.nyg}, n3[3] = {d.nzg, d.nzg, d.nz};
  const double* sh[3] = {&h->sc->shift, &h->sc->shift_v, &h->sc->shift_w};
  for (int c = 0; c < 3; ++c) {
    if (on[c] != 1) continue;
    // with an immersed body the flux is H-weighted (src/mass_flow.f90:160-163)
    const FluxView v = flux_view(h, c, F[c], flux_weight(h, c), true);
    k_flux<<<kRedBlocks, kRedThreads, 0, h->stream>>>(v, (double2*)h->red, h->sc, q0[c], dt, euler ? 2 : 1, c);
    C3D_LAUNCH_CHECK(h);
    k_shift_field<<<148 * 8, 256, 0, h->stream>>>(F[c], n1[c], n2[c], n3[c], c == 1 ? 1 : 0, sh[c]);
    C3D_LAUNCH_CHECK(h);
  }
  return 0;
}

// bulk flux of component comp (flux/norm) of the handle's field; u_view: the
// mis-shaped view of the z correction (comp 2 only)
int massflow(Handle* h, int comp, bool u_view, double* q_out) {
  const double* F = comp == 0 ? h->U : (comp == 1 ? h->V : h->W);
  const FluxView v = flux_view(h, comp, F, flux_weight(h, comp), u_view);
  k_flux<<<kRedBlocks, kRedThreads, 0, h->stream>>>(v, (double2*)h->red, h->sc, 0.0, 1.0, 0, comp);
  C3D_LAUNCH_CHECK(h);
  double q = 0;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(&q, &h->sc->qflow, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  *q_out = q;
  return 0;
}

// compute_mean_mass_flow_V applied to W, as compute_statistics calls it
// (src/statistics.f90:133): W read through V's declared extents (nxg, ny,
// nzg) with V's loops and weights (every offset reached lies inside W)
int massflow_w_as_v(Handle* h, double* q_out) {
  FluxView v = flux_view(h, 1, h->W, flux_weight(h, 1), false);
  k_flux<<<kRedBlocks, kRedThreads, 0, h->stream>>>(v, (double2*)h->red, h->sc, 0.0, 1.0, 0, 1);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(q_out, &h->sc->qflow, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

// ---- max |div u| over cells (i,j,k) in 2..nxg-1 x 2..nyg-1 x 2..nzg-1 ----
__global__ void __launch_bounds__(kRedThreads) k_maxdiv(Dims d, Metric m, const double* __restrict__ U,
                                                       const double* __restrict__ V,
                                                       const double* __restrict__ W,
                                                       double* __restrict__ part) {
  const int ni = d.nxg - 2, nj = d.nyg - 2, nk = d.nzg - 2;
  const int64_t tot = (int64_t)ni * nj * nk;
  double mx = 0.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(t % ni);
    const int j = 2 + (int)((t / ni) % nj);
    const int k = 2 + (int)(t / ((int64_t)ni * nj));
    const double v = (U[idxU(d, i, j, k)] - U[idxU(d, i - 1, j, k)]) * m.rdx[i]
                   + (V[idxV(d, i, j, k)] - V[idxV(d, i, j - 1, k)]) * m.rdy[j]
                   + (W[idxW(d, i, j, k)] - W[idxW(d, i, j, k - 1)]) * m.rdz[k];
    mx = fmax(mx, fabs(v));
  }
  __shared__ double sm[kRedThreads];
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

int max_abs_divergence(Handle* h, const double* U, const double* V, const double* W, double* out) {
  k_maxdiv<<<kRedBlocks, kRedThreads, 0, h->stream>>>(h->d, h->m, U, V, W, h->red);
  C3D_LAUNCH_CHECK(h);
  std::vector<double> part(kRedBlocks);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->red, sizeof(double) * kRedBlocks,
                                  cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  double mx = 0.0;
  for (double v : part) mx = v > mx ? v : mx;
  *out = mx;
  return 0;
}

// ---- finiteness scan of U, V, W ----
__global__ void k_finite(const double* __restrict__ a, int64_t n, int* flag) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (!isfinite(a[t])) { *flag = 1; return; }
  }
}

int check_finite(Handle* h, bool* ok) {
  int* flag = (int*)(h->red + 2 * kRedBlocks + 8);
  C3D_CUDA_TRY(h, cudaMemsetAsync(flag, 0, sizeof(int), h->stream));
  k_finite<<<148 * 4, 256, 0, h->stream>>>(h->U, sizeU(h->d), flag);
  C3D_LAUNCH_CHECK(h);
  k_finite<<<148 * 4, 256, 0, h->stream>>>(h->V, sizeV(h->d), flag);
  C3D_LAUNCH_CHECK(h);
  k_finite<<<148 * 4, 256, 0, h->stream>>>(h->W, sizeW(h->d), flag);
  C3D_LAUNCH_CHECK(h);
  int f = 0;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(&f, flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  *ok = (f == 0);
  return 0;
}

// ---- compute_dt with CFL > 0 (src/time_integration.f90:227-262) ----
__global__ void __launch_bounds__(kRedThreads) k_cfl(Dims d, const double* __restrict__ xg,
                                                    const double* __restrict__ yg,
                                                    const double* __restrict__ zg,
                                                    const double* __restrict__ U,
                                                    const double* __restrict__ V,
                                                    const double* __restrict__ W,
                                                    double* __restrict__ part) {
  const int ni = d.nxg - 2, nj = d.nyg - 2, nk = d.nzg - 2;
  const int64_t tot = (int64_t)ni * nj * nk;
  double mu = 0.0, mv = 0.0, mw = 0.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(t % ni);
    const int j = 2 + (int)((t / ni) % nj);
    const int k = 2 + (int)(t / ((int64_t)ni * nj));
    mu = fmax(mu, (xg[i + 1] - xg[i]) / fabs(U[idxU(d, i, j, k)]));
    mv = fmax(mv, (yg[j + 1] - yg[j]) / fabs(V[idxV(d, i, j, k)]));
    mw = fmax(mw, (zg[k + 1] - zg[k]) / fabs(W[idxW(d, i, j, k)]));
  }
  __shared__ double s[3][kRedThreads];
  s[0][threadIdx.x] = mu; s[1][threadIdx.x] = mv; s[2][threadIdx.x] = mw;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = fmax(s[c][threadIdx.x], s[c][threadIdx.x + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) part[3 * blockIdx.x + c] = s[c][0];
}

int compute_dt_cfl(Handle* h, double* dt) {
  const Params& p = h->p;
  if (p.CFL < 0) { *dt = -p.CFL; return 0; }
  double* xg = nullptr;
  // grids on device: reuse the tail of the reduction buffer for xg, yg, zg
  const Dims& d = h->d;
  double* g = h->red + 4 * kRedBlocks;
  xg = g;
  double* yg = xg + d.nxg + 2;
  double* zg = yg + d.nyg + 2;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(xg, h->xg.data(), sizeof(double) * (d.nxg + 1), cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(yg, h->yg.data(), sizeof(double) * (d.nyg + 1), cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(zg, h->zg.data(), sizeof(double) * (d.nzg + 1), cudaMemcpyHostToDevice, h->stream));
  k_cfl<<<kRedBlocks, kRedThreads, 0, h->stream>>>(d, xg, yg, zg, h->U, h->V, h->W, h->red);
  C3D_LAUNCH_CHECK(h);
  std::vector<double> part(3 * kRedBlocks);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(part.data(), h->red, sizeof(double) * 3 * kRedBlocks,
                                  cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  double lu = 0, lv = 0, lw = 0;
  for (int b = 0; b < kRedBlocks; ++b) {
    lu = part[3 * b] > lu ? part[3 * b] : lu;
    lv = part[3 * b + 1] > lv ? part[3 * b + 1] : lv;
    lw = part[3 * b + 2] > lw ? part[3 * b + 2] : lw;
  }
  double dtc = p.CFL * lu;
  dtc = p.CFL * lv < dtc ? p.CFL * lv : dtc;
  dtc = p.CFL * lw < dtc ? p.CFL * lw : dtc;
  // CFL*dxmin**2/nu in the reference's order (the square first)
  double dtv = p.CFL * (h->dxmin * h->dxmin) / p.nu;
  double t2 = p.CFL * (h->dymin * h->dymin) / p.nu;
  double t3 = p.CFL * (h->dzmin * h->dzmin) / p.nu;
  dtv = t2 < dtv ? t2 : dtv;
  dtv = t3 < dtv ? t3 : dtv;
  double r = dtc < dtv ? dtc : dtv;
  *dt = r < 0.1 ? r : 0.1;
  return 0;
}

}  // namespace c3d
