// Banded z-Fourier preconditioner of the Schur-complement BiCGSTAB.
//
// No counterpart in the reference: its BiCGSTAB (src/projection.f90:146-186)
// is unpreconditioned.  On a moving wall the Schur operator S of
// src/projection.f90:98-144 is indefinite and nearly singular: the diagonal
// terms -E1nH_ext*dudn and -E1nHc_ext*p_jump change sign with the offset of
// a marker inside its y cell, so a wavy plane (which visits every offset)
// has rows whose diagonal nearly cancels the spreading term.  That structure
// is local along the marker lattice; what couples markers over long
// distances is smooth.  The preconditioner therefore solves exactly with
//     B = S restricted to lattice neighbours |d| <= 2 along the first lattice
//         direction (all four components, every z distance),
// which, for bodies whose geometry does not vary along z (every body type
// here except the wall plates), is block-circulant in z: a DFT along z turns
// B into independent banded systems per z wavenumber q and lattice segment
// (a wall row, a cylinder ring), each solved by a banded LU with partial
// pivoting.
//
// B is measured, not modelled: unit probes at z row 0 of one colour class
// of markers (markers of a class are 8 lattice columns apart for the dudn
// components, 32 for the pressure jump, whose Schur response reaches far
// enough that closer probes would alias), one Schur application per class
// and component, give S's columns at every z; the band entries are read
// from them.
//
// Layout:
//   T      [iz][L], L = ((cp*lat + i1)*5 + d)*4 + c: the response in component
//          cp at lattice column nbr(i1, d), z row iz, to a unit in component c
//          at (i1, z row 0);
//   That   [q][L] its DFT over iz (q = 0 .. nzl/2);
//   AB     per system (q, segment): LAPACK band storage (ldab = 2 kl + ku + 1,
//          column-major) of the 4*len x 4*len system, rows and columns ordered
//          by folded lattice position (0, len-1, 1, len-2, ... so that a cyclic
//          band of width 2 has width 4 without wrap) times 4 plus component;
//          after factorisation the diagonal holds the reciprocal pivot.
#include <algorithm>
#include <cmath>
#include <vector>

#include "c3d_internal.cuh"
#include "ib_state.cuh"
#include "bulk.cuh"
#include "fft.cuh"

namespace c3d {

namespace {

constexpr int kKb = 2;                       // lattice neighbours along dim 1
constexpr int kNd = 2 * kKb + 1;
constexpr int kKl = 4 * (2 * kKb) + 3;       // scalar half bandwidth in folded order (19)
constexpr int kKu = kKl;
constexpr int kKv = kKl + kKu;               // 38
constexpr int kLdab = 2 * kKl + kKu + 1;     // 58
constexpr int kSolveChunk = 16;              // band columns staged per copy in the solve
constexpr int kSolveRing = 8;                // chunks in flight (seven ahead of the one in use)
constexpr int kFactorWin = 64;               // band columns resident in the factor kernel

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 crcp(double2 a) {
  // 1/a with scaling against overflow (Smith's method)
  if (fabs(a.x) >= fabs(a.y)) {
    const double r = a.y / a.x, den = a.x + a.y * r;
    return make_double2(1.0 / den, -r / den);
  }
  const double r = a.x / a.y, den = a.y + a.x * r;
  return make_double2(r / den, -1.0 / den);
}

}  // namespace

struct BandState {
  bool ok = false;                 // lattice supports the band form
  int lat = 0, nzl = 0, nq = 0, nseg = 0;
  std::vector<int> seg_start, seg_len;
  int spacing[4] = {8, 8, 8, 32};
  std::vector<std::vector<int>> colours;   // per component: used colour ids
  int* nbr_d = nullptr;            // [lat][5]
  int* pos_d = nullptr;            // [lat] system row block (segment start + folded position)
  int* seg_d = nullptr;            // [lat] segment of the column
  int* segstart_d = nullptr;       // [nseg]
  int* seglen_d = nullptr;         // [nseg]
  int* colour_d = nullptr;         // [4][lat]
  double* T_d = nullptr;           // [nzl][80 lat]
  double2* That_d = nullptr;       // [nq][80 lat]
  double2* AB_d = nullptr;         // [nq][ldab * 4 lat]
  int* ipiv_d = nullptr;           // [nq][4 lat]
  double2* rhs_d = nullptr;        // [nq][4 lat]
  // block-tridiagonal form (16 x 16 blocks: 4 lattice positions x 4 components)
  std::vector<int> nblk, blkoff;   // block rows per segment, their offset within one q
  int NBq = 0;                     // block rows per wavenumber (all segments)
  int nblk_max = 0;                // block rows of the longest segment
  int* nblk_d = nullptr;
  int* blkoff_d = nullptr;
  double2 *Ab_d = nullptr, *Bb_d = nullptr, *Cb_d = nullptr;   // [nq][NBq][16][16]
  double2 *Pb_d = nullptr, *Gb_d = nullptr;                    // Delta^-1 and Delta^-1 C
  bool block = false;              // the factors in use are the block ones
  double* tw_d = nullptr;          // [2][nzl] cos, sin of 2 pi k / nzl
  // z transforms by FFT when nzl = 2^a 3^b (else the direct DFTs)
  bool fft = false;
  FftPasses fftP{};
  double2* ftw_d = nullptr;        // [nzl] exp(-2 pi i m / nzl)
  int* fpos_d = nullptr;           // [nzl] digit-reversed position of coefficient m
  int* flag_d = nullptr;           // [0] zero pivot seen
  bool built = false;
  std::vector<double> yb_at, xb_at;
  double dt_at = 0;
  int builds = 0;
  int64_t probes = 0;
};

void band_free(IbState* s) {
  delete s->band;
  s->band = nullptr;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// unit probes of one colour class in component c at z row 0
__global__ void k_band_probe(int nb, int lat, int c, int colour, const int* __restrict__ col_of,
                             double* __restrict__ out) {
  const int64_t n = 4 * (int64_t)nb;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (t >= (int64_t)c * nb && t < (int64_t)c * nb + lat) {
      const int i1 = (int)(t - (int64_t)c * nb);
      v = col_of[c * lat + i1] == colour ? 1.0 : 0.0;
    }
    out[t] = v;
  }
}

// band entries of the probed columns from the response R = S e
__global__ void k_band_extract(int nb, int lat, int nzl, int c, int colour, const int* __restrict__ col_of,
                               const int* __restrict__ nbr, const double* __restrict__ R,
                               double* __restrict__ T) {
  const int64_t tot = (int64_t)lat * 4 * kNd * nzl;
  const int64_t nl = 80 * (int64_t)lat;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i1 = (int)(t % lat);
    int64_t r = t / lat;
    const int d = (int)(r % kNd); r /= kNd;
    const int cp = (int)(r % 4);
    const int iz = (int)(r / 4);
    if (col_of[c * lat + i1] != colour) continue;
    const int j1 = nbr[i1 * kNd + d];
    const int64_t L = (((int64_t)cp * lat + i1) * kNd + d) * 4 + c;
    T[(int64_t)iz * nl + L] = R[(int64_t)cp * nb + j1 + (int64_t)lat * iz];
  }
}

// That[q][L] = sum_iz T[iz][L] exp(-2 pi i q iz / nzl)
__global__ void k_band_dft_T(int nl, int nzl, int nq, const double* __restrict__ tw,
                             const double* __restrict__ T, double2* __restrict__ That) {
  const int64_t tot = (int64_t)nq * nl;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int L = (int)(t % nl);
    const int q = (int)(t / nl);
    double re = 0.0, im = 0.0;
    int k = 0;
    for (int iz = 0; iz < nzl; ++iz) {
      const double v = T[(int64_t)iz * nl + L];
      re += v * tw[k];
      im -= v * tw[nzl + k];
      k += q;
      if (k >= nzl) k -= nzl;
    }
    That[t] = make_double2(re, im);
  }
}

// scatter the band entries of every system into LAPACK band storage
__global__ void k_band_assemble(int lat, int nq, const int* __restrict__ nbr, const int* __restrict__ pos,
                                const int* __restrict__ seg, const int* __restrict__ segstart,
                                const double2* __restrict__ That, double2* __restrict__ AB) {
  const int nl = 80 * lat;
  const int64_t tot = (int64_t)nq * nl;
  const int64_t abq = (int64_t)kLdab * 4 * lat;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int L = (int)(t % nl);
    const int q = (int)(t / nl);
    const int c = L % 4;
    int r = L / 4;
    const int d = r % kNd; r /= kNd;
    const int i1 = r % lat;
    const int cp = r / lat;
    const int s = seg[i1];
    const int base = 4 * segstart[s];
    const int col = 4 * pos[i1] + c - base;
    const int row = 4 * pos[nbr[i1 * kNd + d]] + cp - base;
    AB[q * abq + (int64_t)kLdab * base + (int64_t)col * kLdab + kKv + row - col] = That[t];
  }
}

// Banded LU with partial pivoting of one system (LAPACK zgbtf2, 0-based),
// band columns j .. j+63 resident in shared memory; the diagonal of U is
// replaced by its reciprocal.  One CTA per system.
__global__ void __launch_bounds__(256) k_band_factor(int lat, int nseg, const int* __restrict__ segstart,
                                                     const int* __restrict__ seglen, double2* __restrict__ AB,
                                                     int* __restrict__ ipiv, int* __restrict__ flag) {
  extern __shared__ double2 win[];    // [kFactorWin][kLdab]
  __shared__ int s_jp, s_ju;
  const int q = blockIdx.x / nseg, s = blockIdx.x % nseg;
  const int m = 4 * seglen[s];
  const int base = 4 * segstart[s];
  double2* A = AB + (int64_t)q * kLdab * 4 * lat + (int64_t)kLdab * base;
  int* piv = ipiv + (int64_t)q * 4 * lat + base;
  const int tid = threadIdx.x;
  const int ncol0 = min(m, kFactorWin);
  for (int e = tid; e < ncol0 * kLdab; e += blockDim.x) win[e] = A[e];
  if (tid == 0) s_ju = 0;
  __syncthreads();
  for (int j = 0; j < m; ++j) {
    const int km = min(kKl, m - 1 - j);
    double2* cj = win + (j % kFactorWin) * kLdab;
    if (tid < 32) {
      // pivot: largest |re| + |im| among rows j .. j+km (the first on ties)
      double best = -1.0;
      int bi = 0;
      for (int t = tid; t <= km; t += 32) {
        const double2 v = cj[kKv + t];
        const double a = fabs(v.x) + fabs(v.y);
        if (a > best) { best = a; bi = t; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (tid == 0) {
        s_jp = bi;
        piv[j] = j + bi;
        if (!(best > 0.0)) atomicExch(flag, 1);
        s_ju = max(s_ju, min(j + kKu + bi, m - 1));
      }
    }
    __syncthreads();
    const int jp = s_jp, ju = s_ju;
    if (jp != 0) {
      for (int col = j + tid; col <= ju; col += blockDim.x) {
        double2* cc = win + (col % kFactorWin) * kLdab;
        const int a = kKv + j - col, b = a + jp;
        const double2 tmp = cc[a];
        cc[a] = cc[b];
        cc[b] = tmp;
      }
      __syncthreads();
    }
    const double2 piv_v = cj[kKv];
    const bool nz = (fabs(piv_v.x) + fabs(piv_v.y)) > 0.0;
    const double2 r = nz ? crcp(piv_v) : make_double2(0.0, 0.0);
    if (km > 0 && nz) {
      for (int t = 1 + tid; t <= km; t += blockDim.x) cj[kKv + t] = cmul(cj[kKv + t], r);
      __syncthreads();
      const int ncols = ju - j;
      for (int e = tid; e < ncols * km; e += blockDim.x) {
        const int col = j + 1 + e / km;
        const int t = 1 + e % km;
        double2* cc = win + (col % kFactorWin) * kLdab;
        const double2 a = cc[kKv + j - col];
        cc[kKv + j + t - col] = csub(cc[kKv + j + t - col], cmul(cj[kKv + t], a));
      }
    }
    __syncthreads();
    // column j is final: store it (diagonal as reciprocal) and bring in column j + win
    const int jn = j + kFactorWin;
    for (int e = tid; e < kLdab; e += blockDim.x) {
      double2 v = cj[e];
      if (e == kKv) v = r;
      A[(int64_t)j * kLdab + e] = v;
      if (jn < m) cj[e] = A[(int64_t)jn * kLdab + e];
    }
    __syncthreads();
  }
}

// rhs[q][4 pos(i1) + c] = sum_iz v[c nb + i1 + lat iz] exp(-2 pi i q iz / nzl).
// A CTA takes 32 lattice columns of one component and a run of kFwdQ
// wavenumbers: the columns' z lines (nzl x 32) and the twiddles are staged
// in shared memory (coalesced along the columns), each thread sums the DFT
// of one column for kFwdQ/8 wavenumbers.
constexpr int kFwdQ = 16;
__global__ void __launch_bounds__(256) k_band_fwd(int nb, int lat, int nzl, int nq, const double* __restrict__ tw,
                                                  const int* __restrict__ pos, const double* __restrict__ v,
                                                  double2* __restrict__ rhs) {
  extern __shared__ double fsm[];
  double* xs = fsm;                    // [nzl][32]
  double* twc = fsm + 32 * nzl;        // [nzl]
  double* tws = twc + nzl;             // [nzl]
  const int c = blockIdx.y;
  const int m0 = blockIdx.x * 32;
  const int q0 = blockIdx.z * kFwdQ;
  const int tid = threadIdx.x;
  // eight loads in flight per thread before any store
  for (int e0 = tid; e0 < 32 * nzl; e0 += 8 * 256) {
    double tv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * 256, iz = e >> 5, mm = e & 31;
      tv[u] = (e < 32 * nzl && m0 + mm < lat) ? v[(int64_t)c * nb + m0 + mm + (int64_t)lat * iz] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (e0 + u * 256 < 32 * nzl) xs[e0 + u * 256] = tv[u];
  }
  for (int e = tid; e < nzl; e += 256) { twc[e] = tw[e]; tws[e] = tw[nzl + e]; }
  __syncthreads();
  const int mm = tid & 31, ql = tid >> 5;
  if (m0 + mm >= lat) return;
  const int row = 4 * pos[m0 + mm] + c;
  for (int qq = ql; qq < kFwdQ; qq += 8) {
    const int q = q0 + qq;
    if (q >= nq) break;
    // two interleaved partial sums (even and odd iz): half-length FMA chains
    double re0 = 0.0, im0 = 0.0, re1 = 0.0, im1 = 0.0;
    int k = 0;
    int iz = 0;
    for (; iz + 1 < nzl; iz += 2) {
      const double x0 = xs[iz * 32 + mm], x1 = xs[(iz + 1) * 32 + mm];
      int k1 = k + q;
      if (k1 >= nzl) k1 -= nzl;
      re0 += x0 * twc[k];
      im0 -= x0 * tws[k];
      re1 += x1 * twc[k1];
      im1 -= x1 * tws[k1];
      k = k1 + q;
      if (k >= nzl) k -= nzl;
    }
    if (iz < nzl) {
      const double x0 = xs[iz * 32 + mm];
      re0 += x0 * twc[k];
      im0 -= x0 * tws[k];
    }
    rhs[(int64_t)q * 4 * lat + row] = make_double2(re0 + re1, im0 + im1);
  }
}

// The same two transforms with the shared-memory FFT engine (nzl = 2^a 3^b):
// two real columns of one component share a complex row, z = a + i b, and a
// CTA transforms kFftRows rows (2 kFftRows lattice columns).  Forward: the
// half spectra A = (Z[q] + conj Z[N-q]) / 2 and B = (Z[q] - conj Z[N-q]) / 2i
// are written to the block rows of the columns, as k_band_fwd writes them.
// Inverse: Z[k] = A[k] + i B[k] on the whole circle from the Hermitian half
// spectra (imaginary parts at q = 0 and q = N/2 dropped, the real part
// k_band_inv takes), one inverse FFT, a = Re z / N and b = Im z / N.
constexpr int kFftRows = 4;
constexpr int kFftThreads = 64;
static size_t fft_smem_bytes(int nzl) { return sizeof(double2) * kFftRows * (size_t)(nzl | 1); }

__global__ void __launch_bounds__(kFftThreads) k_band_fwd_fft(int nb, int lat, int nzl, int nq, FftPasses P,
                                                              const double2* __restrict__ tw,
                                                              const int* __restrict__ fpos,
                                                              const int* __restrict__ pos,
                                                              const double* __restrict__ v,
                                                              double2* __restrict__ rhs) {
  extern __shared__ double2 zs[];   // [kFftRows][nzl | 1]
  const int rs = nzl | 1;
  const int c = blockIdx.y, m0 = blockIdx.x * 2 * kFftRows;
  const int tid = threadIdx.x;
  const int tot = 2 * kFftRows * nzl;   // e = iz * 2 kFftRows + column
  for (int e0 = tid; e0 < tot; e0 += 8 * kFftThreads) {
    double tv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * kFftThreads, iz = e / (2 * kFftRows), mm = e % (2 * kFftRows);
      tv[u] = (e < tot && m0 + mm < lat) ? v[(int64_t)c * nb + m0 + mm + (int64_t)lat * iz] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * kFftThreads, iz = e / (2 * kFftRows), mm = e % (2 * kFftRows);
      if (e < tot) reinterpret_cast<double*>(zs + (mm >> 1) * rs + iz)[mm & 1] = tv[u];
    }
  }
  __syncthreads();
  fft_rows_dif<double, 16>(zs, kFftRows, rs, tw, P);
  for (int e = tid; e < kFftRows * nq; e += kFftThreads) {
    const int r = e / nq, q = e - r * nq;
    const double2 zq = zs[r * rs + fpos[q]];
    const double2 zn = zs[r * rs + fpos[q == 0 ? 0 : nzl - q]];
    const int ma = m0 + 2 * r, mb = ma + 1;
    if (ma < lat) rhs[(int64_t)q * 4 * lat + 4 * pos[ma] + c] = make_double2(0.5 * (zq.x + zn.x), 0.5 * (zq.y - zn.y));
    if (mb < lat) rhs[(int64_t)q * 4 * lat + 4 * pos[mb] + c] = make_double2(0.5 * (zq.y + zn.y), -0.5 * (zq.x - zn.x));
  }
}

__global__ void __launch_bounds__(kFftThreads) k_band_inv_fft(int nb, int lat, int nzl, int nq, FftPasses P,
                                                              const double2* __restrict__ tw,
                                                              const int* __restrict__ fpos,
                                                              const int* __restrict__ pos,
                                                              const double2* __restrict__ rhs,
                                                              double* __restrict__ v) {
  extern __shared__ double2 zs[];   // [kFftRows][nzl | 1]
  const int rs = nzl | 1;
  const int c = blockIdx.y, m0 = blockIdx.x * 2 * kFftRows;
  const int tid = threadIdx.x;
  const double2 zero = make_double2(0.0, 0.0);
  for (int e0 = tid; e0 < kFftRows * nq; e0 += 4 * kFftThreads) {
    double2 A[4], B[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * kFftThreads;
      A[u] = B[u] = zero;
      if (e < kFftRows * nq) {
        const int r = e / nq, q = e - r * nq;
        const int ma = m0 + 2 * r, mb = ma + 1;
        if (ma < lat) A[u] = rhs[(int64_t)q * 4 * lat + 4 * pos[ma] + c];
        if (mb < lat) B[u] = rhs[(int64_t)q * 4 * lat + 4 * pos[mb] + c];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * kFftThreads;
      if (e >= kFftRows * nq) break;
      const int r = e / nq, q = e - r * nq;
      const bool edge = q == 0 || 2 * q == nzl;
      if (edge) { A[u].y = 0.0; B[u].y = 0.0; }
      zs[r * rs + fpos[q]] = make_double2(A[u].x - B[u].y, A[u].y + B[u].x);
      if (!edge) zs[r * rs + fpos[nzl - q]] = make_double2(A[u].x + B[u].y, -A[u].y + B[u].x);
    }
  }
  __syncthreads();
  fft_rows_dit_inv<double, 16>(zs, kFftRows, rs, tw, P);
  const double inv = 1.0 / nzl;
  const int tot = 2 * kFftRows * nzl;
  for (int e = tid; e < tot; e += kFftThreads) {
    const int iz = e / (2 * kFftRows), mm = e % (2 * kFftRows);
    if (m0 + mm < lat)
      v[(int64_t)c * nb + m0 + mm + (int64_t)lat * iz] = inv * reinterpret_cast<const double*>(zs + (mm >> 1) * rs + iz)[mm & 1];
  }
}

// v[c nb + i1 + lat iz] = (1/nzl) sum_q w_q Re(rhs[q][..] exp(+2 pi i q iz / nzl)),
// w_q = 2 except q = 0 and q = nzl/2 (even nzl): the real inverse transform
// of a Hermitian spectrum.  A CTA takes 32 columns of one component and a
// run of kInvZ z rows; the columns' spectra (nq x 32) and the twiddles are
// staged in shared memory.
constexpr int kInvZ = 32;
__global__ void __launch_bounds__(256) k_band_inv(int nb, int lat, int nzl, int nq, const double* __restrict__ tw,
                                                  const int* __restrict__ pos, const double2* __restrict__ rhs,
                                                  double* __restrict__ v) {
  extern __shared__ double ism[];
  double2* xs = reinterpret_cast<double2*>(ism);   // [nq][32]
  double* twc = ism + 2 * 32 * nq;                 // [nzl]
  double* tws = twc + nzl;
  const int c = blockIdx.y;
  const int m0 = blockIdx.x * 32;
  const int z0 = blockIdx.z * kInvZ;
  const int tid = threadIdx.x;
  const int prow = (m0 + (tid & 31) < lat) ? 4 * pos[m0 + (tid & 31)] + c : 0;
  // eight loads in flight per thread before any store
  for (int e0 = tid; e0 < 32 * nq; e0 += 8 * 256) {
    double2 tv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * 256, q = e >> 5;
      tv[u] = (e < 32 * nq && m0 + (e & 31) < lat) ? rhs[(int64_t)q * 4 * lat + prow] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int e = e0 + u * 256, q = e >> 5;
      if (e < 32 * nq) {
        const double w = (q == 0 || 2 * q == nzl) ? 1.0 : 2.0;
        xs[e] = make_double2(w * tv[u].x, w * tv[u].y);
      }
    }
  }
  for (int e = tid; e < nzl; e += 256) { twc[e] = tw[e]; tws[e] = tw[nzl + e]; }
  __syncthreads();
  const int mm = tid & 31, zl = tid >> 5;
  if (m0 + mm >= lat) return;
  const double inv = 1.0 / nzl;
  for (int zz = zl; zz < kInvZ; zz += 8) {
    const int iz = z0 + zz;
    if (iz >= nzl) break;
    // two interleaved partial sums (even and odd q): half-length FMA chains
    double acc0 = 0.0, acc1 = 0.0;
    int k = 0;
    int q = 0;
    for (; q + 1 < nq; q += 2) {
      const double2 x0 = xs[q * 32 + mm], x1 = xs[(q + 1) * 32 + mm];
      int k1 = k + iz;
      if (k1 >= nzl) k1 -= nzl;
      acc0 += x0.x * twc[k] - x0.y * tws[k];
      acc1 += x1.x * twc[k1] - x1.y * tws[k1];
      k = k1 + iz;
      if (k >= nzl) k -= nzl;
    }
    if (q < nq) {
      const double2 x0 = xs[q * 32 + mm];
      acc0 += x0.x * twc[k] - x0.y * tws[k];
    }
    v[(int64_t)c * nb + m0 + mm + (int64_t)lat * iz] = (acc0 + acc1) * inv;
  }
}

// ---------------------------------------------------------------------------
// block-tridiagonal form.  In folded order every band entry couples positions
// at most 4 apart, so with blocks of 4 consecutive positions (16 rows: 4
// markers x 4 components) each system is block tridiagonal; a block LU
// without interchanges between blocks (Gauss-Jordan with partial pivoting
// inside each 16 x 16 diagonal block) makes the solve 2 x (4 len / 16)
// dependent block steps instead of 2 x 4 len scalar ones.
// ---------------------------------------------------------------------------
constexpr int kBs = 16;

__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

// scatter the band symbol into the sub-diagonal (A), diagonal (B) and
// super-diagonal (C) blocks; padding rows of the last block row get a unit
// diagonal (k_blk_pad)
__global__ void k_blk_assemble(int lat, int nq, int NBq, const int* __restrict__ nbr, const int* __restrict__ pos,
                               const int* __restrict__ seg, const int* __restrict__ segstart,
                               const int* __restrict__ blkoff, const double2* __restrict__ That,
                               double2* __restrict__ Ab, double2* __restrict__ Bb, double2* __restrict__ Cb) {
  const int nl = 80 * lat;
  const int64_t tot = (int64_t)nq * nl;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int L = (int)(t % nl);
    const int q = (int)(t / nl);
    const int c = L % 4;
    int r = L / 4;
    const int d = r % kNd; r /= kNd;
    const int i1 = r % lat;
    const int cp = r / lat;
    const int sg = seg[i1];
    const int base = 4 * segstart[sg];
    const int col = 4 * pos[i1] + c - base;
    const int row = 4 * pos[nbr[i1 * kNd + d]] + cp - base;
    const int bi = row / kBs, bj = col / kBs;
    const int64_t o = ((int64_t)q * NBq + blkoff[sg] + bi) * (kBs * kBs) + (row % kBs) * kBs + (col % kBs);
    double2* dst = bj < bi ? Ab : (bj == bi ? Bb : Cb);
    dst[o] = That[t];
  }
}

__global__ void k_blk_pad(int nq, int nseg, int NBq, const int* __restrict__ seglen, const int* __restrict__ nblk,
                          const int* __restrict__ blkoff, double2* __restrict__ Bb) {
  const int q = blockIdx.x / nseg, sg = blockIdx.x % nseg;
  const int m = 4 * seglen[sg];
  const int i = nblk[sg] - 1;
  const int64_t o = ((int64_t)q * NBq + blkoff[sg] + i) * (kBs * kBs);
  for (int rr = threadIdx.x; rr < kBs; rr += blockDim.x)
    if (kBs * i + rr >= m) Bb[o + rr * kBs + rr] = make_double2(1.0, 0.0);
}

// Block LU of one system by one warp: Delta_0 = B_0, Delta_i = B_i -
// A_i G_{i-1}, P_i = Delta_i^-1, G_i = P_i C_i, and Q_i = P_i A_i, which
// replaces A_i (the forward sweep is then y_i = P_i b_i - Q_i y_{i-1}: one
// dependent product per block row).  The block products run over the 256
// entries of a block in shared memory; the inverse is Gauss-Jordan with
// partial pivoting on [Delta_i | I] held by columns in registers (lane c < 16
// holds column c of Delta_i, lane 16 + c column c of the identity), a pivot
// row being marked used rather than swapped, so that row perm[k] ends as row
// k of the inverse.  A pivot below 1e-12 of the block's largest entry sets
// flag[1]: the caller then uses the pivoted banded LU instead.
__global__ void __launch_bounds__(32) k_blk_factor(int nseg, int NBq, const int* __restrict__ nblk,
                                                   const int* __restrict__ blkoff, double2* __restrict__ Ab,
                                                   const double2* __restrict__ Bb, const double2* __restrict__ Cb,
                                                   double2* __restrict__ Pb, double2* __restrict__ Gb,
                                                   int* __restrict__ flag) {
  // A_i, B_i, C_i of block row i arrive by bulk copies into buffer i & 1
  // while block row i - 1 is factored
  __shared__ __align__(128) double2 sIn[2][3][kBs * kBs];
  __shared__ double2 sP[kBs * kBs], sG[kBs * kBs], sD[kBs * kBs];
  __shared__ __align__(8) uint64_t bar[2];
  const int q = blockIdx.x / nseg, sg = blockIdx.x % nseg;
  const int N = nblk[sg];
  const int64_t b0 = ((int64_t)q * NBq + blkoff[sg]) * (kBs * kBs);
  const int lane = threadIdx.x, c = lane & 15;
  const bool left = lane < 16;
  const double2 zero = make_double2(0.0, 0.0);
  constexpr unsigned kBlkBytes = kBs * kBs * sizeof(double2);
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncwarp();
  auto fetch = [&](int i) {          // lane 0: block row i into buffer i & 1
    const int64_t o = b0 + (int64_t)i * kBs * kBs;
    uint64_t* b = &bar[i & 1];
    fence_async_shared();
    mbar_arrive_expect_tx(b, 3 * kBlkBytes);
    bulk_load(sIn[i & 1][0], Ab + o, kBlkBytes, b);
    bulk_load(sIn[i & 1][1], Bb + o, kBlkBytes, b);
    bulk_load(sIn[i & 1][2], Cb + o, kBlkBytes, b);
  };
  if (lane == 0) fetch(0);
  bool ok = true;
  for (int i = 0; i < N; ++i) {
    const int64_t o = b0 + (int64_t)i * kBs * kBs;
    if (!mbar_wait(&bar[i & 1], (unsigned)(i >> 1) & 1u, kWaitCycles)) ok = false;
    __syncwarp();
    if (lane == 0 && i + 1 < N) fetch(i + 1);
    const double2* sA = sIn[i & 1][0];
    const double2* sB = sIn[i & 1][1];
    const double2* sC = sIn[i & 1][2];
    // Delta_i = B_i - A_i G_{i-1} (eight entries per lane, interleaved)
#pragma unroll 4
    for (int e = lane; e < kBs * kBs; e += 32) {
      const int rr = e / kBs, cc = e % kBs;
      double2 d = sB[e];
      if (i > 0) {
        double2 a0 = zero, a1 = zero;
#pragma unroll
        for (int k = 0; k < kBs; k += 2) {
          a0 = cadd(a0, cmul(sA[rr * kBs + k], sG[k * kBs + cc]));
          a1 = cadd(a1, cmul(sA[rr * kBs + k + 1], sG[(k + 1) * kBs + cc]));
        }
        d = csub(d, cadd(a0, a1));
      }
      sD[e] = d;
    }
    __syncwarp();
    double2 col[kBs];
#pragma unroll
    for (int rr = 0; rr < kBs; ++rr)
      col[rr] = left ? sD[rr * kBs + c] : make_double2(rr == c ? 1.0 : 0.0, 0.0);
    // largest entry of Delta_i (the small-pivot test)
    double dmax = 0.0;
    if (left)
#pragma unroll
      for (int rr = 0; rr < kBs; ++rr) dmax = fmax(dmax, cabs1(col[rr]));
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, s));
    unsigned used = 0;
    unsigned long long perm = 0;       // 4 bits per pivot step: the row it took
#pragma unroll 1
    for (int k = 0; k < kBs; ++k) {
      // pivot of column k (lane k): the largest unused row, lowest index on
      // ties, by a tournament over the 16 rows (depth 4)
      double tv[kBs];
      int ti[kBs];
#pragma unroll
      for (int rr = 0; rr < kBs; ++rr) {
        tv[rr] = ((used >> rr) & 1u) ? -1.0 : cabs1(col[rr]);
        ti[rr] = rr;
      }
#pragma unroll
      for (int w = 1; w < kBs; w *= 2)
#pragma unroll
        for (int rr = 0; rr < kBs; rr += 2 * w)
          if (tv[rr + w] > tv[rr]) { tv[rr] = tv[rr + w]; ti[rr] = ti[rr + w]; }
      const double best = tv[0];
      const int bp = ti[0];
      const int p = __shfl_sync(0xffffffffu, bp, k);
      const double bk = __shfl_sync(0xffffffffu, best, k);
      if (lane == 0 && !(bk > 1e-12 * dmax)) atomicExch(flag + 1, 1);
      double2 mine = zero;             // this lane's entry of the pivot row
#pragma unroll
      for (int rr = 0; rr < kBs; ++rr)
        if (rr == p) mine = col[rr];
      double2 pv;
      pv.x = __shfl_sync(0xffffffffu, mine.x, k);
      pv.y = __shfl_sync(0xffffffffu, mine.y, k);
      const double2 rp = cabs1(pv) > 0.0 ? crcp(pv) : zero;
      const double2 vp = cmul(mine, rp);
#pragma unroll
      for (int rr = 0; rr < kBs; ++rr) {
        double2 m;
        m.x = __shfl_sync(0xffffffffu, col[rr].x, k);
        m.y = __shfl_sync(0xffffffffu, col[rr].y, k);
        col[rr] = (rr == p) ? vp : csub(col[rr], cmul(m, vp));
      }
      used |= 1u << p;
      perm |= (unsigned long long)p << (4 * k);
    }
    // P_i: row k of the inverse is row perm[k] of the right half
    if (!left) {
#pragma unroll 1
      for (int k = 0; k < kBs; ++k) {
        const int pk = (int)((perm >> (4 * k)) & 15u);
        double2 v = zero;
#pragma unroll
        for (int rr = 0; rr < kBs; ++rr)
          if (rr == pk) v = col[rr];
        sP[k * kBs + c] = v;
        Pb[o + k * kBs + c] = v;
      }
    }
    __syncwarp();
    // G_i = P_i C_i (kept for the next block row) and Q_i = P_i A_i
#pragma unroll 4
    for (int e = lane; e < 2 * kBs * kBs; e += 32) {
      const bool isg = e < kBs * kBs;
      const int f = isg ? e : e - kBs * kBs;
      const int rr = f / kBs, cc = f % kBs;
      if (isg ? (i + 1 >= N) : (i == 0)) continue;
      const double2* R = isg ? sC : sA;
      double2 a0 = zero, a1 = zero;
#pragma unroll
      for (int k = 0; k < kBs; k += 2) {
        a0 = cadd(a0, cmul(sP[rr * kBs + k], R[k * kBs + cc]));
        a1 = cadd(a1, cmul(sP[rr * kBs + k + 1], R[(k + 1) * kBs + cc]));
      }
      const double2 acc = cadd(a0, a1);
      if (isg) Gb[o + f] = acc;
      else Ab[o + f] = acc;
      if (isg) sD[f] = acc;            // staged; copied to sG below
    }
    __syncwarp();
    for (int e = lane; e < kBs * kBs; e += 32) sG[e] = sD[e];
    __syncwarp();
  }
  if (!ok && lane == 0) atomicOr(flag + 3, 1);
}

// Block forward and back substitution of one system by one CTA of four
// warps: thread (r, p) = (tid / 8, tid % 8) forms the terms of columns p and
// p + 8 of row r of each 16 x 16 product (a quarter warp reads 128
// consecutive bytes of a block row: no bank conflicts), eight threads add
// them by shuffles, and one barrier per block row publishes the new 16-vector
// (double-buffered).  The blocks stream through a shared-memory ring of bulk
// copies (kBlkRing - 1 block rows ahead, issued by thread 0), and the
// system's right-hand side and solution sit in shared memory for the whole
// solve.
constexpr int kBlkRing = 16;    // one 16x16 block per stage: 15 blocks (60 KB) in flight
constexpr int kBlkThreads = 128;
static size_t blk_solve_smem(int nmax) {
  return sizeof(double2) * ((size_t)kBlkRing * kBs * kBs + 2 * (size_t)kBs * nmax);
}
__global__ void __launch_bounds__(kBlkThreads) k_blk_solve(int lat, int nseg, int NBq,
                                                           const int* __restrict__ segstart,
                                                           const int* __restrict__ seglen,
                                                           const int* __restrict__ nblk,
                                                           const int* __restrict__ blkoff,
                                                           const double2* __restrict__ Ab,
                                                           const double2* __restrict__ Pb,
                                                           const double2* __restrict__ Gb,
                                                           double2* __restrict__ rhs, int* __restrict__ flag);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(kBlkThreads) k_blk_solve(int lat, int nseg, int NBq,
                                                           const int* __restrict__ segstart,
                                                           const int* __restrict__ seglen,
                                                           const int* __restrict__ nblk,
                                                           const int* __restrict__ blkoff,
                                                           const double2* __restrict__ Ab,
                                                           const double2* __restrict__ Pb,
                                                           const double2* __restrict__ Gb,
                                                           double2* __restrict__ rhs, int* __restrict__ flag) {
  extern __shared__ __align__(128) double2 bs_smem[];
  double2 (*ring)[kBs * kBs] = reinterpret_cast<double2 (*)[kBs * kBs]>(bs_smem);
  const int q = blockIdx.x / nseg, sg = blockIdx.x % nseg;
  const int N = nblk[sg];
  const int m = 4 * seglen[sg];
  double2* xs = bs_smem + (size_t)kBlkRing * kBs * kBs;   // [kBs * N] right-hand side b
  double2* ys = xs + (size_t)kBs * N;                     // [kBs * N] t, then y, then x
  __shared__ double2 vv[2][kBs];
  __shared__ __align__(8) uint64_t bar[kBlkRing];
  const int64_t b0 = ((int64_t)q * NBq + blkoff[sg]) * (kBs * kBs);
  double2* x = rhs + (int64_t)q * 4 * lat + 4 * segstart[sg];
  const int tid = threadIdx.x;
  const int r = tid >> 3, pp = tid & 7;
  const double2 zero = make_double2(0.0, 0.0);
  if (tid == 0) {
    for (int k = 0; k < kBlkRing; ++k) mbar_init(&bar[k], 1);
    fence_mbar_init();
  }
  for (int e0 = tid; e0 < kBs * N; e0 += 4 * kBlkThreads) {   // four loads in flight
    double2 tv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + kBlkThreads * u;
      tv[u] = e < m ? x[e] : zero;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (e0 + kBlkThreads * u < kBs * N) xs[e0 + kBlkThreads * u] = tv[u];
  }
  __syncthreads();
  // `used` counts the blocks consumed (uniform across the CTA); slot and
  // phase follow from it.
  unsigned used = 0;
  bool ok = true;
  constexpr unsigned kBlkBytes = kBs * kBs * sizeof(double2);
  auto blk = [&](const double2* base, int i) { return base + b0 + (int64_t)i * kBs * kBs; };
  // The three passes consume one sequence of blocks, g = 0 .. 3N-3: P_0 ..
  // P_{N-1}, then Q_1 .. Q_{N-1}, then G_{N-2} .. G_0; block g goes to slot
  // g % kBlkRing.  The first kBlkRing are issued at g = 0, and at every
  // g = 4, 8, ... the four blocks g+12 .. g+15, into the slots of g-4 .. g-1,
  // which the barriers of their block rows have released (one proxy fence
  // per group), so each pass's first blocks arrive during the previous one.
  const int total = 3 * N - 2;
  auto src = [&](int g) -> const double2* {
    if (g < N) return blk(Pb, g);
    if (g < 2 * N - 1) return blk(Ab, g - N + 1);
    return blk(Gb, N - 2 - (g - (2 * N - 1)));
  };
  auto refill = [&](int g) {
    const int lo = g == 0 ? 0 : g + kBlkRing - 4, hi = min(total, g + kBlkRing);
    if (tid == 0 && lo < hi) {
      fence_async_shared();            // the CTA's reads of the slots come first
      for (int k = lo; k < hi; ++k) {
        const unsigned slot = (unsigned)k % kBlkRing;
        mbar_arrive_expect_tx(&bar[slot], kBlkBytes);
        bulk_load(ring[slot], src(k), kBlkBytes, &bar[slot]);
      }
    }
  };
  auto acquire = [&]() -> const double2* {
    const unsigned slot = used % kBlkRing;
    if (!mbar_wait(&bar[slot], (used / kBlkRing) & 1u, kWaitCycles)) ok = false;
    ++used;
    return ring[slot];
  };
  // row r of M times v: columns pp and pp + 8 here, the other six pairs in
  // the seven neighbouring threads (shuffle sum over the group of eight)
  auto rowdot = [&](const double2* M, const double2* v) {
    const double2 p0 = M[r * kBs + pp], y0 = v[pp];
    const double2 p1 = M[r * kBs + pp + 8], y1 = v[pp + 8];
    double2 a;
    a.x = p0.x * y0.x - p0.y * y0.y;
    a.y = p0.x * y0.y + p0.y * y0.x;
    a.x = fma(p1.x, y1.x, fma(-p1.y, y1.y, a.x));
    a.y = fma(p1.x, y1.y, fma(p1.y, y1.x, a.y));
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
      a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
    }
    return a;
  };
  // t_i = P_i b_i for every block row (independent products): four block
  // rows per step, one per warp; lane (r2, hh) forms half (eight terms, in a
  // row-rotated order) of row r2.  P_i is block g = i of the sequence.
  {
    const int warp = tid >> 5, lane = tid & 31, r2 = lane & 15, hh = lane >> 4;
    for (int s4 = 0; s4 < N; s4 += 4) {
      refill(s4);
      const int i = s4 + warp;
      if (i < N) {
        if (!mbar_wait(&bar[i % kBlkRing], (unsigned)(i / kBlkRing) & 1u, kWaitCycles)) ok = false;
        const double2* Pi = ring[i % kBlkRing];
        const double2* v = xs + kBs * i;
        double2 a0 = zero, a1 = zero;
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
          const int k0 = (k + r2) & 7, k1 = (k + 1 + r2) & 7;
          const double2 p0 = Pi[r2 * kBs + 8 * hh + k0], y0 = v[8 * hh + k0];
          const double2 p1 = Pi[r2 * kBs + 8 * hh + k1], y1 = v[8 * hh + k1];
          a0.x += p0.x * y0.x - p0.y * y0.y;
          a0.y += p0.x * y0.y + p0.y * y0.x;
          a1.x += p1.x * y1.x - p1.y * y1.y;
          a1.y += p1.x * y1.y + p1.y * y1.x;
        }
        a0.x += a1.x;
        a0.y += a1.y;
        a0.x += __shfl_xor_sync(0xffffffffu, a0.x, 16);
        a0.y += __shfl_xor_sync(0xffffffffu, a0.y, 16);
        if (hh == 0) ys[kBs * i + r2] = a0;
      }
      __syncthreads();
    }
    used = (unsigned)N;
  }
  // forward: y_i = t_i - Q_i y_{i-1} (Q_i = P_i A_i, stored in place of A_i);
  // vv[i & 1] carries y_i to the next block row
  for (int i = 0; i < N; ++i) {
    if (i > 0 && ((N + i - 1) & 3) == 0) refill(N + i - 1);
    const int row = kBs * i + r;
    double2 y = ys[row];
    if (i > 0) {
      const double2* Qi = acquire();
      y = csub(y, rowdot(Qi, vv[(i - 1) & 1]));
    }
    if (pp == 0) {
      vv[i & 1][r] = y;
      ys[row] = y;
    }
    __syncthreads();
  }
  // backward: x_i = y_i - G_i x_{i+1}; vv[(i + 1) & 1] holds x_{i+1}
  for (int i = N - 2; i >= 0; --i) {
    if (((3 * N - 3 - i) & 3) == 0) refill(3 * N - 3 - i);
    const double2* Gi = acquire();
    const double2 a = rowdot(Gi, vv[(i + 1) & 1]);
    const int row = kBs * i + r;
    if (pp == 0) {
      const double2 xr = csub(ys[row], a);
      vv[i & 1][r] = xr;
      ys[row] = xr;
    }
    __syncthreads();
  }
  for (int e = tid; e < m; e += kBlkThreads) x[e] = ys[e];
  if (!ok && tid == 0) atomicOr(flag + 3, 1);
}

// Forward and back substitution of one system (LAPACK zgbtrs, no transpose)
// by one warp.  The substitutions are sequential in the row index, so the
// entries they are working on stay in registers: in the forward pass lane p
// holds b[i] for the 32 rows i = j .. j+31 with i = p (mod 32) (the kl = 19
// rows a step updates are inside), in the backward pass two registers per
// lane hold the 64 rows j-63 .. j (the kv = 38 rows above the diagonal are
// inside).  A step is one shuffle (the pivot value to every lane, plus two
// for a row interchange) and a complex multiply-add per lane; the lane that
// finishes a row stores it and loads the row 32 (64) further on.  The band
// columns are streamed through a shared-memory ring of kSolveRing chunks of
// kSolveChunk columns (cp.async, seven chunks ahead).
__global__ void __launch_bounds__(32) k_band_solve(int lat, int nseg, const int* __restrict__ segstart,
                                                   const int* __restrict__ seglen, const double2* __restrict__ AB,
                                                   const int* __restrict__ ipiv, double2* __restrict__ rhs) {
  extern __shared__ double2 sm[];
  double2* buf = sm;                                           // [kSolveRing][kSolveChunk][kLdab]
  double2* b = sm + kSolveRing * kSolveChunk * kLdab;          // [m]
  int* spiv = reinterpret_cast<int*>(b + 4 * lat);             // [m] (m <= 4 lat)
  const int q = blockIdx.x / nseg, s = blockIdx.x % nseg;
  const int m = 4 * seglen[s];
  const int base = 4 * segstart[s];
  const double2* A = AB + (int64_t)q * kLdab * 4 * lat + (int64_t)kLdab * base;
  const int* piv = ipiv + (int64_t)q * 4 * lat + base;
  double2* x = rhs + (int64_t)q * 4 * lat + base;
  const int lane = threadIdx.x;
  const double2 zero = make_double2(0.0, 0.0);
  for (int e = lane; e < m; e += 32) { b[e] = x[e]; spiv[e] = piv[e]; }
  const int nch = (m + kSolveChunk - 1) / kSolveChunk;
  auto load_chunk = [&](int ch) {
    if (ch >= 0 && ch < nch) {
      const int c0 = ch * kSolveChunk;
      const int nc = min(kSolveChunk, m - c0);
      const double2* src = A + (int64_t)c0 * kLdab;
      double2* dst = buf + (ch % kSolveRing) * kSolveChunk * kLdab;
      for (int e = lane; e < nc * kLdab; e += 32) cp_async16(dst + e, src + e);
    }
    cp_async_commit();
  };
  auto shfl2 = [](double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
  };
  // ---- forward: b := L^-1 P b
  for (int c = 0; c < kSolveRing - 1; ++c) load_chunk(c);
  __syncwarp();
  double2 w = lane < m ? b[lane] : zero;       // row lane (rows i = p mod 32 in the window)
  for (int ch = 0; ch < nch; ++ch) {
    load_chunk(ch + kSolveRing - 1);
    cp_async_wait<kSolveRing - 1>();
    __syncwarp();
    const double2* cb = buf + (ch % kSolveRing) * kSolveChunk * kLdab;
    const int c0 = ch * kSolveChunk;
    const int nc = min(kSolveChunk, m - c0);
    for (int jj = 0; jj < nc; ++jj) {
      const int j = c0 + jj;
      const int pj = j & 31;
      if (j < m - 1) {
        const int lm = min(kKl, m - 1 - j);
        // this lane's row i = j + t with t in 1..31 (t = 0 is the pivot row)
        const int t = (lane - pj) & 31;
        const double2 lv = (t >= 1 && t <= lm) ? cb[jj * kLdab + kKv + t] : zero;
        const int l = spiv[j] - j;              // row interchange with row j + l
        if (l != 0) {
          const int pl = (pj + l) & 31;
          const double2 vj = shfl2(w, pj), vl = shfl2(w, pl);
          if (lane == pj) w = vl;
          if (lane == pl) w = vj;
        }
        const double2 bj = shfl2(w, pj);
        if (t >= 1 && t <= lm) w = csub(w, cmul(lv, bj));
      }
      // row j is final: store it, take row j + 32
      if (lane == pj) {
        b[j] = w;
        w = (j + 32 < m) ? b[j + 32] : zero;
      }
    }
  }
  cp_async_wait<0>();
  __syncwarp();
  // ---- backward: b := U^-1 b (the stored diagonal is the reciprocal); row
  // i lives in lane i mod 32, register (i / 32) mod 2, for the 64 rows
  // j-63 .. j
  for (int k = 0; k < kSolveRing - 1; ++k) load_chunk(nch - 1 - k);
  double2 w0 = zero, w1 = zero;
  for (int i = lane; i < m; i += 32)
    if (i >= m - 64) {
      if (((i >> 5) & 1) == 0) w0 = b[i]; else w1 = b[i];
    }
  __syncwarp();
  for (int k = 0; k < nch; ++k) {
    const int ch = nch - 1 - k;
    load_chunk(ch - (kSolveRing - 1));
    cp_async_wait<kSolveRing - 1>();
    __syncwarp();
    const double2* cb = buf + (ch % kSolveRing) * kSolveChunk * kLdab;
    const int c0 = ch * kSolveChunk;
    const int nc = min(kSolveChunk, m - c0);
    for (int jj = nc - 1; jj >= 0; --jj) {
      const int j = c0 + jj;
      const double2* col = cb + jj * kLdab;
      const int pj = j & 31;
      // this lane's rows: ia = the largest i <= j with i = lane (mod 32), ib = ia - 32
      const int ta = (j - lane) & 31;             // j - ia, 0..31
      const int ia = j - ta, ib = ia - 32;
      const bool a0 = ((ia >> 5) & 1) == 0;       // ia's register (meaningful for ia >= 0)
      double2 va = a0 ? w0 : w1, vb = a0 ? w1 : w0;
      const double2 ua = (ta >= 1) ? col[kKv - ta] : zero;            // ta <= 31 < kKv
      const double2 ub = (ta + 32 <= kKv) ? col[kKv - ta - 32] : zero;
      if (ta == 0) va = cmul(va, col[kKv]);      // lane pj: row j divided by its pivot
      const double2 bj = shfl2(va, pj);
      if (ta >= 1 && ia >= 0) va = csub(va, cmul(ua, bj));
      if (ta + 32 <= kKv && ib >= 0) vb = csub(vb, cmul(ub, bj));
      if (ta == 0) {                              // row j is final: store it, take row j - 64
        b[j] = va;
        va = (j - 64 >= 0) ? b[j - 64] : zero;
      }
      w0 = a0 ? va : vb;
      w1 = a0 ? vb : va;
    }
  }
  cp_async_wait<0>();
  __syncwarp();
  for (int e = lane; e < m; e += 32) x[e] = b[e];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// Segments of the marker lattice along its first direction, by body type:
// each is a closed ring (a periodic wall row, a cylinder's circumference).
// The band form needs geometry that repeats along z; the wall plates do not.
static bool lattice_segments(const IbState* s, const Params& p, std::vector<int>& start, std::vector<int>& len) {
  start.clear();
  len.clear();
  const std::string& k = s->kind;
  const int lat = s->lat_nx;
  if (k == "center_wall" || k == "wall_standing_wave") {
    start = {0};
    len = {lat};
  } else if (k == "standing_wave" || k == "traveling_wave_x" || k == "two_cylinders_z") {
    if (lat % 2) return false;
    start = {0, lat / 2};
    len = {lat / 2, lat / 2};
  } else if (k == "double_cylinders_z") {
    // each row holds the inner ring's nxb1 markers (body 0), then the outer
    // ring's (src/immersed_boundary_geometry.f90:117-174)
    int n1 = 0;
    for (int i = 0; i < lat; ++i)
      if (s->body[i] == 0) ++n1;
    if (n1 <= 0 || n1 >= lat) return false;
    start = {0, n1};
    len = {n1, lat - n1};
  } else {
    return false;
  }
  (void)p;
  for (int l : len)
    if (l < 5) return false;
  return true;
}

// shared memory of the solve: the band ring, the right-hand side and the pivots
static size_t solve_smem_bytes(int lat) {
  return sizeof(double2) * ((size_t)kSolveRing * kSolveChunk * kLdab + 4 * (size_t)lat) + sizeof(int) * 4 * (size_t)lat;
}

static size_t fwd_smem_bytes(int nzl) { return sizeof(double) * (32 * (size_t)nzl + 2 * (size_t)nzl); }
static size_t inv_smem_bytes(int nzl, int nq) { return sizeof(double) * (64 * (size_t)nq + 2 * (size_t)nzl); }

static int band_setup(Handle* h) {
  IbState* s = h->ib;
  if (s->band) return 0;
  BandState* B = new BandState();
  s->band = B;
  B->ok = lattice_segments(s, h->p, B->seg_start, B->seg_len);
  if (!B->ok) return 0;
  const int lat = s->lat_nx;
  B->lat = lat;
  B->nzl = s->nb / lat;
  B->nq = B->nzl / 2 + 1;
  B->nseg = (int)B->seg_start.size();
  if (B->nzl * lat != s->nb || solve_smem_bytes(lat) > 220 * 1024 || fwd_smem_bytes(B->nzl) > 220 * 1024) {
    B->ok = false;
    return 0;
  }
  // folded positions, neighbours, colours
  std::vector<int> pos(lat), seg(lat), nbr((size_t)lat * kNd), col((size_t)4 * lat);
  for (int sgi = 0; sgi < B->nseg; ++sgi) {
    const int st = B->seg_start[sgi], n = B->seg_len[sgi];
    const int half = (n + 1) / 2;
    for (int i = 0; i < n; ++i) {
      const int fp = i < half ? 2 * i : 2 * (n - 1 - i) + 1;
      pos[st + i] = st + fp;
      seg[st + i] = sgi;
      for (int d = -kKb; d <= kKb; ++d) nbr[(size_t)(st + i) * kNd + d + kKb] = st + ((i + d) % n + n) % n;
    }
  }
  // the folded order keeps every band entry within kKl of the diagonal
  for (int i = 0; i < lat; ++i)
    for (int d = 0; d < kNd; ++d)
      if (std::abs(pos[nbr[(size_t)i * kNd + d]] - pos[i]) > 2 * kKb) {
        B->ok = false;
        return 0;
      }
  B->colours.assign(4, {});
  for (int c = 0; c < 4; ++c) {
    const int P = B->spacing[c];
    std::vector<char> used(2 * P + 1, 0);
    for (int sgi = 0; sgi < B->nseg; ++sgi) {
      const int st = B->seg_start[sgi], n = B->seg_len[sgi];
      const int full = (n / P) * P;
      for (int i = 0; i < n; ++i) {
        // full groups of P share P colours (members P apart, also across the
        // ring's closure); the remainder markers get colours of their own
        const int k = i < full ? i % P : P + (i - full);
        col[(size_t)c * lat + st + i] = k;
        used[k] = 1;
      }
    }
    for (int k = 0; k < (int)used.size(); ++k)
      if (used[k]) B->colours[c].push_back(k);
  }
  const int nzl = B->nzl, nq = B->nq;
  int rc;
  if ((rc = dev_alloc(h, &B->nbr_d, (int64_t)lat * kNd))) return rc;
  if ((rc = dev_alloc(h, &B->pos_d, lat))) return rc;
  if ((rc = dev_alloc(h, &B->seg_d, lat))) return rc;
  if ((rc = dev_alloc(h, &B->segstart_d, B->nseg))) return rc;
  if ((rc = dev_alloc(h, &B->seglen_d, B->nseg))) return rc;
  if ((rc = dev_alloc(h, &B->colour_d, 4 * (int64_t)lat))) return rc;
  if ((rc = dev_alloc(h, &B->T_d, (int64_t)nzl * 80 * lat))) return rc;
  if ((rc = dev_alloc(h, &B->That_d, (int64_t)nq * 80 * lat))) return rc;
  if ((rc = dev_alloc(h, &B->AB_d, (int64_t)nq * kLdab * 4 * lat))) return rc;
  if ((rc = dev_alloc(h, &B->ipiv_d, (int64_t)nq * 4 * lat))) return rc;
  if ((rc = dev_alloc(h, &B->rhs_d, (int64_t)nq * 4 * lat))) return rc;
  B->nblk.resize(B->nseg);
  B->blkoff.resize(B->nseg);
  B->NBq = 0;
  B->nblk_max = 0;
  for (int sgi = 0; sgi < B->nseg; ++sgi) {
    B->nblk[sgi] = (4 * B->seg_len[sgi] + kBs - 1) / kBs;
    B->blkoff[sgi] = B->NBq;
    B->NBq += B->nblk[sgi];
    B->nblk_max = std::max(B->nblk_max, B->nblk[sgi]);
  }
  if (blk_solve_smem(B->nblk_max) > 200 * 1024) {
    h->last_error = "band preconditioner: a lattice segment is too long for the block solve";
    return C3D_ERR_UNSUPPORTED;
  }
  const int64_t nbe = (int64_t)nq * B->NBq * kBs * kBs;
  if ((rc = dev_alloc(h, &B->nblk_d, B->nseg))) return rc;
  if ((rc = dev_alloc(h, &B->blkoff_d, B->nseg))) return rc;
  if ((rc = dev_alloc(h, &B->Ab_d, nbe))) return rc;
  if ((rc = dev_alloc(h, &B->Bb_d, nbe))) return rc;
  if ((rc = dev_alloc(h, &B->Cb_d, nbe))) return rc;
  if ((rc = dev_alloc(h, &B->Pb_d, nbe))) return rc;
  if ((rc = dev_alloc(h, &B->Gb_d, nbe))) return rc;
  if ((rc = dev_alloc(h, &B->tw_d, 2 * (int64_t)nzl))) return rc;
  if ((rc = dev_alloc(h, &B->flag_d, 4))) return rc;
  B->fft = make_fft_passes(nzl, B->fftP, 16) && fft_smem_bytes(nzl) <= 48 * 1024;
  std::vector<double2> ftw;
  std::vector<int> fpos;
  if (B->fft) {
    if ((rc = dev_alloc(h, &B->ftw_d, nzl))) return rc;
    if ((rc = dev_alloc(h, &B->fpos_d, nzl))) return rc;
    ftw.resize(nzl);
    fpos.resize(nzl);
    for (int m = 0; m < nzl; ++m) {
      const long double a = -2.0L * 3.141592653589793238462643383279503L * (long double)m / (long double)nzl;
      ftw[m] = make_double2((double)std::cos(a), (double)std::sin(a));
      fpos[m] = dif_k_to_position(m, B->fftP);
    }
  }
  std::vector<double> tw(2 * (size_t)nzl);
  for (int k = 0; k < nzl; ++k) {
    const long double a = 2.0L * 3.141592653589793238462643383279503L * (long double)k / (long double)nzl;
    tw[k] = (double)std::cos(a);
    tw[nzl + k] = (double)std::sin(a);
  }
  cudaStream_t st = h->stream;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->nbr_d, nbr.data(), 4 * nbr.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->pos_d, pos.data(), 4 * pos.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->seg_d, seg.data(), 4 * seg.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->segstart_d, B->seg_start.data(), 4 * B->nseg, cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->seglen_d, B->seg_len.data(), 4 * B->nseg, cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->colour_d, col.data(), 4 * col.size(), cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->tw_d, tw.data(), 8 * tw.size(), cudaMemcpyHostToDevice, st));
  if (B->fft) {
    C3D_CUDA_TRY(h, cudaMemcpyAsync(B->ftw_d, ftw.data(), sizeof(double2) * nzl, cudaMemcpyHostToDevice, st));
    C3D_CUDA_TRY(h, cudaMemcpyAsync(B->fpos_d, fpos.data(), sizeof(int) * nzl, cudaMemcpyHostToDevice, st));
  }
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->nblk_d, B->nblk.data(), 4 * B->nseg, cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(B->blkoff_d, B->blkoff.data(), 4 * B->nseg, cudaMemcpyHostToDevice, st));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(st));
  const size_t solve_smem = solve_smem_bytes(lat);
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_band_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solve_smem));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_band_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fwd_smem_bytes(nzl)));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_band_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)inv_smem_bytes(nzl, nq)));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_band_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(double2) * kFactorWin * kLdab)));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_blk_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)blk_solve_smem(B->nblk_max)));
  return 0;
}

bool band_supported(Handle* h) {
  IbState* s = h->ib;
  if (!s) return false;
  if (band_setup(h)) return false;
  return s->band && s->band->ok;
}

// Factor the band systems from the symbol in That: the block-tridiagonal
// LU, or, when one of its diagonal blocks has a pivot below 1e-12 of the
// block's largest entry, the banded LU with partial pivoting.
static int band_factor_that(Handle* h) {
  IbState* s = h->ib;
  BandState* B = s->band;
  const int lat = B->lat, nq = B->nq;
  const unsigned gb = 148 * 8;
  const size_t nbe = sizeof(double2) * (size_t)nq * B->NBq * kBs * kBs;
  C3D_CUDA_TRY(h, cudaMemsetAsync(B->Ab_d, 0, nbe, h->stream));
  C3D_CUDA_TRY(h, cudaMemsetAsync(B->Bb_d, 0, nbe, h->stream));
  C3D_CUDA_TRY(h, cudaMemsetAsync(B->Cb_d, 0, nbe, h->stream));
  k_blk_assemble<<<gb, 256, 0, h->stream>>>(lat, nq, B->NBq, B->nbr_d, B->pos_d, B->seg_d, B->segstart_d,
                                            B->blkoff_d, B->That_d, B->Ab_d, B->Bb_d, B->Cb_d);
  C3D_LAUNCH_CHECK(h);
  k_blk_pad<<<nq * B->nseg, 32, 0, h->stream>>>(nq, B->nseg, B->NBq, B->seglen_d, B->nblk_d, B->blkoff_d, B->Bb_d);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemsetAsync(B->flag_d, 0, 8, h->stream));
  k_blk_factor<<<nq * B->nseg, 32, 0, h->stream>>>(B->nseg, B->NBq, B->nblk_d, B->blkoff_d, B->Ab_d, B->Bb_d,
                                                   B->Cb_d, B->Pb_d, B->Gb_d, B->flag_d);
  C3D_LAUNCH_CHECK(h);
  int flag[2] = {0, 0};
  C3D_CUDA_TRY(h, cudaMemcpyAsync(flag, B->flag_d, 8, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  B->block = flag[1] == 0;
  if (B->block) return 0;
  // pivoted banded LU
  C3D_CUDA_TRY(h, cudaMemsetAsync(B->AB_d, 0, sizeof(double2) * (size_t)nq * kLdab * 4 * lat, h->stream));
  k_band_assemble<<<gb, 256, 0, h->stream>>>(lat, nq, B->nbr_d, B->pos_d, B->seg_d, B->segstart_d, B->That_d,
                                             B->AB_d);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemsetAsync(B->flag_d, 0, 4, h->stream));
  k_band_factor<<<nq * B->nseg, 256, sizeof(double2) * kFactorWin * kLdab, h->stream>>>(
      lat, B->nseg, B->segstart_d, B->seglen_d, B->AB_d, B->ipiv_d, B->flag_d);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(flag, B->flag_d, 4, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (flag[0]) { h->last_error = "band preconditioner: singular band system"; return C3D_ERR_NAN; }
  return 0;
}

// factor the band systems from the entries in T_d
static int band_factor_from_T(Handle* h) {
  IbState* s = h->ib;
  BandState* B = s->band;
  const int lat = B->lat, nzl = B->nzl, nq = B->nq, nl = 80 * lat;
  const unsigned gb = 148 * 8;
  k_band_dft_T<<<gb, 256, 0, h->stream>>>(nl, nzl, nq, B->tw_d, B->T_d, B->That_d);
  C3D_LAUNCH_CHECK(h);
  return band_factor_that(h);
}

// Probe the band of S at the current geometry and factor it.
int band_build(Handle* h, double dt) {
  IbState* s = h->ib;
  if (!band_supported(h)) { h->last_error = "band preconditioner: unsupported marker lattice"; return C3D_ERR_UNSUPPORTED; }
  BandState* B = s->band;
  const int nb = s->nb, lat = B->lat, nzl = B->nzl;
  const int64_t n = 4 * (int64_t)nb;
  int rc;
  if (s->prb == nullptr && (rc = dev_alloc(h, &s->prb, 4 * n))) return rc;
  double* probe = s->prb;
  double* resp = s->prb + n;
  const unsigned gb = 148 * 8;
  for (int c = 0; c < 4; ++c)
    for (int colour : B->colours[c]) {
      k_band_probe<<<gb, 256, 0, h->stream>>>(nb, lat, c, colour, B->colour_d, probe);
      C3D_LAUNCH_CHECK(h);
      if ((rc = ib_schur(h, probe, resp, dt))) return rc;
      k_band_extract<<<gb, 256, 0, h->stream>>>(nb, lat, nzl, c, colour, B->colour_d, B->nbr_d, resp, B->T_d);
      C3D_LAUNCH_CHECK(h);
      B->probes++;
    }
  if ((rc = band_factor_from_T(h))) return rc;
  s->have_lrn = false;                 // the factors in use are the probed band's now
  B->built = true;
  B->yb_at = s->yb;
  B->xb_at = s->xb;
  B->dt_at = dt;
  B->builds++;
  h->stats.precond_builds++;
  return 0;
}

// The factors are rebuilt when dt changed or a marker moved by more than
// 0.03 dymin since they were probed (about ten time steps of the cfg2 wave at
// its fastest; a preconditioner 30 steps old no longer converges there).
bool band_stale(Handle* h, double dt) {
  IbState* s = h->ib;
  BandState* B = s->band;
  if (!B || !B->built || B->dt_at != dt || B->yb_at.size() != s->yb.size()) return true;
  double mx = 0.0;
  for (size_t k = 0; k < s->yb.size(); ++k) {
    mx = std::max(mx, std::fabs(s->yb[k] - B->yb_at[k]));
    mx = std::max(mx, std::fabs(s->xb[k] - B->xb_at[k]));
  }
  return mx > 0.03 * h->dymin;
}

void band_invalidate(Handle* h) {
  if (h->ib && h->ib->band) h->ib->band->built = false;
}

// out = B^-1 in
int band_apply(Handle* h, const double* in, double* out) {
  IbState* s = h->ib;
  BandState* B = s->band;
  const int lat = B->lat, nzl = B->nzl, nq = B->nq, nb = s->nb;
  const unsigned nmc = (unsigned)((lat + 31) / 32);
  const unsigned nfc = (unsigned)((lat + 2 * kFftRows - 1) / (2 * kFftRows));
  if (B->fft)
    k_band_fwd_fft<<<dim3(nfc, 4), kFftThreads, fft_smem_bytes(nzl), h->stream>>>(
        nb, lat, nzl, nq, B->fftP, B->ftw_d, B->fpos_d, B->pos_d, in, B->rhs_d);
  else
    k_band_fwd<<<dim3(nmc, 4, (unsigned)((nq + kFwdQ - 1) / kFwdQ)), 256, fwd_smem_bytes(nzl), h->stream>>>(
        nb, lat, nzl, nq, B->tw_d, B->pos_d, in, B->rhs_d);
  C3D_LAUNCH_CHECK(h);
  if (B->block) {
    k_blk_solve<<<nq * B->nseg, kBlkThreads, blk_solve_smem(B->nblk_max), h->stream>>>(
        lat, B->nseg, B->NBq, B->segstart_d, B->seglen_d, B->nblk_d, B->blkoff_d, B->Ab_d, B->Pb_d, B->Gb_d,
        B->rhs_d, B->flag_d);
  } else {
    const size_t smem = solve_smem_bytes(lat);
    k_band_solve<<<nq * B->nseg, 32, smem, h->stream>>>(lat, B->nseg, B->segstart_d, B->seglen_d, B->AB_d,
                                                        B->ipiv_d, B->rhs_d);
  }
  C3D_LAUNCH_CHECK(h);
  if (B->fft)
    k_band_inv_fft<<<dim3(nfc, 4), kFftThreads, fft_smem_bytes(nzl), h->stream>>>(
        nb, lat, nzl, nq, B->fftP, B->ftw_d, B->fpos_d, B->pos_d, B->rhs_d, out);
  else
    k_band_inv<<<dim3(nmc, 4, (unsigned)((nzl + kInvZ - 1) / kInvZ)), 256, inv_smem_bytes(nzl, nq), h->stream>>>(
        nb, lat, nzl, nq, B->tw_d, B->pos_d, B->rhs_d, out);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// whether the factors in use are the block-tridiagonal ones (else the
// pivoted banded LU)
bool band_is_block(Handle* h) {
  const BandState* B = h->ib ? h->ib->band : nullptr;
  return B != nullptr && B->block;
}

// Access for the learned preconditioner (k_mlp.cu): the lattice, the
// neighbour table and the band symbol That, which the network fills before
// band_factor_symbol factors it.
BandView band_view(Handle* h) {
  BandView v{};
  if (!band_supported(h)) return v;
  BandState* B = h->ib->band;
  v.lat = B->lat; v.nzl = B->nzl; v.nq = B->nq;
  v.nbr = B->nbr_d; v.That = B->That_d;
  return v;
}

// factor the band systems from the symbol in That (filled by the network);
// the factors are then those of the learned band, not of a probe
int band_factor_symbol(Handle* h, double dt) {
  (void)dt;
  int rc = band_factor_that(h);
  if (rc) {
    if (rc == C3D_ERR_NAN) h->last_error = "learned band preconditioner: singular band system";
    return rc;
  }
  h->ib->band->built = false;
  return 0;
}
int band_probe_count(Handle* h) {
  if (!band_supported(h)) return 0;
  int n = 0;
  for (auto& v : h->ib->band->colours) n += (int)v.size();
  return n;
}

}  // namespace c3d
