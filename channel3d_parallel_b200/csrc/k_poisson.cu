// Pseudo-pressure Poisson solve and projection.
//
// solve_poisson_equation (src/poisson.f90:33-101) restated for one GPU:
//   per y-plane 2-D DFT over (x, z)   -> k_xfft_fwd: x real-to-complex FFT of
//                                        each (j, k) line (two real lines per
//                                        complex FFT), divergence fused in;
//   per (kx, kz) tridiagonal in y     -> k_spectral_yz: one thread-block
//   (Zgtsv, :50-75)                      cluster per kx slab; each CTA brings
//                                        its rows of the slab into shared
//                                        memory with bulk copies, does the z
//                                        FFT in place, the Thomas elimination
//                                        in j (carried across the cluster's
//                                        CTAs through distributed shared
//                                        memory), the inverse z FFT, and
//                                        copies the rows back;
//   inverse DFT / (nxp*nzp), real     -> k_xfft_inv: complex-to-real x FFT of
//   part, periodic copies (:78-88)       the Hermitian half spectrum.
// gradient (src/differential_operators.f90:16-52) and the projection update
// (src/projection.f90:22-46) are k_grad_sub; in the time step k_grad_sub2,
// which also writes every ghost entry of u, v, w (the boundary conditions)
// and, in the last stage, adds the constant-x-mass-flow shift whose bulk
// flux the forward x FFT reduced (k_xfft_fwd<.., FLUX>).
//
// Two precisions share the kernels (template T): FP64, and FP32 for the
// mixed-precision solve, where the kx = kz = 0 wall-normal mode is computed
// in FP64 (line sums of the right-hand side and an FP64 Thomas solve of the
// pinned mean mode) and the FP32 result is refined by re-projecting with the
// FP64 residual div(u).
//
// Spectrum layout in HBM: spec[(m*Ny + (j-2))*pz + (k-2)], m = 0..Nx/2: a kx
// slab is Ny contiguous rows of pz >= Nz complex values.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "bulk.cuh"
#include "c3d_internal.cuh"
#include "fft.cuh"
#include "ghost_images.cuh"

namespace cg = cooperative_groups;

namespace c3d {

// ---------------------------------------------------------------------------
// host set-up
// ---------------------------------------------------------------------------
// largest FFT radix compiled into the x-FFT kernels and the two slab shapes
// (register budgets: 64-96 registers for the x kernels and the narrow slab
// CTAs, 128 for the wide ones)
constexpr int kXMaxR = 8;
constexpr int kYzMaxRWide = 16;
constexpr int kYzMaxRNarrow = 8;

static bool make_passes(int n, FftPasses& P) { return make_fft_passes(n, P, 8); }

static FftPasses get_passes(int n, int maxr) {
  FftPasses P{};
  make_fft_passes(n, P, maxr);
  return P;
}

template <typename C>
static int make_twiddles(Handle* h, int n, C** out) {
  std::vector<C> t(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < n; ++m) {
    long double a = -2.0L * pi * (long double)m / (long double)n;
    t[m].x = (decltype(t[m].x))cosl(a);
    t[m].y = (decltype(t[m].y))sinl(a);
  }
  if (*out == nullptr) {
    int rc = dev_alloc(h, out, n);
    if (rc) return rc;
  }
  C3D_CUDA_TRY(h, cudaMemcpyAsync(*out, t.data(), sizeof(C) * n, cudaMemcpyHostToDevice, h->stream));
  return 0;
}

// Thomas factorisation of every mode, the no-pivot path of the reference's
// LAPACK zgtsv call (src/poisson.f90:72): MULT = DL(k)/D(k), D(k+1) -= MULT*DU(k).
// Stored: mult_j and 1/d'_j, layout [(m*Ny + j)*nkzs + kz'].
static int build_tri_table(Handle* h) {
  const Dims& d = h->d;
  SpectralState& S = h->sp;
  const int Ny = d.Ny, nkx = d.nkx, nkzs = d.nkzs;
  const int64_t nt = (int64_t)Ny * nkzs * nkx;
  std::vector<double> rdp(nt), mult(nt);
  std::vector<float> rdp32(nt), mult32(nt);
  std::vector<double> D(Ny), dl(Ny, 0.0), du(Ny, 0.0);
  std::vector<float> dl32(Ny, 0.0f), du32(Ny, 0.0f);
  for (int jj = 0; jj + 1 < Ny; ++jj) {
    dl[jj] = h->Dl[jj + 3];   // Dyy(j+1, j), j = jj+2
    du[jj] = h->Du[jj + 2];   // Dyy(j, j+1)
    dl32[jj] = (float)dl[jj];
    du32[jj] = (float)du[jj];
  }
  for (int m = 0; m < nkx; ++m) {
    for (int kzs = 0; kzs < nkzs; ++kzs) {
      for (int jj = 0; jj < Ny; ++jj) D[jj] = (h->Dd[jj + 2] + h->kxx[m]) + h->kzz[kzs];
      if (m == 0 && kzs == 0) D[0] = 3.0 / 2.0 * D[0];       // src/poisson.f90:69
      for (int jj = 0; jj < Ny; ++jj) {
        const int64_t o = ((int64_t)m * Ny + jj) * nkzs + kzs;
        double mu = 0.0;
        if (jj + 1 < Ny) {
          mu = dl[jj] / D[jj];
          D[jj + 1] = D[jj + 1] - mu * du[jj];
        }
        rdp[o] = 1.0 / D[jj];
        mult[o] = mu;
        rdp32[o] = (float)rdp[o];
        mult32[o] = (float)mu;
      }
    }
  }
  int rc;
  if (S.rdp == nullptr) {
    if ((rc = dev_alloc(h, &S.rdp, nt))) return rc;
    if ((rc = dev_alloc(h, &S.mult, nt))) return rc;
    if ((rc = dev_alloc(h, &S.rdp32, nt))) return rc;
    if ((rc = dev_alloc(h, &S.mult32, nt))) return rc;
    if ((rc = dev_alloc(h, &S.dl, Ny))) return rc;
    if ((rc = dev_alloc(h, &S.du, Ny))) return rc;
    if ((rc = dev_alloc(h, &S.dl32, Ny))) return rc;
    if ((rc = dev_alloc(h, &S.du32, Ny))) return rc;
  }
  cudaStream_t s = h->stream;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.rdp, rdp.data(), nt * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.mult, mult.data(), nt * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.rdp32, rdp32.data(), nt * 4, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.mult32, mult32.data(), nt * 4, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.dl, dl.data(), Ny * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.du, du.data(), Ny * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.dl32, dl32.data(), Ny * 4, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.du32, du32.data(), Ny * 4, cudaMemcpyHostToDevice, s));
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : C3D_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// kernel 1: (divergence |) x real-to-complex FFT of (j, k) lines
// ---------------------------------------------------------------------------
// Two real x-lines form one complex line; a block transforms kLinesX complex
// lines in place (rows of stride rs in shared memory) with a thread count
// that is a multiple of Nx, so every FFT stage keeps one butterfly position
// per thread.
constexpr int kLinesX = 8;      // complex x-lines per block
constexpr int kMaxNx = 512;

template <typename T>
struct XfwdArgs {
  Dims d;
  Metric m;
  const double* __restrict__ U;
  const double* __restrict__ V;
  const double* __restrict__ W;
  const double* __restrict__ rhs;             // right-hand side when not fused with div
  typename cplx<T>::t* __restrict__ spec;
  const typename cplx<T>::t* __restrict__ tw;
  double* __restrict__ linesum;               // FP64 line sums (mixed path) or null
  const int* __restrict__ pos;                // digit-reversed position of coefficient m
  FftPasses P;
  int pz;                                     // spectrum row pitch
  int rs;                                     // shared-memory row stride
  int64_t rbase, nlines;                      // lines rbase .. rbase+nlines-1 (a band of j rows)
  // x bulk flux of u (FLUX kernels): per-block partials, the last block
  // writes the constant-mass-flow correction to scw
  double* flux_part;
  DevScalars* scw;
  double q0, norm, dt;
};

// real x-line r = (k-2) + Nz*(j-2); its spectrum goes to slab offset
// (j-2)*pz + (k-2)
__device__ __forceinline__ void line_info(const Dims& d, int pz, int64_t r, int* j, int* k, int* off) {
  const int jj = (int)(r / d.Nz), kk = (int)(r - (int64_t)jj * d.Nz);
  *j = 2 + jj;
  *k = 2 + kk;
  *off = jj * pz + kk;
}

// shared-memory carve-up of the x-FFT kernels
template <typename T>
struct XfftSmem {
  typename cplx<T>::t* tw;     // [N]
  typename cplx<T>::t* buf;    // [kLinesX][rs]
  int* pos;                    // [N] digit-reversed position of coefficient m
  double* sval;                // [2*kLinesX][N] FP64 values for line sums (FP32 path)
};

template <typename T>
__device__ __forceinline__ XfftSmem<T> xfft_carve(unsigned char* base, int N, int rs) {
  using C = typename cplx<T>::t;
  XfftSmem<T> s;
  s.tw = reinterpret_cast<C*>(base);
  s.buf = s.tw + N;
  s.pos = reinterpret_cast<int*>(s.buf + (size_t)kLinesX * rs);
  s.sval = reinterpret_cast<double*>(s.pos + N + (N & 1));   // FP32 path only
  return s;
}

// FLUX: the bulk flux of u (src/mass_flow.f90:24-53, 144-175) is reduced
// from the u values this kernel reads (compute_time_step_RK3's correction,
// src/time_integration.f90:187-193, then needs no pass of its own): weights
// wq(j) + wq(j+1) per row and plane 2 twice (plane nzg-1 is its copy).
template <bool FROM_DIV, typename T, bool FLUX = false>
__global__ void __launch_bounds__(kMaxNx) k_xfft_fwd(XfwdArgs<T> a) {
  using C = typename cplx<T>::t;
  extern __shared__ __align__(16) unsigned char xf_smem[];
  __shared__ int s_j[2 * kLinesX], s_off[2 * kLinesX];
  __shared__ double s_cq[FLUX ? 2 * kLinesX : 1];
  // per real line: offsets of the x = 2 cell of u(j,k), v(j,k), v(j-1,k),
  // w(j,k), w(j,k-1) (FROM_DIV) or of the right-hand side; -1: a zero wall
  // value of v (j-1 = 1 or j = ny), or no line
  __shared__ int64_t s_bu[2 * kLinesX], s_bv[2 * kLinesX], s_bvm[2 * kLinesX];
  __shared__ int64_t s_bw[2 * kLinesX], s_bwm[2 * kLinesX];
  __shared__ double s_ry[2 * kLinesX], s_rz[2 * kLinesX];
  const Dims& d = a.d;
  const int N = d.Nx, RS = a.rs;
  const int tid = threadIdx.x, nt = blockDim.x;
  XfftSmem<T> sm = xfft_carve<T>(xf_smem, N, RS);
  for (int t = tid; t < N; t += nt) {
    sm.tw[t] = a.tw[t];
    sm.pos[t] = a.pos[t];
  }
  const int64_t nreal = a.rbase + a.nlines;
  const int64_t r0 = a.rbase + (int64_t)blockIdx.x * kLinesX * 2;
  if (tid < 2 * kLinesX) {
    const int64_t r = r0 + tid;
    int j = -1, k = -1, off = 0;
    int64_t bu = -1, bv = -1, bvm = -1, bw = 0, bwm = 0;
    double ry = 0.0, rz = 0.0;
    if (r < nreal) {
      line_info(d, a.pz, r, &j, &k, &off);
      if (FROM_DIV) {
        // the ghost values are read as the boundary conditions define them
        // (periodic images in x and z, zero V walls), so the fields need no
        // ghost fill after the stage update
        const int64_t plw = (int64_t)d.nxg * d.nyg;
        const int64_t iv = idxV(d, 2, j, k), iw = idxW(d, 2, j, k);
        bu = idxU(d, 2, j, k);
        bv = j == d.ny ? -1 : iv;
        bvm = j == 2 ? -1 : iv - d.nxg;
        bw = iw;
        bwm = k == 2 ? iw + (int64_t)(d.Nz - 1) * plw : iw - plw;
        ry = a.m.rdy[j];
        rz = a.m.rdz[k];
        if (FLUX) s_cq[tid] = a.m.cqu[j] * (k == 2 ? 2.0 : 1.0);
      } else {
        bu = idxR(d, 2, j, k);
      }
    }
    s_j[tid] = j;
    s_off[tid] = off;
    s_bu[tid] = bu; s_bv[tid] = bv; s_bvm[tid] = bvm; s_bw[tid] = bw; s_bwm[tid] = bwm;
    s_ry[tid] = ry; s_rz[tid] = rz;
    if (FLUX && r >= nreal) s_cq[tid] = 0.0;
  }
  pdl_wait();
  pdl_trigger();
  __syncthreads();
  double facc = 0.0;
  // nt is a multiple of N: thread -> x index ii, real lines rl0, rl0 + nt/N, ...
  // taken four at a time: all loads of a batch are issued before any use.
  // u(i-1) of i = 2 is the periodic image i = N+1.
  const int ii = tid % N, rls = nt / N;
  const int xo = ii == 0 ? N - 1 : ii - 1;
  const double rdx_i = FROM_DIV ? a.m.rdx[2 + ii] : 0.0;
  constexpr int kBatch = 4;
  for (int rb = tid / N; rb < 2 * kLinesX; rb += kBatch * rls) {
    double x0[kBatch], x1[kBatch], y0[kBatch], y1[kBatch], z0[kBatch], z1[kBatch];
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      const int rl = rb + q * rls;
      const int64_t bu = rl < 2 * kLinesX ? s_bu[rl] : -1;
      x0[q] = x1[q] = y0[q] = y1[q] = z0[q] = z1[q] = 0.0;
      if (bu >= 0) {
        if (FROM_DIV) {
          const int64_t bv = s_bv[rl], bvm = s_bvm[rl];
          x1[q] = a.U[bu + ii]; x0[q] = a.U[bu + xo];
          if (bv >= 0) y1[q] = a.V[bv + ii];
          if (bvm >= 0) y0[q] = a.V[bvm + ii];
          z1[q] = a.W[s_bw[rl] + ii]; z0[q] = a.W[s_bwm[rl] + ii];
        } else {
          x1[q] = a.rhs[bu + ii];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      const int rl = rb + q * rls;
      if (rl >= 2 * kLinesX) continue;
      const double val = FROM_DIV ? (x1[q] - x0[q]) * rdx_i + (y1[q] - y0[q]) * s_ry[rl] + (z1[q] - z0[q]) * s_rz[rl]
                                  : x1[q];
      if (FLUX) facc += s_cq[rl] * x1[q];
      C& zz = sm.buf[(rl >> 1) * RS + ii];
      if (rl & 1) zz.y = (T)val; else zz.x = (T)val;
      if (a.linesum) sm.sval[rl * N + ii] = val;
    }
  }
  __syncthreads();
  if (a.linesum) {   // FP64 line sums: one full warp per line, a fixed shuffle tree
    const int warp = tid >> 5, lane = tid & 31;
    for (int rl = warp; rl < 2 * kLinesX && (warp + 1) * 32 <= nt; rl += nt >> 5) {
      double sum = 0.0;
      for (int q = lane; q < N; q += 32) sum += sm.sval[rl * N + q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (lane == 0 && r0 + rl < nreal) a.linesum[r0 + rl] = sum;
    }
  }
  fft_rows_dif<T, kXMaxR>(sm.buf, kLinesX, RS, sm.tw, a.P);
  // split Z = A + iB of the two real lines: A = (Z_m + conj Z_{N-m})/2,
  // B = (Z_m - conj Z_{N-m})/(2i), m = 0..N/2
  const int nk = d.nkx;
  for (int t = tid; t < kLinesX * nk; t += nt) {
    const int pl = t % kLinesX;
    const int mm = t / kLinesX;
    const int64_t ra = r0 + 2 * pl;
    if (ra >= nreal) continue;
    const C Z = sm.buf[pl * RS + sm.pos[mm]];
    const C Zr = sm.buf[pl * RS + sm.pos[mm == 0 ? 0 : N - mm]];
    C A, B;
    A.x = (T)0.5 * (Z.x + Zr.x);
    A.y = (T)0.5 * (Z.y - Zr.y);
    B.x = (T)0.5 * (Z.y + Zr.y);
    B.y = (T)-0.5 * (Z.x - Zr.x);
    C* out = a.spec + (int64_t)mm * d.Ny * a.pz;
    out[s_off[2 * pl]] = A;
    if (ra + 1 < nreal) out[s_off[2 * pl + 1]] = B;
  }
  if (FLUX) {
    // block partial by a fixed tree (any thread count up to kMaxNx); the last
    // block adds the partials the same way, then shift = Qflow_x_0 -
    // flux/norm and dPdx = (dPdx + shift/dt)/2
    __shared__ double red[kMaxNx];
    __shared__ bool last;
    auto tree = [&](double v) {
      red[tid] = v;
      __syncthreads();
      for (int st = kMaxNx / 2; st > 0; st >>= 1) {
        if (tid < st && tid + st < nt) red[tid] += red[tid + st];
        __syncthreads();
      }
      const double r = red[0];
      __syncthreads();
      return r;
    };
    const double bsum = tree(facc);
    if (tid == 0) {
      a.flux_part[blockIdx.x] = bsum;
      __threadfence();
      last = atomicAdd(&a.scw->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
      __threadfence();
      double t = 0.0;
      for (unsigned b = tid; b < gridDim.x; b += nt) t += __ldcg(a.flux_part + b);
      const double q = tree(t) / a.norm;
      if (tid == 0) {
        const double shift = a.q0 - q;
        DevScalars* sc = a.scw;
        sc->qflow = q;
        sc->shift = shift;
        sc->dpdx_prev = sc->dPdx;
        sc->dPdx = 0.5 * (sc->dPdx + shift / a.dt);
        sc->ticket = 0u;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// kernel 2: z FFT, Thomas in y, inverse z FFT of one kx slab per cluster
// ---------------------------------------------------------------------------
// Two launch shapes: wide CTAs (at most 256 threads, two per SM) and narrow
// CTAs (at most 192 threads, three per SM, half the rows).  The whole FP64
// spectrum does not fit the aggregate shared memory at once, so the grid runs
// in two waves either way; narrow CTAs keep more warps per SM in flight and
// shorten each CTA's sequential sweeps.  yz_jmax: rows of j per CTA (the
// pivots of one column are held in registers).
template <typename T, bool NARROW>
__host__ __device__ constexpr int yz_jmax() { return (sizeof(T) == 8 ? 32 : 64) / (NARROW ? 2 : 1); }
template <bool NARROW>
__host__ __device__ constexpr int yz_threads() { return NARROW ? 192 : 256; }
template <bool NARROW>
__host__ __device__ constexpr int yz_min_blocks() { return NARROW ? 3 : 2; }

template <typename T>
struct YzArgs {
  Dims d;
  typename cplx<T>::t* __restrict__ spec;
  const typename cplx<T>::t* __restrict__ tw;
  const T* __restrict__ rdp;     // 1/D'(j) per (m, j, kz')
  const T* __restrict__ dl;      // Dyy(j+1, j)
  const T* __restrict__ du;      // Dyy(j, j+1)
  unsigned long long* err;       // sticky error bits
  FftPasses P;
  int cs;        // CTAs per cluster
  int jc;        // j rows per CTA
  int rs;        // shared-memory row stride (complex values)
  int pz;        // HBM row pitch (complex values)
  int zero00;    // 1: leave the kx = kz = 0 column to the FP64 mean-mode solve
  int rlo, rhi;  // rows (j-2) with a nonzero right-hand side and rows of the
                 // solution needed: the band [rlo, rhi]; other rows start at
                 // zero and are not transformed back or stored
};

// CTA c of the cluster owns rows j0 = c*jc .. j0+jn-1 of the slab.  Shared
// memory: rows [jc][rs] (the z FFT runs along a row), twiddles, DL and DU.
// The Thomas sweeps walk a column (one kz per thread) down the rows, CTA by
// CTA: forward elimination from CTA 0 to cs-1, back substitution from cs-1 to
// 0, each CTA starting from the neighbour row read through distributed
// shared memory.  After the forward transform column `col` holds wavenumber
// kz = dif_position_to_k(col); the inverse transform takes that order back.
template <typename T, bool NARROW>
__global__ void __launch_bounds__(yz_threads<NARROW>(), yz_min_blocks<NARROW>()) k_spectral_yz(YzArgs<T> a) {
  using C = typename cplx<T>::t;
  constexpr int JM = yz_jmax<T, NARROW>();
  extern __shared__ __align__(128) unsigned char yz_smem[];
  __shared__ __align__(8) uint64_t bar;
  cg::cluster_group cl = cg::this_cluster();
  const Dims& d = a.d;
  const int cs = a.cs;
  const int crank = (int)cl.block_rank();
  const int m = blockIdx.x / cs;
  const int Ny = d.Ny, Nz = d.Nz, nkzs = d.nkzs;
  const int RS = a.rs, Jc = a.jc;
  const int j0 = crank * Jc;
  const int jn = min(Jc, Ny - j0);             // rows owned by this CTA (>= 1)
  C* data = reinterpret_cast<C*>(yz_smem);
  C* tw = data + (size_t)Jc * RS;
  C* ylast = tw + Nz;                          // local forward value of the last row
  C* xfirst = ylast + Nz;                      // local back-substituted first row
  C* yin = xfirst + Nz;                        // carry Y_in of this CTA
  T* sdl = reinterpret_cast<T*>(yin + Nz);
  T* sdu = sdl + Ny;
  const int tid = threadIdx.x, nt = blockDim.x;
  C* g = a.spec + ((int64_t)m * Ny + j0) * a.pz;
  const unsigned rowbytes = (unsigned)(a.pz * sizeof(C));

  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  pdl_wait();
  pdl_trigger();
  __syncthreads();
  // this CTA's rows of the band: [blo, bhi)
  const int blo = min(max(a.rlo - j0, 0), jn), bhi = max(min(a.rhi + 1 - j0, jn), blo);
  if (tid < 32) {
    if (tid == 0) mbar_arrive_expect_tx(&bar, rowbytes * (unsigned)(bhi - blo));
    __syncwarp();
    for (int r = blo + tid; r < bhi; r += 32)
      bulk_load(data + (size_t)r * RS, g + (int64_t)r * a.pz, rowbytes, &bar);
  }
  for (int t = tid; t < (jn - (bhi - blo)) * Nz; t += nt) {   // rows outside the band start at zero
    const int rr = t / Nz, col = t - rr * Nz;
    const int r = rr < blo ? rr : rr + (bhi - blo);
    data[(size_t)r * RS + col] = C{(T)0, (T)0};
  }
  for (int t = tid; t < Nz; t += nt) tw[t] = a.tw[t];
  for (int t = tid; t < Ny; t += nt) { sdl[t] = a.dl[t]; sdu[t] = a.du[t]; }

  const bool loaded = mbar_wait(&bar, 0, kWaitCycles);
  if (!loaded) atomicOr(a.err, 1ull);
  __syncthreads();

  fft_rows_dif<T, (NARROW ? kYzMaxRNarrow : kYzMaxRWide)>(data + (size_t)blo * RS, bhi - blo, RS, tw, a.P);

  // pivots of this thread's column for rows j0-1 .. j0+jn-1 (one column per
  // thread when Nz <= blockDim; otherwise reloaded per column below)
  const T* rdp_m = a.rdp + (int64_t)m * Ny * nkzs;
  const bool one_col = Nz <= nt;
  T rdv[JM];
  T rdm1 = (T)0;                               // pivot of row j0-1 (previous CTA)
  auto load_pivots = [&](int col) {
    const int kz = dif_position_to_k(col, a.P);
    const int kzs = kz <= Nz - kz ? kz : Nz - kz;
#pragma unroll
    for (int jl = 0; jl < JM; ++jl)
      rdv[jl] = jl < jn ? __ldg(rdp_m + (int64_t)(j0 + jl) * nkzs + kzs) : (T)0;
    rdm1 = j0 > 0 ? __ldg(rdp_m + (int64_t)(j0 - 1) * nkzs + kzs) : (T)0;
  };
  if (one_col && tid < Nz) load_pivots(tid);

  // Partitioned elimination: every CTA sweeps its own rows at once, then
  // corrects them with carries from its neighbours (no tables):
  //   forward: y(j) = yl(j) + h(j) Y_in,  h(j0-1) = 1, h(j) = -MULT(j-1) h(j-1),
  //            Y_in(c+1) = yl_c(j1) + h_c(j1) Y_in(c);
  //   backward (on the corrected y): x(j) = xl(j) + g(j) X_in,  g(j1+1) = 1,
  //            g(j) = -DU(j)/D'(j) g(j+1),  X_in(c-1) = xl_c(j0) + g_c(j0) X_in(c).
  // The sweeps take rows in chunks of kCh: loads of a chunk are issued
  // together, the recurrence runs in registers, then the chunk is stored.
  constexpr int kCh = 4;
  // ylast / xfirst: published end values; hg[col] = (h(j1), g(j0))
  C* hg = yin;
  for (int col = tid; col < Nz; col += nt) {
    if (!one_col) load_pivots(col);
    // local forward elimination B(j) -= DL(j-1)/D'(j-1) * B(j-1) from y(j0-1) = 0
    C prev = C{(T)0, (T)0};
    T hcur = (T)1;
#pragma unroll
    for (int c0 = 0; c0 < JM; c0 += kCh) {
      if (c0 < jn) {
        C bv[kCh];
        T dlv[kCh];
#pragma unroll
        for (int u = 0; u < kCh; ++u) {
          const int jl = c0 + u;
          bv[u] = C{(T)0, (T)0};
          dlv[u] = (T)0;
          if (jl < jn) {
            bv[u] = data[jl * RS + col];
            if (j0 + jl > 0) dlv[u] = sdl[j0 + jl - 1];
          }
        }
#pragma unroll
        for (int u = 0; u < kCh; ++u) {
          const int jl = c0 + u;
          if (jl < jn) {
            const T mu = dlv[u] * (jl == 0 ? rdm1 : rdv[jl > 0 ? jl - 1 : 0]);
            if (jl > 0) {
              bv[u].x = bv[u].x - mu * prev.x;
              bv[u].y = bv[u].y - mu * prev.y;
            }
            hcur = -mu * hcur;
            prev = bv[u];
          }
        }
#pragma unroll
        for (int u = 0; u < kCh; ++u)
          if (c0 + u < jn) data[(c0 + u) * RS + col] = bv[u];
      }
    }
    ylast[col] = prev;
    hg[col].x = hcur;
  }
  cl.sync();
  for (int col = tid; col < Nz; col += nt) {
    if (!one_col) load_pivots(col);
    // Y_in = y(j0-1) from the predecessors' end values
    C Y = C{(T)0, (T)0};
    for (int c = 0; c < crank; ++c) {
      const C yl = cl.map_shared_rank(ylast, c)[col];
      const T he = cl.map_shared_rank(hg, c)[col].x;
      const T yx = yl.x + he * Y.x, yy = yl.y + he * Y.y;
      Y.x = yx;
      Y.y = yy;
    }
    // forward correction y += h Y_in (h recomputed), then the local back
    // substitution x(j) = (y(j) - DU(j) x(j+1)) / D'(j) from x(j1+1) = 0
    T hcur = (T)1;
#pragma unroll
    for (int c0 = 0; c0 < JM; c0 += kCh) {
      if (c0 < jn && crank > 0) {
        C bv[kCh];
        T dlv[kCh];
#pragma unroll
        for (int u = 0; u < kCh; ++u) {
          const int jl = c0 + u;
          bv[u] = C{(T)0, (T)0};
          dlv[u] = (T)0;
          if (jl < jn) {
            bv[u] = data[jl * RS + col];
            dlv[u] = sdl[j0 + jl - 1];
          }
        }
#pragma unroll
        for (int u = 0; u < kCh; ++u) {
          const int jl = c0 + u;
          if (jl < jn) {
            const T mu = dlv[u] * (jl == 0 ? rdm1 : rdv[jl > 0 ? jl - 1 : 0]);
            hcur = -mu * hcur;
            bv[u].x += hcur * Y.x;
            bv[u].y += hcur * Y.y;
          }
        }
#pragma unroll
        for (int u = 0; u < kCh; ++u)
          if (c0 + u < jn) data[(c0 + u) * RS + col] = bv[u];
      }
    }
    C xn = C{(T)0, (T)0};
    T gcur = (T)1;
#pragma unroll
    for (int c0 = JM - kCh; c0 >= 0; c0 -= kCh) {
      if (c0 < jn) {
        C bv[kCh];
        T duv[kCh];
#pragma unroll
        for (int u = 0; u < kCh; ++u) {
          const int jl = c0 + u;
          bv[u] = C{(T)0, (T)0};
          duv[u] = (T)0;
          if (jl < jn) {
            bv[u] = data[jl * RS + col];
            duv[u] = sdu[j0 + jl];
          }
        }
#pragma unroll
        for (int u = kCh - 1; u >= 0; --u) {
          const int jl = c0 + u;
          if (jl < jn) {
            bv[u].x = (bv[u].x - duv[u] * xn.x) * rdv[jl];
            bv[u].y = (bv[u].y - duv[u] * xn.y) * rdv[jl];
            gcur = -duv[u] * rdv[jl] * gcur;
            xn = bv[u];
          }
        }
#pragma unroll
        for (int u = 0; u < kCh; ++u)
          if (c0 + u < jn) data[(c0 + u) * RS + col] = bv[u];
      }
    }
    xfirst[col] = xn;
    hg[col].y = gcur;
  }
  cl.sync();
  for (int col = tid; col < Nz; col += nt) {
    if (!one_col) load_pivots(col);
    // X_in = x(j1+1) from the successors' first values
    C X = C{(T)0, (T)0};
    for (int c = cs - 1; c > crank; --c) {
      const C xf = cl.map_shared_rank(xfirst, c)[col];
      const T ge = cl.map_shared_rank(hg, c)[col].y;
      const T xx = xf.x + ge * X.x, xy = xf.y + ge * X.y;
      X.x = xx;
      X.y = xy;
    }
    // backward correction x += g X_in (g recomputed from the last row up)
    T gcur = (T)1;
#pragma unroll
    for (int c0 = JM - kCh; c0 >= 0; c0 -= kCh) {
      if (c0 < jn && crank < cs - 1) {
        C bv[kCh];
        T duv[kCh];
#pragma unroll
        for (int u = 0; u < kCh; ++u) {
          const int jl = c0 + u;
          bv[u] = C{(T)0, (T)0};
          duv[u] = (T)0;
          if (jl < jn) {
            bv[u] = data[jl * RS + col];
            duv[u] = sdu[j0 + jl];
          }
        }
#pragma unroll
        for (int u = kCh - 1; u >= 0; --u) {
          const int jl = c0 + u;
          if (jl < jn) {
            gcur = -duv[u] * rdv[jl] * gcur;
            bv[u].x += gcur * X.x;
            bv[u].y += gcur * X.y;
          }
        }
#pragma unroll
        for (int u = 0; u < kCh; ++u)
          if (c0 + u < jn) data[(c0 + u) * RS + col] = bv[u];
      }
    }
    if (a.zero00 && m == 0 && col == 0)
      for (int jl = 0; jl < jn; ++jl) data[jl * RS] = C{(T)0, (T)0};
  }
  __syncthreads();

  fft_rows_dit_inv<T, (NARROW ? kYzMaxRNarrow : kYzMaxRWide)>(data + (size_t)blo * RS, bhi - blo, RS, tw, a.P);
  // no CTA leaves while another may still read its ylast / xfirst
  cl.sync();

  fence_async_shared();
  __syncthreads();
  if (tid < 32) {
    if (loaded) {
      for (int r = blo + tid; r < bhi; r += 32) bulk_store(g + (int64_t)r * a.pz, data + (size_t)r * RS, rowbytes);
      bulk_commit();
      bulk_wait_read_all();
    } else {
      // the rows never arrived: let the copies in flight finish before exit
      mbar_wait(&bar, 0, kWaitCycles);
    }
  }
}

// ---------------------------------------------------------------------------
// Band-restricted z transform and y solve (FP64), for the Poisson solve of
// the Schur complement: the right-hand side is zero outside the rows
// [rlo, rhi] and only those rows of the solution are read.  Thomas on the
// band alone: the forward sweep starts at rlo from zero, and the back
// substitution starts from x(rhi+1) = S(rhi+1) y(rhi+1), y(rhi+1) =
// -MULT(rhi) y(rhi), where S(j) = x(j)/y(j) of the homogeneous tail is
// tabulated once (build_tail_table).  One CTA per kx slab, the band rows in
// shared memory; the same z transform as k_spectral_yz.
// ---------------------------------------------------------------------------
struct BandYzArgs {
  Dims d;
  double2* __restrict__ spec;
  const double2* __restrict__ tw;
  const double* __restrict__ rdp;
  const double* __restrict__ tail;
  const double* __restrict__ dl;
  const double* __restrict__ du;
  FftPasses P;
  int rs, pz;
  int rlo, rhi;
};

__global__ void __launch_bounds__(256) k_spectral_band(BandYzArgs a) {
  extern __shared__ __align__(16) unsigned char sb_smem[];
  const int m = blockIdx.x;
  const int Ny = a.d.Ny, Nz = a.d.Nz, nkzs = a.d.nkzs, RS = a.rs;
  const int nr = a.rhi - a.rlo + 1;
  double2* data = reinterpret_cast<double2*>(sb_smem);   // [nr][RS]
  double2* tw = data + (size_t)nr * RS;                   // [Nz]
  const int tid = threadIdx.x, nt = blockDim.x;
  double2* g = a.spec + ((int64_t)m * Ny + a.rlo) * a.pz;
  for (int t = tid; t < Nz; t += nt) tw[t] = a.tw[t];
  pdl_wait();
  pdl_trigger();
  // eight loads in flight per thread before any store
  for (int t0 = tid; t0 < nr * Nz; t0 += 8 * nt) {
    double2 tv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * nt, r = t / Nz, c = t - r * Nz;
      tv[u] = t < nr * Nz ? g[(int64_t)r * a.pz + c] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * nt, r = t / Nz, c = t - r * Nz;
      if (t < nr * Nz) data[r * RS + c] = tv[u];
    }
  }
  __syncthreads();
  fft_rows_dif<double, kYzMaxRWide>(data, nr, RS, tw, a.P);
  const double* rdp_m = a.rdp + (int64_t)m * Ny * nkzs;
  const double* tail_m = a.tail + (int64_t)m * Ny * nkzs;
  for (int col = tid; col < Nz; col += nt) {
    const int kz = dif_position_to_k(col, a.P);
    const int kzs = kz <= Nz - kz ? kz : Nz - kz;
    // forward: y(j) = b(j) - DL(j-1)/D'(j-1) y(j-1), y(rlo-1) = 0
    double2 prev = make_double2(0.0, 0.0);
    for (int r = 0; r < nr; ++r) {
      const int j = a.rlo + r;
      double2 b = data[r * RS + col];
      if (r > 0) {
        const double mu = a.dl[j - 1] * rdp_m[(int64_t)(j - 1) * nkzs + kzs];
        b.x -= mu * prev.x;
        b.y -= mu * prev.y;
      }
      data[r * RS + col] = b;
      prev = b;
    }
    // the rows above the band, through the tail ratio
    double2 xn = make_double2(0.0, 0.0);
    if (a.rhi + 1 < Ny) {
      const double mu = a.dl[a.rhi] * rdp_m[(int64_t)a.rhi * nkzs + kzs];
      const double sx = -mu * tail_m[(int64_t)(a.rhi + 1) * nkzs + kzs];
      xn.x = sx * prev.x;
      xn.y = sx * prev.y;
    }
    // back substitution x(j) = (y(j) - DU(j) x(j+1)) / D'(j)
    for (int r = nr - 1; r >= 0; --r) {
      const int j = a.rlo + r;
      const double rp = rdp_m[(int64_t)j * nkzs + kzs];
      const double u = a.du[j];
      double2 b = data[r * RS + col];
      b.x = (b.x - u * xn.x) * rp;
      b.y = (b.y - u * xn.y) * rp;
      data[r * RS + col] = b;
      xn = b;
    }
  }
  __syncthreads();
  fft_rows_dit_inv<double, kYzMaxRWide>(data, nr, RS, tw, a.P);
  for (int t = tid; t < nr * Nz; t += nt) {
    const int r = t / Nz, c = t - r * Nz;
    g[(int64_t)r * a.pz + c] = data[r * RS + c];
  }
}

// S(j) = x(j)/y(j) when the right-hand side vanishes from row j on:
// S(Ny-1) = 1/D'(Ny-1), S(j) = (1 + DU(j) MULT(j) S(j+1)) / D'(j), with
// MULT(j) = DL(j)/D'(j) formed as the solves form it
static int build_tail_table(Handle* h) {
  const Dims& d = h->d;
  SpectralState& S = h->sp;
  const int Ny = d.Ny, nkx = d.nkx, nkzs = d.nkzs;
  const int64_t nt = (int64_t)Ny * nkzs * nkx;
  std::vector<double> rdp(nt), tail(nt), dl(Ny), du(Ny);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(rdp.data(), S.rdp, 8 * nt, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(dl.data(), S.dl, 8 * Ny, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(du.data(), S.du, 8 * Ny, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int m = 0; m < nkx; ++m)
    for (int kzs = 0; kzs < nkzs; ++kzs) {
      auto o = [&](int j) { return ((int64_t)m * Ny + j) * nkzs + kzs; };
      double sj = rdp[o(Ny - 1)];
      tail[o(Ny - 1)] = sj;
      for (int j = Ny - 2; j >= 0; --j) {
        const double mu = dl[j] * rdp[o(j)];
        sj = (1.0 + du[j] * mu * sj) * rdp[o(j)];
        tail[o(j)] = sj;
      }
    }
  int rc;
  if ((rc = dev_alloc(h, &S.tail, nt))) return rc;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S.tail, tail.data(), 8 * nt, cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

static size_t band_yz_smem(const Dims& d, int rs, int nr) {
  return sizeof(double2) * ((size_t)nr * rs + d.Nz);
}
static const size_t kBandYzSmemMax = 200 * 1024;

// the band solve of rows [blo, bhi] when it fits in shared memory; false
// (nothing launched) otherwise
static int launch_band_yz(Handle* h, int blo, int bhi, bool* done) {
  const Dims& d = h->d;
  SpectralState& S = h->sp;
  *done = false;
  const int nr = bhi - blo + 1;
  const size_t smem = band_yz_smem(d, S.rs64, nr);
  if (nr <= 0 || smem > kBandYzSmemMax) return 0;
  int rc;
  if (!S.tail) {   // first use (outside any graph capture: the table build synchronises)
    if ((rc = build_tail_table(h))) return rc;
    C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_spectral_band, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kBandYzSmemMax));
  }
  BandYzArgs a{};
  a.d = d; a.spec = S.spec; a.tw = S.twz; a.rdp = S.rdp; a.tail = S.tail; a.dl = S.dl; a.du = S.du;
  a.P = get_passes(d.Nz, kYzMaxRWide); a.rs = S.rs64; a.pz = S.pz64; a.rlo = blo; a.rhi = bhi;
  C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_spectral_band, dim3((unsigned)d.nkx), dim3(256), smem, h->stream, a));
  C3D_LAUNCH_CHECK(h);
  *done = true;
  return 0;
}

// ---------------------------------------------------------------------------
// FP64 kx = kz = 0 mode of the mixed path: plane sums and the pinned solve
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_mode00(Dims d, const double* __restrict__ linesum,
                                                 const double* __restrict__ mult, const double* __restrict__ rdp,
                                                 const double* __restrict__ du, double* __restrict__ phi00) {
  extern __shared__ double m00[];
  const int Ny = d.Ny, Nz = d.Nz, nkzs = d.nkzs;
  double* b00 = m00;                 // plane sums, then the solution
  double* sm_ = m00 + Ny;            // the (0, 0) rows of the factor tables
  double* sr = m00 + 2 * Ny;
  double* su = m00 + 3 * Ny;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  // plane sums: one warp per row j, a fixed shuffle tree over its z lines
  for (int j = warp; j < Ny; j += nw) {
    double s = 0.0;
    for (int k = lane; k < Nz; k += 32) s += linesum[(int64_t)j * Nz + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) b00[j] = s;
  }
  for (int j = threadIdx.x; j < Ny; j += blockDim.x) {
    sm_[j] = j > 0 ? mult[(int64_t)(j - 1) * nkzs] : 0.0;
    sr[j] = rdp[(int64_t)j * nkzs];
    su[j] = du[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // mode (0, 0): table entries (m = 0, kz' = 0), elimination in shared memory
    for (int j = 1; j < Ny; ++j) b00[j] = b00[j] - sm_[j] * b00[j - 1];
    double xn = b00[Ny - 1] * sr[Ny - 1];
    b00[Ny - 1] = xn;
    for (int j = Ny - 2; j >= 0; --j) {
      xn = (b00[j] - su[j] * xn) * sr[j];
      b00[j] = xn;
    }
  }
  __syncthreads();
  const double sd = (double)d.Nx * (double)d.Nz;
  for (int j = threadIdx.x; j < Ny; j += blockDim.x) phi00[j] = b00[j] / sd;
}

// ---------------------------------------------------------------------------
// kernel 3: x complex-to-real inverse FFT, write phi into rhs_p layout
// ---------------------------------------------------------------------------
template <typename T>
struct XinvArgs {
  Dims d;
  const typename cplx<T>::t* __restrict__ spec;
  const typename cplx<T>::t* __restrict__ tw;
  double* __restrict__ rhs;      // output phi (rhs_p layout)
  double* __restrict__ phi1;     // optional second copy (P side effect)
  const double* __restrict__ phi00;   // FP64 mean mode added to the output (mixed path)
  int accumulate;                // 1: rhs += result (refinement)
  const int* __restrict__ pos;   // digit-reversed position of coefficient m
  FftPasses P;
  int pz;                        // spectrum row pitch
  int rs;                        // shared-memory row stride
  int64_t rbase, nlines;         // lines rbase .. rbase+nlines-1 (a band of j rows)
  double inv_scale;              // 1/(nxp*nzp)
};

template <typename T>
__global__ void __launch_bounds__(kMaxNx) k_xfft_inv(XinvArgs<T> a) {
  using C = typename cplx<T>::t;
  extern __shared__ __align__(16) unsigned char xi_smem[];
  __shared__ int s_j[2 * kLinesX], s_off[2 * kLinesX];
  // per real line: offset of the x = 2 value of phi(j,k), and of phi(j,nzp+2)
  // for the plane k = 2 that the reference duplicates (else -1)
  __shared__ int64_t s_bo[2 * kLinesX], s_bo2[2 * kLinesX];
  __shared__ double s_p00[2 * kLinesX];   // FP64 mean mode of each line's row (mixed path)
  const Dims& d = a.d;
  const int N = d.Nx, nk = d.nkx, RS = a.rs;
  const int tid = threadIdx.x, nt = blockDim.x;
  XfftSmem<T> sm = xfft_carve<T>(xi_smem, N, RS);
  for (int t = tid; t < N; t += nt) {
    sm.tw[t] = a.tw[t];
    sm.pos[t] = a.pos[t];
  }
  const int64_t nreal = a.rbase + a.nlines;
  const int64_t r0 = a.rbase + (int64_t)blockIdx.x * kLinesX * 2;
  if (tid < 2 * kLinesX) {
    const int64_t r = r0 + tid;
    int j = -1, k = -1, off = 0;
    int64_t bo = -1, bo2 = -1;
    if (r < nreal) {
      line_info(d, a.pz, r, &j, &k, &off);
      bo = idxR(d, 2, j, k);
      if (k == 2) bo2 = idxR(d, 2, j, d.Nz + 2);
    }
    s_j[tid] = j;
    s_off[tid] = off;
    s_bo[tid] = bo;
    s_bo2[tid] = bo2;
  }
  pdl_wait();
  pdl_trigger();
  if (a.phi00 && tid < 2 * kLinesX) s_p00[tid] = s_j[tid] >= 2 ? a.phi00[s_j[tid] - 2] : 0.0;
  __syncthreads();
  // Z = A + iB on the full circle from the two half spectra, placed at the
  // digit-reversed positions the inverse transform expects
  // the spectrum values of kU items are loaded before any of them is placed
  constexpr int kU = 4;
  for (int t0 = tid; t0 < kLinesX * nk; t0 += kU * nt) {
    C Ab[kU], Bb[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int t = t0 + u * nt;
      Ab[u] = Bb[u] = C{(T)0, (T)0};
      if (t < kLinesX * nk) {
        const int pl = t % kLinesX, mm = t / kLinesX;
        const int64_t ra = r0 + 2 * pl;
        const C* in = a.spec + (int64_t)mm * d.Ny * a.pz;
        if (ra < nreal) Ab[u] = in[s_off[2 * pl]];
        if (ra + 1 < nreal) Bb[u] = in[s_off[2 * pl + 1]];
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int t = t0 + u * nt;
      if (t >= kLinesX * nk) break;
      const int pl = t % kLinesX, mm = t / kLinesX;
      C A = Ab[u], B = Bb[u];
      if (mm == 0 || 2 * mm == N) { A.y = (T)0; B.y = (T)0; }   // Hermitian projection
      C Z;
      Z.x = A.x - B.y;
      Z.y = A.y + B.x;
      sm.buf[pl * RS + sm.pos[mm]] = Z;
      if (mm > 0 && 2 * mm < N) {
        C Zc;
        Zc.x = A.x + B.y;
        Zc.y = -A.y + B.x;
        sm.buf[pl * RS + sm.pos[N - mm]] = Zc;
      }
    }
  }
  __syncthreads();
  fft_rows_dit_inv<T, kXMaxR>(sm.buf, kLinesX, RS, sm.tw, a.P);
  const double rsd = a.inv_scale;
  const int ii = tid % N, rls = nt / N;
  // apply_periodic_xz_centers (src/poisson.f90:106-125): x plane nxg-1 and
  // z plane nzp+2 duplicate plane 2
#pragma unroll 4
  for (int rl = tid / N; rl < 2 * kLinesX; rl += rls) {
    const int64_t bo = s_bo[rl], bo2 = s_bo2[rl];
    if (bo < 0) continue;
    const C z = sm.buf[(rl >> 1) * RS + ii];
    double v = (double)((rl & 1) ? z.y : z.x) * rsd;
    if (a.phi00) v += s_p00[rl];
    const int64_t o = bo + ii;
    if (a.accumulate) v += a.rhs[o];
    a.rhs[o] = v;
    if (ii == 0) a.rhs[bo + N] = v;
    if (bo2 >= 0) {
      a.rhs[bo2 + ii] = v;
      if (ii == 0) a.rhs[bo2 + N] = v;
    }
    if (a.phi1) {
      a.phi1[o] = v;
      if (ii == 0) a.phi1[bo + N] = v;
      if (bo2 >= 0) {
        a.phi1[bo2 + ii] = v;
        if (ii == 0) a.phi1[bo2 + N] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
// x-FFT launch shape: threads a multiple of Nx (at least 128), shared-memory
// rows padded (FP64: rs = 1 mod 8, FP32: rs odd) so that the line-parallel
// accesses are conflict-free
static int xfft_threads(const Dims& d) {
  int nt = d.Nx;
  while (nt < 128) nt += d.Nx;
  return nt;
}

template <typename T>
static int xfft_rs(const Dims& d) {
  int rs = d.Nx;
  if (sizeof(T) == 8) { while (rs % 8 != 1) ++rs; }
  else { while (rs % 2 != 1) ++rs; }
  return rs;
}

template <typename T>
static int xfft_smem(const Dims& d) {
  return (int)(sizeof(typename cplx<T>::t) * ((size_t)d.Nx + (size_t)kLinesX * xfft_rs<T>(d)) +
               sizeof(int) * (d.Nx + (d.Nx & 1)) +
               (sizeof(T) == 4 ? sizeof(double) * 2 * kLinesX * d.Nx : 0));
}

// cluster decomposition of a kx slab: the narrow shape when it fits (Nz <=
// 192, a CTA within 72 KB so three share an SM), else the wide shape (two
// CTAs per SM within 112 KB; 16-CTA clusters may use up to one SM each); in
// each the smallest power-of-two cluster whose CTAs own at most yz_jmax rows.
// Row stride: FP64 rows of 16-byte values padded to rs = 1 (mod 8) make
// row-to-row steps conflict-free; FP32 rows stay 16-byte aligned for the
// bulk copies (rs even) with rs = 2 (mod 4).
template <typename T, bool NARROW>
static bool choose_shape(const Dims& d, int rs, int& cs, int& jc, int& nt, int& smem) {
  const size_t esz = sizeof(typename cplx<T>::t);
  const int ntmax = yz_threads<NARROW>();
  // a multiple of Nz (one column per thread, fixed FFT butterflies) when
  // Nz <= ntmax
  nt = ntmax;
  if (d.Nz <= ntmax) {
    nt = d.Nz * (ntmax / d.Nz);
    if (nt > 128 && d.Nz >= 128) nt = d.Nz;
  } else if (NARROW) {
    return false;
  }
  const size_t limit = NARROW ? 72 * 1024 : 112 * 1024;
  for (cs = 1; cs <= 16; cs *= 2) {
    jc = (d.Ny + cs - 1) / cs;
    if ((cs - 1) * jc >= d.Ny) continue;      // every CTA must own a row
    if (jc > yz_jmax<T, NARROW>()) continue;
    const size_t bytes = esz * ((size_t)jc * rs + 4 * (size_t)d.Nz) + 2 * sizeof(T) * d.Ny;
    if (bytes <= limit || (!NARROW && cs == 16 && bytes <= 224 * 1024)) {
      smem = (int)bytes;
      return true;
    }
  }
  return false;
}

// Function attributes are process-wide and handles of different sizes share
// them, so a kernel's dynamic shared-memory limit only ever grows (per
// device; handles are created from one host thread at a time).
template <auto KERN>
static cudaError_t raise_smem_limit(int bytes) {
  static int cur[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (bytes <= cur[dev]) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(KERN, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) cur[dev] = bytes;
  return e;
}

template <typename T, bool NARROW>
static int active_clusters(int cs, int nt, int smem) {
  if (raise_smem_limit<k_spectral_yz<T, NARROW>>(smem) != cudaSuccess) return 0;
  if (cs > 8 &&
      cudaFuncSetAttribute(k_spectral_yz<T, NARROW>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return 0;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)cs, 1, 1);
  cfg.blockDim = dim3((unsigned)nt, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_spectral_yz<T, NARROW>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Picks the shape whose kx slabs (one cluster each) run in fewer waves of
// co-resident clusters, as the device reports them; the narrow shape on a tie.
template <typename T>
static bool choose_cluster(const Dims& d, int pz, int& cs, int& jc, int& rs, int& nt, int& smem, int& narrow) {
  rs = pz;
  if (sizeof(T) == 8) { while (rs % 8 != 1) ++rs; }
  else { while (rs % 4 != 2) ++rs; }
  int ncs, njc, nnt, nsm, wcs, wjc, wnt, wsm;
  const bool okn = choose_shape<T, true>(d, rs, ncs, njc, nnt, nsm);
  const bool okw = choose_shape<T, false>(d, rs, wcs, wjc, wnt, wsm);
  auto waves = [&](int active) { return active > 0 ? (d.nkx + active - 1) / active : 1 << 30; };
  const int wn = okn ? waves(active_clusters<T, true>(ncs, nnt, nsm)) : 1 << 30;
  const int ww = okw ? waves(active_clusters<T, false>(wcs, wnt, wsm)) : 1 << 30;
  if (okn && (!okw || wn <= ww)) {
    narrow = 1; cs = ncs; jc = njc; nt = nnt; smem = nsm;
    return true;
  }
  if (!okw) return false;
  narrow = 0; cs = wcs; jc = wjc; nt = wnt; smem = wsm;
  return true;
}

template <typename T>
static int launch_yz(Handle* h, typename cplx<T>::t* spec, const typename cplx<T>::t* tw, const T* rdp,
                     const T* dl, const T* du, int cs, int jc, int rs, int pz, int nt, int smem, int narrow,
                     int zero00, int rlo, int rhi) {
  const Dims& d = h->d;
  YzArgs<T> a{};
  a.d = d; a.spec = spec; a.tw = tw; a.rdp = rdp; a.dl = dl; a.du = du;
  a.err = &h->sc->err;
  a.P = get_passes(d.Nz, narrow ? kYzMaxRNarrow : kYzMaxRWide); a.cs = cs; a.jc = jc; a.rs = rs; a.pz = pz; a.zero00 = zero00;
  a.rlo = rlo; a.rhi = rhi;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(cs * d.nkx), 1, 1);
  cfg.blockDim = dim3((unsigned)nt, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = h->use_pdl ? 2 : 1;
  if (narrow) C3D_CUDA_TRY(h, cudaLaunchKernelEx(&cfg, k_spectral_yz<T, true>, a));
  else C3D_CUDA_TRY(h, cudaLaunchKernelEx(&cfg, k_spectral_yz<T, false>, a));
  C3D_LAUNCH_CHECK(h);
  return 0;
}

template <typename T>
static int set_limits(Handle* h, int smem_yz, int cs) {
  const Dims& d = h->d;
  const int smx = xfft_smem<T>(d);
  C3D_CUDA_TRY(h, (raise_smem_limit<k_xfft_fwd<true, T>>(smx)));
  C3D_CUDA_TRY(h, (raise_smem_limit<k_xfft_fwd<false, T>>(smx)));
  C3D_CUDA_TRY(h, (raise_smem_limit<k_xfft_fwd<true, T, true>>(smx)));
  C3D_CUDA_TRY(h, (raise_smem_limit<k_xfft_inv<T>>(smx)));
  C3D_CUDA_TRY(h, (raise_smem_limit<k_spectral_yz<T, true>>(smem_yz)));
  C3D_CUDA_TRY(h, (raise_smem_limit<k_spectral_yz<T, false>>(smem_yz)));
  if (cs > 8) {
    C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_spectral_yz<T, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_spectral_yz<T, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  }
  return 0;
}

// parts: bit0 x FFT, bit1 yz, bit2 inverse x FFT
template <typename T>
static int run_spectral_t(Handle* h, bool from_div, const double* U, const double* V, const double* W,
                          const double* rhs_in, double* out, double* phi1, int accumulate, int parts,
                          int blo = 0, int bhi = -1, double flux_dt = 0.0) {
  const Dims& d = h->d;
  SpectralState& S = h->sp;
  cudaStream_t s = h->stream;
  const bool f32 = sizeof(T) == 4;
  using C = typename cplx<T>::t;
  C* spec;
  const C *twx, *twz;
  const T *rdp, *dl, *du;
  int cs, jc, rs, pz, nt, smem, narrow;
  if (f32) {
    spec = (C*)S.spec32; twx = (const C*)S.twx32; twz = (const C*)S.twz32;
    rdp = (const T*)S.rdp32; dl = (const T*)S.dl32; du = (const T*)S.du32;
    cs = S.cs32; jc = S.jc32; rs = S.rs32; pz = S.pz32; nt = S.nt32; smem = S.smem32; narrow = S.nw32;
  } else {
    spec = (C*)S.spec; twx = (const C*)S.twx; twz = (const C*)S.twz;
    rdp = (const T*)S.rdp; dl = (const T*)S.dl; du = (const T*)S.du;
    cs = S.cs64; jc = S.jc64; rs = S.rs64; pz = S.pz64; nt = S.nt64; smem = S.smem64; narrow = S.nw64;
  }
  const FftPasses Px = get_passes(d.Nx, kXMaxR);
  if (bhi < 0) bhi = d.Ny - 1;                 // band of j rows (0-based j-2); full by default
  const int64_t rbase = (int64_t)blo * d.Nz, nlines = (int64_t)(bhi - blo + 1) * d.Nz;
  const int64_t npairs = (nlines + 1) / 2;
  const unsigned nbx = (unsigned)((npairs + kLinesX - 1) / kLinesX);
  const int smx = xfft_smem<T>(d);
  const int ntx = xfft_threads(d);
  const int rsx = xfft_rs<T>(d);
  if (parts & 1) {
    XfwdArgs<T> a{};
    a.d = d; a.m = h->m; a.U = U; a.V = V; a.W = W; a.rhs = rhs_in;
    a.spec = spec; a.tw = twx; a.P = Px; a.pz = pz; a.rs = rsx; a.rbase = rbase; a.nlines = nlines;
    a.linesum = f32 ? S.linesum : nullptr;
    a.pos = S.posx;
    if (flux_dt > 0.0 && from_div && nlines == (int64_t)d.Ny * d.Nz) {
      // the x bulk flux of U reduced on the way (constant x mass flow)
      if (h->flux_part_len < (int64_t)nbx) {
        h->last_error = "x bulk-flux partials not allocated";
        return C3D_ERR_CUDA;
      }
      a.flux_part = h->flux_part; a.scw = h->sc;
      a.q0 = h->Qflow_x_0; a.norm = h->norm_u; a.dt = flux_dt;
      C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_xfft_fwd<true, T, true>, nbx, ntx, smx, s, a));
    } else if (from_div) {
      C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_xfft_fwd<true, T>, nbx, ntx, smx, s, a));
    } else {
      C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_xfft_fwd<false, T>, nbx, ntx, smx, s, a));
    }
    C3D_LAUNCH_CHECK(h);
    if (f32) {
      k_mode00<<<1, 1024, 4 * sizeof(double) * d.Ny, s>>>(d, S.linesum, S.mult, S.rdp, S.du, S.phi00);
      C3D_LAUNCH_CHECK(h);
    }
  }
  if (parts & 2) {
    bool band_done = false;
    if (!f32 && (blo > 0 || bhi < d.Ny - 1)) {   // a band of rows: the band-restricted solve
      int rc = launch_band_yz(h, blo, bhi, &band_done);
      if (rc) return rc;
    }
    if (!band_done) {
      int rc = launch_yz<T>(h, spec, twz, rdp, dl, du, cs, jc, rs, pz, nt, smem, narrow, f32 ? 1 : 0, blo, bhi);
      if (rc) return rc;
    }
  }
  if (parts & 4) {
    XinvArgs<T> a{};
    a.d = d; a.spec = spec; a.tw = twx; a.rhs = out; a.phi1 = phi1;
    a.phi00 = f32 ? S.phi00 : nullptr; a.accumulate = accumulate;
    a.pos = S.posx;
    a.P = Px; a.pz = pz; a.rs = rsx; a.rbase = rbase; a.nlines = nlines;
    a.inv_scale = 1.0 / ((double)d.Nx * (double)d.Nz);
    C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_xfft_inv<T>, nbx, ntx, smx, s, a));
    C3D_LAUNCH_CHECK(h);
  }
  if (parts == 7) h->stats.poisson_solves++;
  return 0;
}

int profile_spectral(Handle* h, int part) {
  return run_spectral_t<double>(h, true, h->Us, h->Vs, h->Ws, nullptr, h->rhs_p, nullptr, 0, 1 << part);
}

// divergence only (fine entry and diagnostics): rhs_p = div(U,V,W) incl. the
// reference's duplicated planes i = nxg-1 and k = nzg-1, and zero plane nzg
__global__ void k_divergence(Dims d, Metric m, const double* __restrict__ U,
                             const double* __restrict__ V, const double* __restrict__ W,
                             double* __restrict__ rhs) {
  const int64_t n1 = d.nxg - 2, n2 = d.nyg - 2, n3 = d.nzg - 1;
  const int64_t tot = n1 * n2 * n3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 2 + (int)(t % n1);
    const int j = 2 + (int)((t / n1) % n2);
    const int k = 2 + (int)(t / (n1 * n2));
    double v = 0.0;
    if (k <= d.nzg - 1) {
      v = (U[idxU(d, i, j, k)] - U[idxU(d, i - 1, j, k)]) * m.rdx[i]
        + (V[idxV(d, i, j, k)] - V[idxV(d, i, j - 1, k)]) * m.rdy[j]
        + (W[idxW(d, i, j, k)] - W[idxW(d, i, j, k - 1)]) * m.rdz[k];
    }
    rhs[t] = v;
  }
}

int launch_divergence(Handle* h, const double* U, const double* V, const double* W, double* rhs) {
  k_divergence<<<148 * 8, 256, 0, h->stream>>>(h->d, h->m, U, V, W, rhs);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// in place on an rhs_p-shaped array; always FP64 (fine entry, IB operators)
int launch_poisson_solve(Handle* h, double* rhs, int rk_step, double dt) {
  int rc = run_spectral_t<double>(h, false, nullptr, nullptr, nullptr, rhs, rhs,
                                  rk_step == 1 ? h->phi1 : nullptr, 0, 7);
  if (rc) return rc;
  if (rk_step == 1) { h->P_pending = true; h->P_pending_dt = dt; }
  return 0;
}

// solve for the divergence of (U, V, W) into out (rhs_p layout), the
// divergence computed inside the forward x FFT (divergence followed by
// solve_poisson_equation, src/differential_operators.f90:54-74 and
// src/poisson.f90:33-101); P side effect at rk_step 1
int launch_poisson_of_div(Handle* h, const double* U, const double* V, const double* W, double* out,
                          int rk_step, double dt) {
  int rc = run_spectral_t<double>(h, true, U, V, W, nullptr, out, rk_step == 1 ? h->phi1 : nullptr, 0, 7);
  if (rc) return rc;
  if (rk_step == 1) { h->P_pending = true; h->P_pending_dt = dt; }
  return 0;
}

// the same restricted to a band of j rows (Fortran j = jlo..jhi): the
// divergence of (U, V, W) is zero outside the band and the caller reads the
// solution only inside it (the Schur complement's spread field and its
// gathers); rows of `out` outside the band are left as they were
int launch_poisson_of_div_band(Handle* h, const double* U, const double* V, const double* W, double* out,
                               int jlo, int jhi) {
  const int blo = std::max(jlo - 2, 0), bhi = std::min(jhi - 2, h->d.Ny - 1);
  if (bhi < blo) return 0;
  return run_spectral_t<double>(h, true, U, V, W, nullptr, out, nullptr, 0, 7, blo, bhi);
}

// ---------------------------------------------------------------------------
// projection: U = Ui - G phi at interior points (src/projection.f90:40-44),
// optional P_interim = phi/dt; ghosts are filled by the caller
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 6) k_grad_sub(Dims d, Metric m, const double* __restrict__ Ui,
                                                  const double* __restrict__ Vi,
                                                  const double* __restrict__ Wi,
                                                  const double* __restrict__ phi,
                                                  double* __restrict__ Uo, double* __restrict__ Vo,
                                                  double* __restrict__ Wo,
                                                  double* __restrict__ Pint, double rdt, int dup) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.Nx + 1 || j > d.Ny + 1 || k > d.Nz + 1) return;
  const double p0 = __ldg(phi + idxR(d, i, j, k));
  const double px = __ldg(phi + idxR(d, i + 1, j, k));
  const double pz = __ldg(phi + idxR(d, i, j, k + 1));
  const int64_t iu = idxU(d, i, j, k), iw = idxW(d, i, j, k);
  const double un = __ldg(Ui + iu) - (px - p0) * m.rdxg[i];
  const double wn = __ldg(Wi + iw) - (pz - p0) * m.rdzg[k];
  double py = 0.0, vn = 0.0;
  if (j <= d.Ny) {
    py = __ldg(phi + idxR(d, i, j + 1, k));
    vn = __ldg(Vi + idxV(d, i, j, k)) - (py - p0) * m.rdyg[j];
  }
  Uo[iu] = un;
  Wo[iw] = wn;
  if (j <= d.Ny) Vo[idxV(d, i, j, k)] = vn;
  if (dup && k == 2) {
    // the reference's gradient also covers plane nzg-1 (the duplicate of
    // plane 2) for the x and y components (src/differential_operators.f90:38-52);
    // the input's duplicate plane is read as the periodic image of plane 2.
    // Skipped (dup = 0) where the boundary conditions are applied next.
    const int kd = d.Nz + 2;
    Uo[idxU(d, i, j, kd)] = __ldg(Ui + iu) - (px - p0) * m.rdxg[i];
    if (j <= d.Ny) Vo[idxV(d, i, j, kd)] = __ldg(Vi + idxV(d, i, j, k)) - (py - p0) * m.rdyg[j];
  }
  if (Pint) {
    Pint[idxR(d, i, j, k)] = p0 * rdt;
    if (i == 2) Pint[idxR(d, d.Nx + 2, j, k)] = p0 * rdt;
    if (k == 2) {
      Pint[idxR(d, i, j, d.Nz + 2)] = p0 * rdt;
      if (i == 2) Pint[idxR(d, d.Nx + 2, j, d.Nz + 2)] = p0 * rdt;
    }
  }
}

// The same update for two cells (k, k+1) per thread, without the duplicate
// plane and P_interim (the time step's case): both cells' loads are issued
// before any store, and phi(k+1) serves both.  With ghosts = 1 every ghost
// entry of the results is written as well (the boundary conditions of the
// projected field): the x images by the threads of the boundary columns,
// the z and y images (whole blocks and warps) out of line.
__global__ void __launch_bounds__(256, 4) k_grad_sub2(Dims d, Metric m, const double* __restrict__ Ui,
                                                   const double* __restrict__ Vi,
                                                   const double* __restrict__ Wi,
                                                   const double* __restrict__ phi,
                                                   double* __restrict__ Uo, double* __restrict__ Vo,
                                                   double* __restrict__ Wo, int ghosts,
                                                   const double* __restrict__ ushift) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + 2 * (int)blockIdx.z;
  pdl_wait();
  pdl_trigger();
  if (i > d.Nx + 1 || j > d.Ny + 1) return;
  const bool two = k + 1 <= d.Nz + 1;
  const bool hv = j <= d.Ny;
  const int64_t pr = idxR(d, i, j, k), plr = (int64_t)(d.nxg - 2) * (d.nyg - 2);
  const int64_t iu = idxU(d, i, j, k), iv = idxV(d, i, j, k), iw = idxW(d, i, j, k);
  const int64_t plu = (int64_t)d.nx * d.nyg, plv = (int64_t)d.nxg * d.ny, plw = (int64_t)d.nxg * d.nyg;
  const double p0 = __ldg(phi + pr), px = __ldg(phi + pr + 1), p1 = __ldg(phi + pr + plr);
  const double u0 = __ldg(Ui + iu), w0 = __ldg(Wi + iw);
  double py = 0.0, v0 = 0.0, p1x = 0.0, p2 = 0.0, u1 = 0.0, w1 = 0.0, p1y = 0.0, v1 = 0.0;
  if (hv) {
    py = __ldg(phi + pr + (d.nxg - 2));
    v0 = __ldg(Vi + iv);
  }
  if (two) {
    p1x = __ldg(phi + pr + plr + 1);
    p2 = __ldg(phi + pr + 2 * plr);
    u1 = __ldg(Ui + iu + plu);
    w1 = __ldg(Wi + iw + plw);
    if (hv) {
      p1y = __ldg(phi + pr + plr + (d.nxg - 2));
      v1 = __ldg(Vi + iv + plv);
    }
  }
  const double rx = m.rdxg[i], ry = m.rdyg[j];
  double un0 = u0 - (px - p0) * rx;
  const double wn0 = w0 - (p1 - p0) * m.rdzg[k], vn0 = v0 - (py - p0) * ry;
  double un1 = u1 - (p1x - p1) * rx;
  const double wn1 = w1 - (p2 - p1) * m.rdzg[k + 1], vn1 = v1 - (p1y - p1) * ry;
  if (ushift) {
    // constant-mass-flow correction of u after the projection
    // (src/time_integration.f90:187-193), ghosts included
    const double sh = *ushift;
    un0 += sh;
    un1 += sh;
  }
  if (!ghosts) {
    Uo[iu] = un0;
    Wo[iw] = wn0;
    if (hv) Vo[iv] = vn0;
    if (two) {
      Uo[iu + plu] = un1;
      Wo[iw + plw] = wn1;
      if (hv) Vo[iv + plv] = vn1;
    }
    return;
  }
  // cells k (c = 0) and k+1 (c = 1)
  const bool yu = j == 2 || j == d.nyg - 1;                 // u, w: odd y reflections
  const bool yv = j == 2 || j == d.Ny;                      // v: next to a zero wall
  const XImages xu = x_images(i, d.Nx, d.nx), xw = x_images(i, d.Nx, d.nxg);
  for (int c = 0; c <= (two ? 1 : 0); ++c) {
    const int kc = k + c;
    const double un = c ? un1 : un0, wn = c ? wn1 : wn0, vn = c ? vn1 : vn0;
    const int64_t ou = iu + c * plu, ow = iw + c * plw, ov = iv + c * plv;
    if (yu || kc == d.Nz + 1 || kc + d.Nz <= d.nzg) put_images_all(Uo, d.nx, d.nyg, d.nzg, d.Nx, d.Nz, false, i, j, kc, un);
    else put_row(Uo + ou - (i - 1), i, xu, un);
    if (yu || kc == d.Nz + 1 || kc + d.Nz <= d.nz) put_images_all(Wo, d.nxg, d.nyg, d.nz, d.Nx, d.Nz, false, i, j, kc, wn);
    else put_row(Wo + ow - (i - 1), i, xw, wn);
    if (hv) {
      if (yv || kc == d.Nz + 1 || kc + d.Nz <= d.nzg) {
        put_images_all(Vo, d.nxg, d.ny, d.nzg, d.Nx, d.Nz, true, i, j, kc, vn);
        if (j == 2) put_images_all(Vo, d.nxg, d.ny, d.nzg, d.Nx, d.Nz, true, i, 1, kc, 0.0);
        if (j == d.Ny) put_images_all(Vo, d.nxg, d.ny, d.nzg, d.Nx, d.Nz, true, i, d.ny, kc, 0.0);
      } else {
        put_row(Vo + ov - (i - 1), i, xw, vn);
      }
    }
  }
}

int launch_gradient_subtract(Handle* h, const double* Ui, const double* Vi, const double* Wi,
                             const double* phi, double dt, double* Uo, double* Vo, double* Wo,
                             bool dup_plane, bool with_ghosts, const double* ushift) {
  const Dims& d = h->d;
  dim3 b(32, 4, 2);
  dim3 g((d.Nx + 31) / 32, (d.Ny + 3) / 4, (d.Nz + 1) / 2);
  double* Pint = (h->ib != nullptr || h->write_pinterim) ? h->P_interim : nullptr;
  if (!dup_plane && !Pint) {
    const dim3 b2(32, 8, 1), g2((d.Nx + 31) / 32, (d.Ny + 7) / 8, (d.Nz + 1) / 2);
    C3D_CUDA_TRY(h, launch_pdl(h->use_pdl, k_grad_sub2, g2, b2, 0, h->stream, d, h->m, Ui, Vi, Wi, phi, Uo, Vo, Wo,
                               with_ghosts ? 1 : 0, ushift));
    C3D_LAUNCH_CHECK(h);
    return 0;
  }
  if (ushift) {
    h->last_error = "mass-flow correction inside the projection needs the time step's update kernel";
    return C3D_ERR_UNSUPPORTED;
  }
  k_grad_sub<<<g, b, 0, h->stream>>>(d, h->m, Ui, Vi, Wi, phi, Uo, Vo, Wo, Pint, 1.0 / dt, dup_plane ? 1 : 0);
  C3D_LAUNCH_CHECK(h);
  return with_ghosts ? launch_fill_ghosts3(h, Uo, Vo, Wo) : 0;
}

// compute_non_IB_projection with U* in (Us,Vs,Ws) and the result in (U,V,W),
// ghosts filled.  FP64: one solve.  Mixed: an FP32 solve, then refinement
// sweeps that solve again for the FP64 residual div(U) and re-project U* with
// the accumulated potential.
int launch_projection_step(Handle* h, int rk_step, double dt, const double* ushift) {
  const bool stage1 = (rk_step == 1 && h->ib == nullptr);
  int rc;
  double* phi = h->rhs_p;
  if (h->poisson_mode == C3D_POISSON_MIXED) {
    // with ushift the first forward transform (of U*) also yields the x
    // mass-flow correction: the flux of the refined projection is still U*'s
    const int sweeps = h->refine_sweeps;
    rc = run_spectral_t<float>(h, true, h->Us, h->Vs, h->Ws, nullptr, h->rhs_p,
                               (stage1 && sweeps == 0) ? h->phi1 : nullptr, 0, 7, 0, -1, ushift ? dt : 0.0);
    if (rc) return rc;
    for (int sw = 1; sw <= sweeps; ++sw) {
      rc = launch_gradient_subtract(h, h->Us, h->Vs, h->Ws, h->rhs_p, dt, h->U, h->V, h->W, false, true);
      if (rc) return rc;
      rc = run_spectral_t<float>(h, true, h->U, h->V, h->W, nullptr, h->rhs_p,
                                 (stage1 && sw == sweeps) ? h->phi1 : nullptr, 1, 7);
      if (rc) return rc;
    }
    h->stats.refinement_sweeps = sweeps;
  } else {
    // with ushift, the forward x FFT also yields the x mass-flow correction
    // (the bulk flux of d(phi)/dx over the periodic uniform x grid is zero,
    // so the flux of the projected u is that of U*).  The stage-1 potential,
    // kept for the pressure (src/poisson.f90:91-99), is solved straight into
    // its own array, which the update then reads: no second copy.
    phi = stage1 ? h->phi1 : h->rhs_p;
    rc = run_spectral_t<double>(h, true, h->Us, h->Vs, h->Ws, nullptr, phi, nullptr, 0, 7, 0, -1,
                                ushift ? dt : 0.0);
    if (rc) return rc;
  }
  if (stage1) { h->P_pending = true; h->P_pending_dt = dt; }
  // the projected fields with all their ghost entries (and the x mass-flow
  // correction when ushift is given)
  return launch_gradient_subtract(h, h->Us, h->Vs, h->Ws, phi, dt, h->U, h->V, h->W, false, true, ushift);
}

// P = phi1/(dt*rk_coef(1,1)) with the copies of src/poisson.f90:92-98
__global__ void k_build_P(Dims d, const double* __restrict__ phi, double* __restrict__ P, double den) {
  const int64_t tot = (int64_t)d.nxg * d.nyg * d.nzg;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i = 1 + (int)(t % d.nxg);
    int j = 1 + (int)((t / d.nxg) % d.nyg);
    int k = 1 + (int)(t / ((int64_t)d.nxg * d.nyg));
    // P(1,:,:)=P(2,:,:), P(nxg,:,:)=P(nxg-1,:,:), same in y and z
    if (i == 1) i = 2;
    if (i == d.nxg) i = d.nxg - 1;
    if (j == 1) j = 2;
    if (j == d.nyg) j = d.nyg - 1;
    if (k == 1) k = 2;
    if (k == d.nzg) k = d.nzg - 1;
    P[t] = phi[idxR(d, i, j, k)] / den;
  }
}

int rebuild_pressure(Handle* h) {
  if (!h->P_pending) return 0;
  const double den = h->P_pending_dt * (8.0 / 15.0);
  k_build_P<<<148 * 8, 256, 0, h->stream>>>(h->d, h->phi1, h->P, den);
  C3D_LAUNCH_CHECK(h);
  h->P_pending = false;
  return 0;
}

int poisson_setup(Handle* h) {
  const Dims& d = h->d;
  SpectralState& S = h->sp;
  FftPasses P;
  if (!make_passes(d.Nx, P) || !make_passes(d.Nz, P)) {
    h->last_error = "nxp and nzp must be products of 2 and 3 (nx_global-2, nz_global-2)";
    return C3D_ERR_PARAM;
  }
  if (d.Nx % 2) {
    h->last_error = "nx_global must be even";
    return C3D_ERR_PARAM;
  }
  if (d.Nx > kMaxNx) {
    h->last_error = "nx_global too large for the x FFT kernels (nx_global - 2 <= 512)";
    return C3D_ERR_UNSUPPORTED;
  }
  int rc;
  if (S.spec == nullptr) {
    S.pz64 = d.Nz;
    if (!choose_cluster<double>(d, S.pz64, S.cs64, S.jc64, S.rs64, S.nt64, S.smem64, S.nw64)) {
      h->last_error = "ny_global too large for one 16-CTA cluster per kx slab";
      return C3D_ERR_UNSUPPORTED;
    }
    if ((rc = make_twiddles(h, d.Nx, &S.twx))) return rc;
    if ((rc = make_twiddles(h, d.Nz, &S.twz))) return rc;
    {
      const FftPasses Px = get_passes(d.Nx, kXMaxR);
      std::vector<int> pos(d.Nx);
      for (int m = 0; m < d.Nx; ++m) pos[m] = dif_k_to_position(m, Px);
      if ((rc = dev_alloc(h, &S.posx, d.Nx))) return rc;
      C3D_CUDA_TRY(h, cudaMemcpy(S.posx, pos.data(), sizeof(int) * d.Nx, cudaMemcpyHostToDevice));
    }
    const int64_t ns = (int64_t)d.Ny * S.pz64 * d.nkx;
    if ((rc = dev_alloc(h, &S.spec, ns))) return rc;
    if ((rc = set_limits<double>(h, S.smem64, S.cs64))) return rc;
    const int64_t nbx = (((int64_t)d.Ny * d.Nz + 1) / 2 + kLinesX - 1) / kLinesX;
    if ((rc = dev_alloc(h, &h->flux_part, nbx))) return rc;
    h->flux_part_len = nbx;
  }
  return build_tri_table(h);
}

int mixed_setup(Handle* h) {
  const Dims& d = h->d;
  SpectralState& S = h->sp;
  if (S.spec32 != nullptr) return 0;
  S.pz32 = d.Nz + (d.Nz & 1);
  if (!choose_cluster<float>(d, S.pz32, S.cs32, S.jc32, S.rs32, S.nt32, S.smem32, S.nw32)) {
    h->last_error = "ny_global too large for the FP32 cluster decomposition";
    return C3D_ERR_UNSUPPORTED;
  }
  int rc;
  if ((rc = make_twiddles(h, d.Nx, &S.twx32))) return rc;
  if ((rc = make_twiddles(h, d.Nz, &S.twz32))) return rc;
  const int64_t ns = (int64_t)d.Ny * S.pz32 * d.nkx;
  if ((rc = dev_alloc(h, &S.spec32, ns))) return rc;
  if ((rc = dev_alloc(h, &S.linesum, (int64_t)d.Ny * d.Nz))) return rc;
  if ((rc = dev_alloc(h, &S.phi00, d.Ny))) return rc;
  if ((rc = set_limits<float>(h, S.smem32, S.cs32))) return rc;
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

void mixed_free(Handle* h) { (void)h; }

}  // namespace c3d
