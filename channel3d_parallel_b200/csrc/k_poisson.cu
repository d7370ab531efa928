// Pseudo-pressure Poisson solve and projection.
//
// solve_poisson_equation (src/poisson.f90:33-101) restated for one GPU:
//   per y-plane 2-D DFT over (x, z)      -> x real-to-complex FFT of each
//                                           (j, k) line (pairs of real lines
//                                           packed as one complex line) and a
//                                           complex FFT of each (j, kx) z-line;
//   per (kx, kz) tridiagonal in y        -> Thomas elimination with the
//                                           factorisation of every mode
//                                           precomputed once (the matrix is
//                                           fixed: Dyy + kxx + kzz, with the
//                                           00-mode pin D(2) *= 3/2);
//   inverse DFT / (nxp*nzp), real part   -> inverse z FFT, complex-to-real x
//                                           FFT of the Hermitian half spectrum.
// divergence (src/differential_operators.f90:54-74) is fused into the first
// FFT kernel; gradient (:16-52) and the projection update
// (src/projection.f90:22-46) are one kernel.
//
// Spectrum layout in HBM: spec[((j-2)*Nz + (k-2))*nkx + m], m = 0..Nx/2.
#include <cmath>
#include <vector>

#include "c3d_internal.cuh"
#include "fft.cuh"

namespace c3d {

// ---------------------------------------------------------------------------
// host set-up
// ---------------------------------------------------------------------------
static bool make_passes(int n, FftPasses& P) {
  P.n = n;
  P.npass = 0;
  int m = n;
  while (m % 4 == 0 && P.npass < 8) { P.radix[P.npass++] = 4; m /= 4; }
  while (m % 2 == 0 && P.npass < 8) { P.radix[P.npass++] = 2; m /= 2; }
  while (m % 3 == 0 && P.npass < 8) { P.radix[P.npass++] = 3; m /= 3; }
  return m == 1 && n >= 2;
}

static int make_twiddles(Handle* h, int n, double2** out) {
  std::vector<double2> t(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < n; ++m) {
    long double a = -2.0L * pi * (long double)m / (long double)n;
    t[m].x = (double)cosl(a);
    t[m].y = (double)sinl(a);
  }
  double2* d = nullptr;
  int rc = dev_alloc(h, &d, n);
  if (rc) return rc;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(d, t.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, h->stream));
  *out = d;
  return 0;
}

// Thomas factorisation of every mode, exactly the no-pivot path of the
// reference's LAPACK zgtsv call (src/poisson.f90:72): MULT = DL(k)/D(k),
// D(k+1) -= MULT*DU(k).  Stored: mult_j and 1/d'_j.
static int build_tri_table(Handle* h) {
  const Dims& d = h->d;
  const int Ny = d.Ny, nkx = d.nkx, nkzs = d.nkzs;
  const int64_t nt = (int64_t)Ny * nkzs * nkx;
  std::vector<double> rdp(nt), mult(nt);
  std::vector<float> rdp32(nt), mult32(nt);
  std::vector<double> D(Ny);
  std::vector<double> dl(Ny, 0.0), du(Ny, 0.0);
  for (int jj = 0; jj + 1 < Ny; ++jj) {
    dl[jj] = h->Dl[jj + 3];   // Dyy(j+1, j), j = jj+2
    du[jj] = h->Du[jj + 2];   // Dyy(j, j+1)
  }
  for (int kzs = 0; kzs < nkzs; ++kzs) {
    for (int m = 0; m < nkx; ++m) {
      for (int jj = 0; jj < Ny; ++jj) D[jj] = (h->Dd[jj + 2] + h->kxx[m]) + h->kzz[kzs];
      if (m == 0 && kzs == 0) D[0] = 3.0 / 2.0 * D[0];
      for (int jj = 0; jj < Ny; ++jj) {
        const int64_t o = ((int64_t)jj * nkzs + kzs) * nkx + m;
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
  if (h->tri.rdp == nullptr) {
    if ((rc = dev_alloc(h, &h->tri.rdp, nt))) return rc;
    if ((rc = dev_alloc(h, &h->tri.mult, nt))) return rc;
    if ((rc = dev_alloc(h, &h->tri.rdp32, nt))) return rc;
    if ((rc = dev_alloc(h, &h->tri.mult32, nt))) return rc;
    if ((rc = dev_alloc(h, &h->tri.dl, Ny))) return rc;
    if ((rc = dev_alloc(h, &h->tri.du, Ny))) return rc;
    if ((rc = dev_alloc(h, &h->tri.dl32, Ny))) return rc;
    if ((rc = dev_alloc(h, &h->tri.du32, Ny))) return rc;
  }
  std::vector<float> dl32(Ny), du32(Ny);
  for (int jj = 0; jj < Ny; ++jj) { dl32[jj] = (float)dl[jj]; du32[jj] = (float)du[jj]; }
  cudaStream_t s = h->stream;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.rdp, rdp.data(), nt * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.mult, mult.data(), nt * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.rdp32, rdp32.data(), nt * 4, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.mult32, mult32.data(), nt * 4, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.dl, dl.data(), Ny * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.du, du.data(), Ny * 8, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.dl32, dl32.data(), Ny * 4, cudaMemcpyHostToDevice, s));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->tri.du32, du32.data(), Ny * 4, cudaMemcpyHostToDevice, s));
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : C3D_ERR_CUDA;
}

static FftPasses get_passes(int n) {
  FftPasses P{};
  make_passes(n, P);
  return P;
}

// ---------------------------------------------------------------------------
// kernel 1: (divergence |) x real-to-complex FFT of (j, k) lines
// ---------------------------------------------------------------------------
struct XfwdArgs {
  Dims d;
  Metric m;
  const double* __restrict__ U;
  const double* __restrict__ V;
  const double* __restrict__ W;
  const double* __restrict__ rhs;   // FROM_RHS mode input
  double2* __restrict__ spec;
  const double2* __restrict__ tw;
  FftPasses P;
  int lpb;                          // complex lines per block
};

// one complex line = two real lines r = 2p, 2p+1 with r = (j-2) + Ny*(k-2)
template <bool FROM_DIV>
__global__ void __launch_bounds__(256) k_xfft_fwd(XfwdArgs a) {
  extern __shared__ double2 smem[];
  const Dims& d = a.d;
  const int N = d.Nx;
  const int L = a.lpb;
  double2* tw = smem;
  double2* b0 = smem + N;
  double2* b1 = b0 + L * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = a.tw[t];
  const int64_t nreal = (int64_t)d.Ny * d.Nz;
  const int64_t p0 = (int64_t)blockIdx.x * L;   // first complex line
  // gather
  for (int t = threadIdx.x; t < 2 * L * N; t += blockDim.x) {
    const int ii = t % N;
    const int rl = t / N;                       // local real line 0..2L-1
    const int64_t r = 2 * p0 + rl;
    double val = 0.0;
    if (r < nreal) {
      const int j = 2 + (int)(r % d.Ny);
      const int k = 2 + (int)(r / d.Ny);
      const int i = 2 + ii;
      if (FROM_DIV) {
        val = (a.U[idxU(d, i, j, k)] - a.U[idxU(d, i - 1, j, k)]) * a.m.rdx[i]
            + (a.V[idxV(d, i, j, k)] - a.V[idxV(d, i, j - 1, k)]) * a.m.rdy[j]
            + (a.W[idxW(d, i, j, k)] - a.W[idxW(d, i, j, k - 1)]) * a.m.rdz[k];
      } else {
        val = a.rhs[idxR(d, i, j, k)];
      }
    }
    double2& z = b0[(rl >> 1) * N + ii];
    if (rl & 1) z.y = val; else z.x = val;
  }
  __syncthreads();
  double2* res = fft_lines<double, false>(b0, b1, L, tw, a.P);
  // split the two real transforms, write m = 0..N/2
  const int nk = d.nkx;
  for (int t = threadIdx.x; t < L * nk; t += blockDim.x) {
    const int mm = t % nk;
    const int pl = t / nk;
    const int64_t r0 = 2 * (p0 + pl);
    if (r0 >= nreal) continue;
    const double2 Z = res[pl * N + mm];
    const double2 Zr = res[pl * N + ((N - mm) % N)];
    // A = (Z + conj(Zr))/2,  B = (Z - conj(Zr))/(2i)
    double2 A, B;
    A.x = 0.5 * (Z.x + Zr.x);
    A.y = 0.5 * (Z.y - Zr.y);
    const double dx_ = Z.x - Zr.x, dy_ = Z.y + Zr.y;
    B.x = 0.5 * dy_;
    B.y = -0.5 * dx_;
    // spectrum index: line r -> (j-2) = r % Ny, (k-2) = r / Ny
    const int64_t l0 = (r0 % d.Ny) * (int64_t)d.Nz + (r0 / d.Ny);
    const int64_t r1 = r0 + 1;
    const int64_t l1 = (r1 % d.Ny) * (int64_t)d.Nz + (r1 / d.Ny);
    a.spec[l0 * nk + mm] = A;
    if (r1 < nreal) a.spec[l1 * nk + mm] = B;
  }
}

// ---------------------------------------------------------------------------
// kernel 2: complex FFT along z of (j, m) lines, in place in the spectrum
// ---------------------------------------------------------------------------
struct ZfftArgs {
  Dims d;
  double2* spec;
  const double2* tw;
  FftPasses P;
  int mc;   // m values per block
};

template <bool INV>
__global__ void __launch_bounds__(256) k_zfft(ZfftArgs a) {
  extern __shared__ double2 smem[];
  const Dims& d = a.d;
  const int N = d.Nz, nk = d.nkx, MC = a.mc;
  double2* tw = smem;
  double2* b0 = smem + N;
  double2* b1 = b0 + MC * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = a.tw[t];
  const int jj = blockIdx.y;
  const int m0 = blockIdx.x * MC;
  double2* base = a.spec + (int64_t)jj * d.Nz * nk;
  for (int t = threadIdx.x; t < MC * N; t += blockDim.x) {
    const int mm = t % MC;
    const int kk = t / MC;
    double2 v = make_double2(0.0, 0.0);
    if (m0 + mm < nk) v = base[(int64_t)kk * nk + m0 + mm];
    b0[mm * N + kk] = v;
  }
  __syncthreads();
  double2* res = fft_lines<double, INV>(b0, b1, MC, tw, a.P);
  for (int t = threadIdx.x; t < MC * N; t += blockDim.x) {
    const int mm = t % MC;
    const int kk = t / MC;
    if (m0 + mm < nk) base[(int64_t)kk * nk + m0 + mm] = res[mm * N + kk];
  }
}

// ---------------------------------------------------------------------------
// kernel 3: Thomas solve in y for every (kz, m) mode
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_tridiag(Dims d, double2* __restrict__ spec,
                                                 const double* __restrict__ mult,
                                                 const double* __restrict__ rdp,
                                                 const double* __restrict__ du) {
  const int nk = d.nkx;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;   // kz*nk + m
  if (q >= d.Nz * nk) return;
  const int kz = q / nk, m = q - kz * nk;
  const int kzs = kz <= d.Nz - kz ? kz : d.Nz - kz;
  const int64_t sstride = (int64_t)d.Nz * nk;
  const int64_t tstride = (int64_t)d.nkzs * nk;
  const int64_t t0 = (int64_t)kzs * nk + m;
  double2* s = spec + q;
  // forward elimination: B(j+1) -= MULT_j * B(j)
  double2 prev = s[0];
  for (int jj = 1; jj < d.Ny; ++jj) {
    const double mu = __ldg(mult + (jj - 1) * tstride + t0);
    double2 b = s[jj * sstride];
    b.x = b.x - mu * prev.x;
    b.y = b.y - mu * prev.y;
    s[jj * sstride] = b;
    prev = b;
  }
  // back substitution: x(j) = (B(j) - DU(j) x(j+1)) / D'(j)
  const int jl = d.Ny - 1;
  double rd = __ldg(rdp + jl * tstride + t0);
  double2 xn;
  xn.x = prev.x * rd;
  xn.y = prev.y * rd;
  s[jl * sstride] = xn;
  for (int jj = jl - 1; jj >= 0; --jj) {
    const double u = __ldg(du + jj);
    rd = __ldg(rdp + jj * tstride + t0);
    double2 b = s[jj * sstride];
    b.x = (b.x - u * xn.x) * rd;
    b.y = (b.y - u * xn.y) * rd;
    s[jj * sstride] = b;
    xn = b;
  }
}

// ---------------------------------------------------------------------------
// kernel 4: x complex-to-real inverse FFT, write phi into rhs_p layout
// ---------------------------------------------------------------------------
struct XinvArgs {
  Dims d;
  const double2* __restrict__ spec;
  const double2* __restrict__ tw;
  double* __restrict__ rhs;    // output phi (rhs_p layout)
  double* __restrict__ phi1;   // optional second copy (P side effect)
  FftPasses P;
  int lpb;
  double scale_div;            // nxp*nzp
};

__global__ void __launch_bounds__(256) k_xfft_inv(XinvArgs a) {
  extern __shared__ double2 smem[];
  const Dims& d = a.d;
  const int N = d.Nx, L = a.lpb, nk = d.nkx;
  double2* tw = smem;
  double2* b0 = smem + N;
  double2* b1 = b0 + L * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tw[t] = a.tw[t];
  const int64_t nreal = (int64_t)d.Ny * d.Nz;
  const int64_t p0 = (int64_t)blockIdx.x * L;
  // build Z = A + iB on the full circle from the two half spectra
  for (int t = threadIdx.x; t < L * nk; t += blockDim.x) {
    const int mm = t % nk;
    const int pl = t / nk;
    const int64_t r0 = 2 * (p0 + pl), r1 = r0 + 1;
    double2 A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
    if (r0 < nreal) {
      const int64_t l0 = (r0 % d.Ny) * (int64_t)d.Nz + (r0 / d.Ny);
      A = a.spec[l0 * nk + mm];
    }
    if (r1 < nreal) {
      const int64_t l1 = (r1 % d.Ny) * (int64_t)d.Nz + (r1 / d.Ny);
      B = a.spec[l1 * nk + mm];
    }
    if (mm == 0 || 2 * mm == N) { A.y = 0.0; B.y = 0.0; }   // Hermitian projection
    double2 Z;
    Z.x = A.x - B.y;
    Z.y = A.y + B.x;
    b0[pl * N + mm] = Z;
    if (mm > 0 && 2 * mm < N) {
      double2 Zc;
      Zc.x = A.x + B.y;
      Zc.y = -A.y + B.x;
      b0[pl * N + (N - mm)] = Zc;
    }
  }
  __syncthreads();
  double2* res = fft_lines<double, true>(b0, b1, L, tw, a.P);
  const double sd = a.scale_div;
  for (int t = threadIdx.x; t < 2 * L * N; t += blockDim.x) {
    const int ii = t % N;
    const int rl = t / N;
    const int64_t r = 2 * p0 + rl;
    if (r >= nreal) continue;
    const double2 z = res[(rl >> 1) * N + ii];
    const double v = ((rl & 1) ? z.y : z.x) / sd;
    const int j = 2 + (int)(r % d.Ny);
    const int k = 2 + (int)(r / d.Ny);
    const int i = 2 + ii;
    // apply_periodic_xz_centers (src/poisson.f90:106-125): x plane nxg-1 and
    // z plane nzp+2 duplicate plane 2
    a.rhs[idxR(d, i, j, k)] = v;
    if (i == 2) a.rhs[idxR(d, d.Nx + 2, j, k)] = v;
    if (k == 2) {
      a.rhs[idxR(d, i, j, d.Nz + 2)] = v;
      if (i == 2) a.rhs[idxR(d, d.Nx + 2, j, d.Nz + 2)] = v;
    }
    if (a.phi1) {
      a.phi1[idxR(d, i, j, k)] = v;
      if (i == 2) a.phi1[idxR(d, d.Nx + 2, j, k)] = v;
      if (k == 2) {
        a.phi1[idxR(d, i, j, d.Nz + 2)] = v;
        if (i == 2) a.phi1[idxR(d, d.Nx + 2, j, d.Nz + 2)] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
static const int kLinesX = 8;   // complex x-lines per block
static const int kLinesZ = 8;   // z-lines per block

static int set_fft_smem_limits(Handle* h) {
  const Dims& d = h->d;
  const int smx = (int)(sizeof(double2) * (d.Nx + 2 * kLinesX * d.Nx));
  const int smz = (int)(sizeof(double2) * (d.Nz + 2 * kLinesZ * d.Nz));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_xfft_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smx));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_xfft_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smx));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_xfft_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, smx));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_zfft<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smz));
  C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_zfft<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smz));
  return 0;
}

static int run_spectral_parts(Handle* h, bool from_div, const double* U, const double* V,
                              const double* W, double* rhs, double* phi1, int only);

static int run_spectral(Handle* h, bool from_div, const double* U, const double* V,
                        const double* W, double* rhs, double* phi1) {
  return run_spectral_parts(h, from_div, U, V, W, rhs, phi1, -1);
}

int profile_spectral(Handle* h, int part) {
  return run_spectral_parts(h, true, h->Us, h->Vs, h->Ws, h->rhs_p, nullptr, part);
}

static int run_spectral_parts(Handle* h, bool from_div, const double* U, const double* V,
                              const double* W, double* rhs, double* phi1, int only) {
  const Dims& d = h->d;
  cudaStream_t s = h->stream;
  FftPasses Px = get_passes(d.Nx), Pz = get_passes(d.Nz);
  const int64_t npairs = ((int64_t)d.Ny * d.Nz + 1) / 2;
  // 1: div | rhs -> x FFT
  if (only < 0 || only == 0) {
    XfwdArgs a{};
    a.d = d; a.m = h->m; a.U = U; a.V = V; a.W = W; a.rhs = rhs;
    a.spec = h->spec; a.tw = h->fx.tw; a.P = Px; a.lpb = kLinesX;
    const size_t sm = sizeof(double2) * (d.Nx + 2 * kLinesX * d.Nx);
    const unsigned nb = (unsigned)((npairs + kLinesX - 1) / kLinesX);
    if (from_div) {
      k_xfft_fwd<true><<<nb, 128, sm, s>>>(a);
    } else {
      k_xfft_fwd<false><<<nb, 128, sm, s>>>(a);
    }
    C3D_LAUNCH_CHECK(h);
  }
  // 2: z FFT forward
  ZfftArgs za{};
  za.d = d; za.spec = h->spec; za.tw = h->fz.tw; za.P = Pz; za.mc = kLinesZ;
  const size_t smz = sizeof(double2) * (d.Nz + 2 * kLinesZ * d.Nz);
  dim3 gz((d.nkx + kLinesZ - 1) / kLinesZ, d.Ny);
  if (only < 0 || only == 1) {
    k_zfft<false><<<gz, 128, smz, s>>>(za);
    C3D_LAUNCH_CHECK(h);
  }
  // 3: tridiagonal
  if (only < 0 || only == 2) {
    const int nm = d.Nz * d.nkx;
    k_tridiag<<<(nm + 127) / 128, 128, 0, s>>>(d, h->spec, h->tri.mult, h->tri.rdp, h->tri.du);
    C3D_LAUNCH_CHECK(h);
  }
  // 4: z FFT inverse
  if (only < 0 || only == 3) {
    k_zfft<true><<<gz, 128, smz, s>>>(za);
    C3D_LAUNCH_CHECK(h);
  }
  // 5: x inverse FFT -> phi
  if (only < 0 || only == 4) {
    XinvArgs a{};
    a.d = d; a.spec = h->spec; a.tw = h->fx.tw; a.rhs = rhs; a.phi1 = phi1;
    a.P = Px; a.lpb = kLinesX; a.scale_div = (double)d.Nx * (double)d.Nz;
    const size_t sm = sizeof(double2) * (d.Nx + 2 * kLinesX * d.Nx);
    const unsigned nb = (unsigned)((npairs + kLinesX - 1) / kLinesX);
    k_xfft_inv<<<nb, 128, sm, s>>>(a);
    C3D_LAUNCH_CHECK(h);
  }
  if (only < 0) h->stats.poisson_solves++;
  return 0;
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

int launch_poisson_solve(Handle* h, double* rhs, int rk_step, double dt) {
  (void)dt;
  int rc = run_spectral(h, false, nullptr, nullptr, nullptr, rhs, rk_step == 1 ? h->phi1 : nullptr);
  if (rc) return rc;
  if (rk_step == 1) { h->P_pending = true; h->P_pending_dt = dt; }
  return 0;
}

// ---------------------------------------------------------------------------
// projection: U = Ui - G phi at interior points (src/projection.f90:40-44),
// optional P_interim = phi/dt; ghosts are filled by the caller
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_grad_sub(Dims d, Metric m, const double* __restrict__ Ui,
                                                  const double* __restrict__ Vi,
                                                  const double* __restrict__ Wi,
                                                  const double* __restrict__ phi,
                                                  double* __restrict__ Uo, double* __restrict__ Vo,
                                                  double* __restrict__ Wo,
                                                  double* __restrict__ Pint, double rdt) {
  const int i = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 2 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.Nx + 1 || j > d.Ny + 1 || k > d.Nz + 1) return;
  const double p0 = __ldg(phi + idxR(d, i, j, k));
  const double px = __ldg(phi + idxR(d, i + 1, j, k));
  const double pz = __ldg(phi + idxR(d, i, j, k + 1));
  const int64_t iu = idxU(d, i, j, k), iw = idxW(d, i, j, k);
  Uo[iu] = __ldg(Ui + iu) - (px - p0) * m.rdxg[i];
  Wo[iw] = __ldg(Wi + iw) - (pz - p0) * m.rdzg[k];
  double py = 0.0;
  if (j <= d.Ny) {
    py = __ldg(phi + idxR(d, i, j + 1, k));
    const int64_t iv = idxV(d, i, j, k);
    Vo[iv] = __ldg(Vi + iv) - (py - p0) * m.rdyg[j];
  }
  if (k == 2) {
    // the reference's gradient also covers plane nzg-1 (the duplicate of
    // plane 2) for the x and y components (src/differential_operators.f90:38-52)
    const int kd = d.Nz + 2;
    const int64_t iud = idxU(d, i, j, kd);
    Uo[iud] = __ldg(Ui + iud) - (px - p0) * m.rdxg[i];
    if (j <= d.Ny) {
      const int64_t ivd = idxV(d, i, j, kd);
      Vo[ivd] = __ldg(Vi + ivd) - (py - p0) * m.rdyg[j];
    }
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

int launch_gradient_subtract(Handle* h, const double* Ui, const double* Vi, const double* Wi,
                             const double* phi, double dt, double* Uo, double* Vo, double* Wo) {
  const Dims& d = h->d;
  dim3 b(32, 4, 2);
  dim3 g((d.Nx + 31) / 32, (d.Ny + 3) / 4, (d.Nz + 1) / 2);
  double* Pint = (h->ib != nullptr || h->write_pinterim) ? h->P_interim : nullptr;
  k_grad_sub<<<g, b, 0, h->stream>>>(d, h->m, Ui, Vi, Wi, phi, Uo, Vo, Wo, Pint, 1.0 / dt);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// compute_non_IB_projection with U* in (Us,Vs,Ws) and the result in (U,V,W),
// ghosts filled: one div+FFT, z FFT, Thomas, z iFFT, iFFT, gradient, BC.
int launch_projection_step(Handle* h, int rk_step, double dt) {
  int rc = run_spectral(h, true, h->Us, h->Vs, h->Ws, h->rhs_p,
                        (rk_step == 1 && h->ib == nullptr) ? h->phi1 : nullptr);
  if (rc) return rc;
  if (rk_step == 1 && h->ib == nullptr) { h->P_pending = true; h->P_pending_dt = dt; }
  rc = launch_gradient_subtract(h, h->Us, h->Vs, h->Ws, h->rhs_p, dt, h->U, h->V, h->W);
  if (rc) return rc;
  return launch_fill_ghosts3(h, h->U, h->V, h->W);
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
  FftPasses P;
  if (!make_passes(d.Nx, P) || !make_passes(d.Nz, P)) {
    h->last_error = "nxp and nzp must be products of 2 and 3 (nx_global-2, nz_global-2)";
    return C3D_ERR_PARAM;
  }
  if (d.Nx % 2) {
    h->last_error = "nx_global must be even";
    return C3D_ERR_PARAM;
  }
  int rc;
  if (h->spec == nullptr) {
    h->fx.n = d.Nx;
    h->fz.n = d.Nz;
    if ((rc = make_twiddles(h, d.Nx, &h->fx.tw))) return rc;
    if ((rc = make_twiddles(h, d.Nz, &h->fz.tw))) return rc;
    const int64_t ns = (int64_t)d.Ny * d.Nz * d.nkx;
    if ((rc = dev_alloc(h, &h->spec, ns))) return rc;
    if ((rc = set_fft_smem_limits(h))) return rc;
  }
  return build_tri_table(h);
}


int mixed_setup(Handle* h) { (void)h; return 0; }
void mixed_free(Handle* h) { (void)h; }

}  // namespace c3d
