// On-device diagnostics: compute_statistics (src/statistics.f90:22-148) and
// the reductions of output_monitor (src/monitor.f90:21-110), one domain.
//
// Statistics: with term_1 = interpolate_x(U) = (U(i-1)+U(i))/2 and term_2 =
// interpolate_y(V) = (V(j-1)+V(j))/2 (rows 1 and nyg the negatives of rows 2
// and nyg-1), per y row jj = 1..nyg the sums over i = 2..nxg-2 and
// k = 2..nzg-2 (W: k = 2..nz-1) of term_1, term_2, W, their squares and
// term_1*term_2, divided by (nxg-3)(nzg-3) (W: (nxg-3)(nz-2)); the wall
// derivatives of the mean profiles give utau, wtau and Retau.  Row sums are
// per (row, z chunk) block partials added in chunk order (deterministic).
#include <cmath>
#include <vector>

#include "c3d_internal.cuh"

namespace c3d {

namespace {
constexpr int kStatQ = 7;        // Umean, Vmean, Wmean, U2mean, V2mean, W2mean, UVmean
constexpr int kStatChunks = 12;  // z chunks per y row
constexpr int kStatThreads = 256;
constexpr int kBoxBlocks = 148 * 4;
}  // namespace

__global__ void __launch_bounds__(kStatThreads) k_stat_rows(Dims d, const double* __restrict__ U,
                                                           const double* __restrict__ V,
                                                           const double* __restrict__ W,
                                                           double* __restrict__ part) {
  const int j = 1 + blockIdx.x;
  const int c = blockIdx.y;
  const int ni = d.nxg - 3, nk = d.nzg - 3;
  const int k0 = 2 + (int)((int64_t)c * nk / gridDim.y), k1 = 2 + (int)((int64_t)(c + 1) * nk / gridDim.y);
  double s[kStatQ] = {0, 0, 0, 0, 0, 0, 0};
  for (int t = threadIdx.x; t < ni * (k1 - k0); t += blockDim.x) {
    const int i = 2 + t % ni, k = k0 + t / ni;
    const double t1 = 0.5 * (U[idxU(d, i - 1, j, k)] + U[idxU(d, i, j, k)]);
    double t2;
    if (j == 1) t2 = -(0.5 * (V[idxV(d, i, 1, k)] + V[idxV(d, i, 2, k)]));
    else if (j == d.nyg) t2 = -(0.5 * (V[idxV(d, i, d.nyg - 2, k)] + V[idxV(d, i, d.nyg - 1, k)]));
    else t2 = 0.5 * (V[idxV(d, i, j - 1, k)] + V[idxV(d, i, j, k)]);
    const double w = W[idxW(d, i, j, k)];
    s[0] += t1; s[1] += t2; s[2] += w;
    s[3] += t1 * t1; s[4] += t2 * t2; s[5] += w * w;
    s[6] += t1 * t2;
  }
  __shared__ double red[kStatQ][kStatThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kStatQ; ++q) {
    double v = s[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kStatQ) {
    double v = 0.0;
    for (int w_ = 0; w_ < kStatThreads / 32; ++w_) v += red[threadIdx.x][w_];
    part[((int64_t)(j - 1) * gridDim.y + c) * kStatQ + threadIdx.x] = v;
  }
}

// out[q*nyg + jj-1] = (sum over chunks in order) / count
__global__ void k_stat_final(int nyg, int nch, double cnt_uv, double cnt_w, const double* __restrict__ part,
                             double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nyg * kStatQ) return;
  const int q = t / nyg, j = t - q * nyg;
  double v = 0.0;
  for (int c = 0; c < nch; ++c) v += part[((int64_t)j * nch + c) * kStatQ + q];
  out[t] = v / ((q == 2 || q == 5) ? cnt_w : cnt_uv);
}

// (sum, max) of F(i,j,k) over the box, F of extents (n1, n2, .)
__global__ void __launch_bounds__(256) k_box_sum_max(const double* __restrict__ F, int n1, int n2, int i0, int ni,
                                                    int j0, int nj, int k0, int nk, double2* __restrict__ part) {
  const int64_t tot = (int64_t)ni * nj * nk;
  double s = 0.0, mx = -INFINITY;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = i0 + (int)(t % ni);
    const int j = j0 + (int)((t / ni) % nj);
    const int k = k0 + (int)(t / ((int64_t)ni * nj));
    const double v = F[(int64_t)(i - 1) + (int64_t)n1 * ((j - 1) + (int64_t)n2 * (k - 1))];
    s += v;
    mx = fmax(mx, v);
  }
  __shared__ double ss[8], sm[8];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { ss[wid] = s; sm[wid] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = -INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += ss[w]; b = fmax(b, sm[w]); }
    part[blockIdx.x] = make_double2(a, b);
  }
}

int massflow_w_as_v(Handle* h, double* q_out);

// compute_statistics: profiles[7*nyg] (Umean, Vmean, Wmean, U2mean, V2mean,
// W2mean, UVmean at yg(1:nyg)); scalars[8] = utau, wtau, Retau_u, Retau_w,
// Qflow_x, Qflow_y, Qflow_z, and 1 if U, V or W holds a NaN or infinity
// (the reference stops there, src/statistics.f90:142-144)
int compute_statistics(Handle* h, double* profiles, double* scalars) {
  const Dims& d = h->d;
  const int nyg = d.nyg;
  double* part = nullptr;
  int rc;
  const int64_t need = (int64_t)nyg * kStatChunks * kStatQ + (int64_t)nyg * kStatQ;
  if (h->stat_cap < need) {
    if ((rc = dev_alloc(h, &h->stat_buf, need))) return rc;
    h->stat_cap = need;
  }
  part = h->stat_buf;
  double* out = h->stat_buf + (int64_t)nyg * kStatChunks * kStatQ;
  k_stat_rows<<<dim3((unsigned)nyg, kStatChunks), kStatThreads, 0, h->stream>>>(d, h->U, h->V, h->W, part);
  C3D_LAUNCH_CHECK(h);
  const double cnt = (double)(d.nxg - 3) * (double)(d.nzg - 3), cntw = (double)(d.nxg - 3) * (double)(d.nz - 2);
  k_stat_final<<<(nyg * kStatQ + 127) / 128, 128, 0, h->stream>>>(nyg, kStatChunks, cnt, cntw, part, out);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(profiles, out, sizeof(double) * nyg * kStatQ, cudaMemcpyDeviceToHost,
                                  h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  const double* Um = profiles;
  const double* Wm = profiles + 2 * nyg;
  const std::vector<double>& yg = h->yg;
  const std::vector<double>& y = h->y;
  const double nu = h->p.nu;
  // src/statistics.f90:109-127 (the wall Reynolds stresses are zero)
  const double dUb = (Um[1] - Um[0]) / (yg[2] - yg[1]);
  const double dUt = (Um[nyg - 1] - Um[nyg - 2]) / (yg[nyg] - yg[nyg - 1]);
  const double dWb = (Wm[1] - Wm[0]) / (yg[2] - yg[1]);
  const double dWt = (Wm[nyg - 1] - Wm[nyg - 2]) / (yg[nyg] - yg[nyg - 1]);
  const double utau = std::pow((0.0 - 0.0 - nu * dUt + nu * dUb) / h->Ly, 0.5);
  const double wtau = std::pow((0.0 - 0.0 - nu * dWt + nu * dWb) / h->Ly, 0.5);
  scalars[0] = utau;
  scalars[1] = wtau;
  scalars[2] = utau * (y[d.ny] - y[1]) / 2.0 / nu;
  scalars[3] = wtau * (y[d.ny] - y[1]) / 2.0 / nu;
  // src/statistics.f90:130-133; the z flow is compute_mean_mass_flow_V
  // applied to W, as the reference calls it
  if ((rc = massflow(h, 0, false, &scalars[4]))) return rc;
  if ((rc = massflow(h, 1, false, &scalars[5]))) return rc;
  if ((rc = massflow_w_as_v(h, &scalars[6]))) return rc;
  bool ok = true;
  if ((rc = check_finite(h, &ok))) return rc;
  scalars[7] = ok ? 0.0 : 1.0;
  return 0;
}

static int box_sum_max(Handle* h, const double* F, int n1, int n2, int i0, int i1, int j0, int j1, int k0, int k1,
                       double* sum, double* mx) {
  double2* part = (double2*)h->red;
  k_box_sum_max<<<kBoxBlocks, 256, 0, h->stream>>>(F, n1, n2, i0, i1 - i0 + 1, j0, j1 - j0 + 1, k0, k1 - k0 + 1,
                                                  part);
  C3D_LAUNCH_CHECK(h);
  std::vector<double2> p(kBoxBlocks);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(p.data(), part, sizeof(double2) * kBoxBlocks, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  double s = 0.0, m = -INFINITY;
  for (const double2& v : p) { s += v.x; m = v.y > m ? v.y : m; }
  *sum = s;
  *mx = m;
  return 0;
}

// output_monitor (src/monitor.f90:21-50): out[0..2] mean U, V, W over the
// interior divided by nxm*nym*nzm (as printed, :78-80), out[3..5] their
// maxima, out[6] the maximum |div u| (check_divergence, :210-221)
int monitor_values(Handle* h, double* out) {
  const Dims& d = h->d;
  int rc;
  const double vol = (double)(d.nx - 1) * (double)(d.ny - 1) * (double)(d.nz - 1);
  double s, m;
  if ((rc = box_sum_max(h, h->U, d.nx, d.nyg, 2, d.nx - 1, 2, d.nyg - 1, 2, d.nzg - 1, &s, &m))) return rc;
  out[0] = s / vol; out[3] = m;
  if ((rc = box_sum_max(h, h->V, d.nxg, d.ny, 2, d.nxg - 1, 2, d.ny - 1, 2, d.nzg - 1, &s, &m))) return rc;
  out[1] = s / vol; out[4] = m;
  if ((rc = box_sum_max(h, h->W, d.nxg, d.nyg, 2, d.nxg - 1, 2, d.nyg - 1, 2, d.nz - 1, &s, &m))) return rc;
  out[2] = s / vol; out[5] = m;
  return max_abs_divergence(h, h->U, h->V, h->W, &out[6]);
}

}  // namespace c3d
