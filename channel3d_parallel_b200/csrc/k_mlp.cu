// Learned preconditioner / warm start for the BiCGSTAB Schur solve of the IB
// forces (the solve itself: compute_IB_projection / bicgstab,
// src/projection.f90:48-186; the reference has no preconditioner).
//
// Model.  For marker b the preconditioner is a 4x4 block acting on the
// marker's residual components r_b = (r[b], r[nb+b], r[2nb+b], r[3nb+b]):
//   z_b = A_b r_b,   A_b = diag(sig_e) Ahat(g_b) diag(1/sig_r),
// where g_b are 32 geometry features of the marker (position within the
// staggered cells, normal, surface element, spacing ratios, wall distance)
// and Ahat is the output of an MLP 32 -> 128 -> 128 -> 16 (ReLU), BF16
// weights and activations, FP32 accumulation on the tensor cores.  The
// preconditioner is linear in r, so BiCGSTAB keeps its usual form.
//
// Training data.  While collection is on, every iterate (x_k, r_k) of a
// converged solve is kept; afterwards e_k = x* - x_k solves S e_k = r_k, and
// with rh = r_k/|r_k|, eh = e_k/|r_k| each marker accumulates the moments
//   Crr = sum rh rh^T,  Cer = sum eh rh^T,  Cee = diag sum eh eh^T.
// The least-squares loss of A_b over all pairs is then
//   L = sum_b tr(A Crr A^T) - 2 tr(A Cer^T) + tr(Cee),
// normalised by sum_b tr(Cee); dL/dA = 2 (A Crr - Cer).  One geometry (one
// solve) forms one training set of nb markers.
//
// Kernels.  k_mlp_fwd: one CTA per 128 markers, three tcgen05.mma GEMMs
// (M = 128 markers) with operands in shared memory (K-major, no swizzle) and
// the accumulator in tensor memory.  k_mlp_bwd: persistent CTAs, per tile the
// data-gradient GEMMs dH2 = dO W3, dH1 = dZ2 W2 (K-major) and the weight
// gradients dW3^T = H2^T dO, dW2 = dZ2^T H1, dW1 = dZ1^T X (MN-major
// operands, K = markers) accumulated in tensor memory across tiles.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "bulk.cuh"
#include "c3d_internal.cuh"
#include "ib_state.cuh"

namespace c3d {

constexpr int kF = 32;    // features
constexpr int kH = 128;   // hidden width
constexpr int kO = 16;    // outputs (4x4 block)
constexpr int kTile = 128;
constexpr int kMom = 36;  // Crr(16), Cer(16), Cee diag(4)
// packed parameters: W1[H][F], b1[H], W2[H][H], b2[H], W3[O][H], b3[O]
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kF, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kO * kH, kNParam = kOffB3 + kO;
// packed BF16 operand copies: W1[H][F], W2[H][H], W3[O][H], W2t[H][H], W3t[H][O]
constexpr int kBW1 = 0, kBW2 = kBW1 + kH * kF, kBW3 = kBW2 + kH * kH, kBW2t = kBW3 + kO * kH,
              kBW3t = kBW2t + kH * kH, kNBf = kBW3t + kH * kO;

struct MlpState {
  float* w = nullptr;        // master parameters (FP32)
  float* g = nullptr;        // gradients
  float* m = nullptr;        // Adam moments
  float* v = nullptr;
  __nv_bfloat16* wb = nullptr;   // BF16 operand copies
  float sig_r[4] = {1, 1, 1, 1}, sig_e[4] = {1, 1, 1, 1};
  int adam_t = 0;
  bool trained = false;
  // training sets
  int nb = 0, cap_sets = 0, nsets = 0, next_set = 0;
  __nv_bfloat16* feats = nullptr;   // [cap_sets*nb][F]
  float* mom = nullptr;             // [cap_sets*nb][36]
  // training scratch
  int cap_rows = 0;
  __nv_bfloat16 *H1 = nullptr, *H2 = nullptr, *dO = nullptr;
  float* out = nullptr;             // [rows][O]
  double* lossacc = nullptr;        // [2]: loss, normaliser
  // collection
  bool collecting = false;
  int max_store = 0;
  double *xs = nullptr, *rs = nullptr, *rn = nullptr;   // stored iterates and |r_k|
  int64_t pairs = 0;
  int kind = -1;                    // pairs of the sets: 0 solver iterates, 1 probes (SPAI target)
  double last_loss = -1.0;
  int epochs = 0;
  // inference scratch
  __nv_bfloat16* fq = nullptr;      // [nb][F]
  float* oq = nullptr;              // [nb][O]
  int* err = nullptr;               // device error flag (bounded waits)
  float* sig_d = nullptr;           // sig_r, sig_e on the device
  // caller-data evaluation scratch
  int eval_cap = 0;
  __nv_bfloat16* eval_f = nullptr;
  float* eval_m = nullptr;
};

// ---------------------------------------------------------------------------
// tcgen05 helpers (inline PTX)
// ---------------------------------------------------------------------------
// byte offset of element (row, col) of a [rows][C] BF16 matrix stored as
// 8x8 core matrices (8 rows of 16 bytes, 128 contiguous bytes), core (g, c)
// at (g*(C/8) + c)*128
__device__ __forceinline__ int core_off(int row, int col, int C) {
  return (((row >> 3) * (C >> 3) + (col >> 3)) << 7) + ((row & 7) << 4) + ((col & 7) << 1);
}

// shared-memory matrix descriptor, no swizzle: lbo = stride between core
// matrices along K, sbo = stride between core matrices along M/N (bytes)
__device__ __forceinline__ uint64_t make_sdesc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = smem_addr(p);
  return ((a >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> FP32, M x N, operand majors
__host__ __device__ constexpr uint32_t make_idesc(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// copy a row-major [R][C] BF16 matrix (global) into the core layout
__device__ __forceinline__ void load_core(unsigned char* dst, const __nv_bfloat16* src, int R, int C, int rows_valid) {
  const int cpr = C >> 3;
  for (int t = threadIdx.x; t < R * cpr; t += blockDim.x) {
    const int row = t / cpr, ch = t - row * cpr;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (row < rows_valid) v = *reinterpret_cast<const uint4*>(src + (size_t)row * C + ch * 8);
    *reinterpret_cast<uint4*>(dst + core_off(row, ch * 8, C)) = v;
  }
}

// store 8 consecutive BF16 values of one row into the core layout
__device__ __forceinline__ void store_core8(unsigned char* dst, int row, int col, int C, const float* v) {
  __align__(16) __nv_bfloat16 b[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) b[q] = __float2bfloat16_rn(v[q]);
  *reinterpret_cast<uint4*>(dst + core_off(row, col, C)) = *reinterpret_cast<const uint4*>(b);
}

// K-major operand [rows][K] at K offset k0 (multiple of 16)
__device__ __forceinline__ uint64_t desc_k(const unsigned char* base, int K, int k0) {
  return make_sdesc(base + (k0 >> 3) * 128, 128u, (uint32_t)(K >> 3) * 128u);
}
// MN-major operand: matrix stored [rows = K][C = MN]; K offset k0 (rows)
__device__ __forceinline__ uint64_t desc_mn(const unsigned char* base, int C, int k0) {
  return make_sdesc(base + (k0 >> 3) * (C >> 3) * 128, (uint32_t)(C >> 3) * 128u, 128u);
}

// bounded wait on an mbarrier phase; records an error instead of hanging
__device__ __forceinline__ bool mma_wait(uint64_t* bar, unsigned phase, int* err) {
  const bool ok = mbar_wait(bar, phase, kWaitCycles);
  if (!ok) atomicExch(err, 1);
  return ok;
}

// ---------------------------------------------------------------------------
// forward: O = W3 relu(W2 relu(W1 x + b1) + b2) + b3 for 128 rows per CTA
// ---------------------------------------------------------------------------
struct FwdArgs {
  const __nv_bfloat16* X;   // [M][F]
  const __nv_bfloat16* wb;  // packed BF16 weights
  const float* w;           // master parameters (biases)
  float* out;               // [M][O]
  __nv_bfloat16* H1;        // [M][H] (training) or null
  __nv_bfloat16* H2;
  int M;
  int* err;
};

constexpr int kFwdSmem = kTile * kF * 2 + kH * kF * 2 + kH * kH * 2 + kO * kH * 2 + 2 * kTile * kH * 2 +
                         (2 * kH + kO) * 4;

__global__ void __launch_bounds__(kTile, 1) k_mlp_fwd(FwdArgs a) {
  extern __shared__ __align__(128) unsigned char fsm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tbase;
  unsigned char* sX = fsm;
  unsigned char* sW1 = sX + kTile * kF * 2;
  unsigned char* sW2 = sW1 + kH * kF * 2;
  unsigned char* sW3 = sW2 + kH * kH * 2;
  unsigned char* sH1 = sW3 + kO * kH * 2;
  unsigned char* sH2 = sH1 + kTile * kH * 2;
  float* sb = reinterpret_cast<float*>(sH2 + kTile * kH * 2);   // b1, b2, b3
  const int tid = threadIdx.x;
  const int m0 = blockIdx.x * kTile;
  const int rows = min(kTile, a.M - m0);
  if (tid < 32) tmem_alloc(&tbase, kH);
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  load_core(sX, a.X + (size_t)m0 * kF, kTile, kF, rows);
  load_core(sW1, a.wb + kBW1, kH, kF, kH);
  load_core(sW2, a.wb + kBW2, kH, kH, kH);
  load_core(sW3, a.wb + kBW3, kO, kH, kO);
  for (int t = tid; t < kH; t += blockDim.x) { sb[t] = a.w[kOffB1 + t]; sb[kH + t] = a.w[kOffB2 + t]; }
  for (int t = tid; t < kO; t += blockDim.x) sb[2 * kH + t] = a.w[kOffB3 + t];
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tbase;
  const uint32_t lane_base = tm + ((uint32_t)(tid & ~31) << 16);   // this warp's 32 lanes
  unsigned phase = 0;
  bool ok = true;
  // layer 1: D = X W1^T (K = 32)
  if (tid == 0) {
    for (int k = 0; k < kF; k += 16)
      umma(tm, desc_k(sX, kF, k), desc_k(sW1, kF, k), make_idesc(128, kH, false, false), k > 0);
    umma_commit(&bar);
  }
  ok = mma_wait(&bar, phase, a.err) && ok;
  phase ^= 1;
  tc_fence_after();
  for (int c0 = 0; c0 < kH; c0 += 16) {
    float v[16];
    tmem_ld16(lane_base + c0, v);
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = fmaxf(v[q] + sb[c0 + q], 0.f);
    store_core8(sH1, tid, c0, kH, v);
    store_core8(sH1, tid, c0 + 8, kH, v + 8);
  }
  if (a.H1 && tid < rows)
    for (int c = 0; c < kH; c += 8)
      *reinterpret_cast<uint4*>(a.H1 + (size_t)(m0 + tid) * kH + c) =
          *reinterpret_cast<const uint4*>(sH1 + core_off(tid, c, kH));
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // layer 2: D = H1 W2^T (K = 128)
  if (tid == 0) {
    for (int k = 0; k < kH; k += 16)
      umma(tm, desc_k(sH1, kH, k), desc_k(sW2, kH, k), make_idesc(128, kH, false, false), k > 0);
    umma_commit(&bar);
  }
  ok = mma_wait(&bar, phase, a.err) && ok;
  phase ^= 1;
  tc_fence_after();
  for (int c0 = 0; c0 < kH; c0 += 16) {
    float v[16];
    tmem_ld16(lane_base + c0, v);
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = fmaxf(v[q] + sb[kH + c0 + q], 0.f);
    store_core8(sH2, tid, c0, kH, v);
    store_core8(sH2, tid, c0 + 8, kH, v + 8);
  }
  if (a.H2 && tid < rows)
    for (int c = 0; c < kH; c += 8)
      *reinterpret_cast<uint4*>(a.H2 + (size_t)(m0 + tid) * kH + c) =
          *reinterpret_cast<const uint4*>(sH2 + core_off(tid, c, kH));
  fence_async_shared();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // layer 3: D = H2 W3^T (K = 128, N = 16)
  if (tid == 0) {
    for (int k = 0; k < kH; k += 16)
      umma(tm, desc_k(sH2, kH, k), desc_k(sW3, kH, k), make_idesc(128, kO, false, false), k > 0);
    umma_commit(&bar);
  }
  ok = mma_wait(&bar, phase, a.err) && ok;
  tc_fence_after();
  {
    float v[16];
    tmem_ld16(lane_base, v);
    if (tid < rows && ok)
      for (int q = 0; q < kO; ++q) a.out[(size_t)(m0 + tid) * kO + q] = v[q] + sb[2 * kH + q];
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) tmem_free(tm, kH);
}

// ---------------------------------------------------------------------------
// loss: per row, Ahat = out (4x4, row-major); moments normalised by sig
// ---------------------------------------------------------------------------
__global__ void k_mlp_loss(const float* __restrict__ out, const float* __restrict__ mom, int M,
                           const float* __restrict__ sig, __nv_bfloat16* __restrict__ dO,
                           double* __restrict__ acc) {
  // sig[0..3] = sig_r, sig[4..7] = sig_e
  double lsum = 0.0, nsum = 0.0;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < M; b += gridDim.x * blockDim.x) {
    const float* mb = mom + (size_t)b * kMom;
    float A[16], Crr[16], Cer[16], G[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) A[q] = out[(size_t)b * kO + q];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        Crr[4 * i + j] = mb[4 * i + j] / (sig[i] * sig[j]);
        Cer[4 * i + j] = mb[16 + 4 * i + j] / (sig[4 + i] * sig[j]);
      }
    float tee = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) tee += mb[32 + i] / (sig[4 + i] * sig[4 + i]);
    // AC = A Crr;  L = tr(AC A^T) - 2 tr(A Cer^T) + tr(Cee);  G = 2 (AC - Cer)
    float L = tee;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float ac = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) ac += A[4 * i + k] * Crr[4 * k + j];
        L += ac * A[4 * i + j] - 2.f * A[4 * i + j] * Cer[4 * i + j];
        G[4 * i + j] = 2.f * (ac - Cer[4 * i + j]);
      }
    lsum += L;
    nsum += tee;
#pragma unroll
    for (int q = 0; q < 16; ++q) dO[(size_t)b * kO + q] = __float2bfloat16_rn(G[q]);
  }
  __shared__ double sl[256], sn[256];
  sl[threadIdx.x] = lsum;
  sn[threadIdx.x] = nsum;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) { sl[threadIdx.x] += sl[threadIdx.x + st]; sn[threadIdx.x] += sn[threadIdx.x + st]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { atomicAdd(acc, sl[0]); atomicAdd(acc + 1, sn[0]); }
}

// ---------------------------------------------------------------------------
// backward (persistent): gradients of sum_b L_b w.r.t. all parameters
// ---------------------------------------------------------------------------
struct BwdArgs {
  const __nv_bfloat16* X;
  const __nv_bfloat16* H1;
  const __nv_bfloat16* H2;
  const __nv_bfloat16* dO;
  const __nv_bfloat16* wb;
  float* g;                 // gradients (accumulated)
  int M;
  int* err;
};

constexpr int kBwdSmem = kH * kH * 2 + kH * kO * 2 + kTile * kF * 2 + 4 * kTile * kH * 2 + kTile * kO * 2 +
                         (2 * kH + kO) * 4;
constexpr uint32_t kColWork = 0, kColW2 = 128, kColW1 = 256, kColW3 = 288, kBwdCols = 512;

__global__ void __launch_bounds__(kTile, 1) k_mlp_bwd(BwdArgs a) {
  extern __shared__ __align__(128) unsigned char bsm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tbase;
  unsigned char* sW2t = bsm;
  unsigned char* sW3t = sW2t + kH * kH * 2;
  unsigned char* sX = sW3t + kH * kO * 2;
  unsigned char* sH1 = sX + kTile * kF * 2;
  unsigned char* sH2 = sH1 + kTile * kH * 2;
  unsigned char* sZ2 = sH2 + kTile * kH * 2;
  unsigned char* sZ1 = sZ2 + kTile * kH * 2;
  unsigned char* sdO = sZ1 + kTile * kH * 2;
  float* sdb = reinterpret_cast<float*>(sdO + kTile * kO * 2);   // db1, db2, db3
  const int tid = threadIdx.x;
  if (tid < 32) tmem_alloc(&tbase, kBwdCols);
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  for (int t = tid; t < 2 * kH + kO; t += blockDim.x) sdb[t] = 0.f;
  load_core(sW2t, a.wb + kBW2t, kH, kH, kH);
  load_core(sW3t, a.wb + kBW3t, kH, kO, kH);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tbase;
  const uint32_t lane_base = tm + ((uint32_t)(tid & ~31) << 16);
  unsigned phase = 0;
  bool ok = true;
  bool first = true;
  const int ntiles = (a.M + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int m0 = tile * kTile;
    const int rows = min(kTile, a.M - m0);
    load_core(sX, a.X + (size_t)m0 * kF, kTile, kF, rows);
    load_core(sH1, a.H1 + (size_t)m0 * kH, kTile, kH, rows);
    load_core(sH2, a.H2 + (size_t)m0 * kH, kTile, kH, rows);
    load_core(sdO, a.dO + (size_t)m0 * kO, kTile, kO, rows);
    if (tid < rows)
      for (int q = 0; q < kO; ++q) atomicAdd(&sdb[2 * kH + q], __bfloat162float(a.dO[(size_t)(m0 + tid) * kO + q]));
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      // dH2 = dO W3: A = dO [rows][16] K-major, B = W3^T [in][out] K-major (K = 16)
      umma(tm + kColWork, desc_k(sdO, kO, 0), desc_k(sW3t, kO, 0), make_idesc(128, kH, false, false), 0);
      // dW3^T += H2^T dO: A = H2 (M = in, K = rows) MN-major, B = dO (N = out) MN-major
      for (int k = 0; k < kTile; k += 16)
        umma(tm + kColW3, desc_mn(sH2, kH, k), desc_mn(sdO, kO, k), make_idesc(128, kO, true, true),
             (first && k == 0) ? 0u : 1u);
      umma_commit(&bar);
    }
    ok = mma_wait(&bar, phase, a.err) && ok;
    phase ^= 1;
    tc_fence_after();
    for (int c0 = 0; c0 < kH; c0 += 16) {
      float v[16];
      tmem_ld16(lane_base + kColWork + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h2 = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(sH2 + core_off(tid, c0 + q, kH)));
        v[q] = h2 > 0.f ? v[q] : 0.f;
      }
      store_core8(sZ2, tid, c0, kH, v);
      store_core8(sZ2, tid, c0 + 8, kH, v + 8);
      if (tid < rows)
        for (int q = 0; q < 16; ++q) atomicAdd(&sdb[kH + c0 + q], v[q]);
    }
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      // dH1 = dZ2 W2: A = dZ2 K-major (K = out), B = W2^T [in][out] K-major
      for (int k = 0; k < kH; k += 16)
        umma(tm + kColWork, desc_k(sZ2, kH, k), desc_k(sW2t, kH, k), make_idesc(128, kH, false, false), k > 0);
      // dW2 += dZ2^T H1: A = dZ2 (M = out) MN-major, B = H1 (N = in) MN-major
      for (int k = 0; k < kTile; k += 16)
        umma(tm + kColW2, desc_mn(sZ2, kH, k), desc_mn(sH1, kH, k), make_idesc(128, kH, true, true),
             (first && k == 0) ? 0u : 1u);
      umma_commit(&bar);
    }
    ok = mma_wait(&bar, phase, a.err) && ok;
    phase ^= 1;
    tc_fence_after();
    for (int c0 = 0; c0 < kH; c0 += 16) {
      float v[16];
      tmem_ld16(lane_base + kColWork + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h1 = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(sH1 + core_off(tid, c0 + q, kH)));
        v[q] = h1 > 0.f ? v[q] : 0.f;
      }
      store_core8(sZ1, tid, c0, kH, v);
      store_core8(sZ1, tid, c0 + 8, kH, v + 8);
      if (tid < rows)
        for (int q = 0; q < 16; ++q) atomicAdd(&sdb[c0 + q], v[q]);
    }
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      // dW1 += dZ1^T X: A = dZ1 (M = out) MN-major, B = X (N = in = 32) MN-major
      for (int k = 0; k < kTile; k += 16)
        umma(tm + kColW1, desc_mn(sZ1, kH, k), desc_mn(sX, kF, k), make_idesc(128, kF, true, true),
             (first && k == 0) ? 0u : 1u);
      umma_commit(&bar);
    }
    ok = mma_wait(&bar, phase, a.err) && ok;
    phase ^= 1;
    tc_fence_after();
    tc_fence_before();
    __syncthreads();
    first = false;
  }
  // accumulated weight gradients -> global (lane = output row); the flag is
  // made block-uniform so that the aligned TMEM loads run in whole warps
  ok = __syncthreads_and(ok ? 1 : 0) != 0;
  if (!first && ok) {
    for (int c0 = 0; c0 < kH; c0 += 16) {
      float v[16];
      tmem_ld16(lane_base + kColW2 + c0, v);
      for (int q = 0; q < 16; ++q) atomicAdd(&a.g[kOffW2 + tid * kH + c0 + q], v[q]);
    }
    for (int c0 = 0; c0 < kF; c0 += 16) {
      float v[16];
      tmem_ld16(lane_base + kColW1 + c0, v);
      for (int q = 0; q < 16; ++q) atomicAdd(&a.g[kOffW1 + tid * kF + c0 + q], v[q]);
    }
    {
      float v[16];
      tmem_ld16(lane_base + kColW3, v);    // lane = in, columns = out
      for (int q = 0; q < kO; ++q) atomicAdd(&a.g[kOffW3 + q * kH + tid], v[q]);
    }
  }
  __syncthreads();
  for (int t = tid; t < kH; t += blockDim.x) {
    atomicAdd(&a.g[kOffB1 + t], sdb[t]);
    atomicAdd(&a.g[kOffB2 + t], sdb[kH + t]);
  }
  for (int t = tid; t < kO; t += blockDim.x) atomicAdd(&a.g[kOffB3 + t], sdb[2 * kH + t]);
  tc_fence_before();
  __syncthreads();
  if (tid < 32) tmem_free(tm, kBwdCols);
}

// ---------------------------------------------------------------------------
// Adam step on the master parameters, then the BF16 operand copies
// ---------------------------------------------------------------------------
__global__ void k_mlp_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1c, float b2c, float scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNParam; i += gridDim.x * blockDim.x) {
    const float gi = g[i] * scale;
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / b1c) / (sqrtf(vi / b2c) + 1e-8f);
  }
}

__global__ void k_mlp_pack(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kH * kH; i += gridDim.x * blockDim.x) {
    const int o = i / kH, in = i - o * kH;
    wb[kBW2 + i] = __float2bfloat16_rn(w[kOffW2 + i]);
    wb[kBW2t + in * kH + o] = __float2bfloat16_rn(w[kOffW2 + i]);
    if (i < kH * kF) wb[kBW1 + i] = __float2bfloat16_rn(w[kOffW1 + i]);
    if (i < kO * kH) {
      const int o3 = i / kH, i3 = i - o3 * kH;
      wb[kBW3 + i] = __float2bfloat16_rn(w[kOffW3 + i]);
      wb[kBW3t + i3 * kO + o3] = __float2bfloat16_rn(w[kOffW3 + i]);
    }
  }
}

// ---------------------------------------------------------------------------
// geometry features of the markers
// ---------------------------------------------------------------------------
struct FeatArgs {
  const double *xb, *yb, *zb, *nrm, *sb;
  const double* yf;    // y faces, Fortran index 1..ny at yf[0..ny-1]
  int ny, nb;
  double dx, dz, dymin, Ly, dtnu;
  __nv_bfloat16* F;    // [nb][32]
};

__global__ void k_mlp_features(FeatArgs a) {
  const double tp = 6.283185307179586;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < a.nb; b += gridDim.x * blockDim.x) {
    const double x = a.xb[b], y = a.yb[b], z = a.zb[b];
    // y cell containing the marker
    int lo = 0, hi = a.ny - 1;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (a.yf[mid] <= y) lo = mid; else hi = mid;
    }
    const double dyl = a.yf[hi] - a.yf[lo];
    const double fy = (y - a.yf[lo]) / dyl;
    const double fx = x / a.dx - floor(x / a.dx), fz = z / a.dz - floor(z / a.dz);
    const double nx = a.nrm[b], ny = a.nrm[a.nb + b], nz = a.nrm[2 * a.nb + b];
    const double wd = fmax(fmin(y - a.yf[0], a.yf[a.ny - 1] - y), 1e-12);
    float f[kF];
    f[0] = 1.f;
    f[1] = (float)sin(tp * fx); f[2] = (float)cos(tp * fx);
    f[3] = (float)sin(tp * fy); f[4] = (float)cos(tp * fy);
    f[5] = (float)sin(tp * fz); f[6] = (float)cos(tp * fz);
    f[7] = (float)sin(2 * tp * fx); f[8] = (float)cos(2 * tp * fx);
    f[9] = (float)sin(2 * tp * fy); f[10] = (float)cos(2 * tp * fy);
    f[11] = (float)sin(2 * tp * fz); f[12] = (float)cos(2 * tp * fz);
    f[13] = (float)nx; f[14] = (float)ny; f[15] = (float)nz;
    f[16] = (float)(a.sb[b] / (a.dx * a.dz));
    f[17] = (float)(log10(a.dtnu / (a.dymin * a.dymin)) / 10.0);
    f[18] = (float)(a.dx / a.dymin / 10.0);
    f[19] = (float)(a.dz / a.dymin / 10.0);
    f[20] = (float)(dyl / a.dymin);
    f[21] = (float)(wd / a.Ly);
    f[22] = (float)(log(wd / a.dymin) / 5.0);
    f[23] = (float)(nx * nx); f[24] = (float)(ny * ny); f[25] = (float)(nz * nz);
    f[26] = (float)(nx * ny); f[27] = (float)(nx * nz); f[28] = (float)(ny * nz);
    f[29] = 0.f; f[30] = 0.f; f[31] = 0.f;
#pragma unroll
    for (int q = 0; q < kF; ++q) a.F[(size_t)b * kF + q] = __float2bfloat16_rn(f[q]);
  }
}

// A_b = diag(sig_e) Ahat diag(1/sig_r) in FP64 for the solver; networks
// trained on probe pairs predict A = M^T (the SPAI loss in the same form)
__global__ void k_mlp_blocks(const float* __restrict__ out, int nb, const float* __restrict__ sig,
                             int transpose, double* __restrict__ blk) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double a = (double)out[(size_t)b * kO + 4 * i + j] * sig[4 + i] / sig[j];
        if (transpose) blk[16 * (size_t)b + 4 * j + i] = a;
        else blk[16 * (size_t)b + 4 * i + j] = a;
      }
}

// ---------------------------------------------------------------------------
// training-pair moments of one converged solve
// ---------------------------------------------------------------------------
__global__ void k_mlp_rnorm(const double* __restrict__ rs, int64_t n, double* __restrict__ rn) {
  const double* r = rs + (size_t)blockIdx.x * n;
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += r[i] * r[i];
  __shared__ double sa[256];
  sa[threadIdx.x] = acc;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sa[threadIdx.x] += sa[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) rn[blockIdx.x] = sqrt(sa[0]);
}

__global__ void k_mlp_moments(const double* __restrict__ xs, const double* __restrict__ rs,
                              const double* __restrict__ rn, const double* __restrict__ xstar, int nk,
                              double rfinal, int nb, float* __restrict__ mom) {
  const int64_t n = 4 * (int64_t)nb;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double Crr[16] = {0}, Cer[16] = {0}, Cee[4] = {0};
    for (int k = 0; k < nk; ++k) {
      const double nr = rn[k];
      if (!(nr > 100.0 * rfinal) || !(nr > 0.0)) continue;   // x* must be accurate relative to e_k
      double r[4], e[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int64_t i = (int64_t)c * nb + b;
        r[c] = rs[(size_t)k * n + i] / nr;
        e[c] = (xstar[i] - xs[(size_t)k * n + i]) / nr;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          Crr[4 * i + j] += r[i] * r[j];
          Cer[4 * i + j] += e[i] * r[j];
        }
        Cee[i] += e[i] * e[i];
      }
    }
    float* mb = mom + (size_t)b * kMom;
    for (int q = 0; q < 16; ++q) { mb[q] = (float)Crr[q]; mb[16 + q] = (float)Cer[q]; }
    for (int q = 0; q < 4; ++q) mb[32 + q] = (float)Cee[q];
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int mlp_ensure(Handle* h) {
  if (h->mlp) return 0;
  MlpState* M = new MlpState();
  h->mlp = M;
  int rc;
  if ((rc = dev_alloc(h, &M->w, kNParam))) return rc;
  if ((rc = dev_alloc(h, &M->g, kNParam))) return rc;
  if ((rc = dev_alloc(h, &M->m, kNParam))) return rc;
  if ((rc = dev_alloc(h, &M->v, kNParam))) return rc;
  if ((rc = dev_alloc(h, &M->wb, kNBf))) return rc;
  if ((rc = dev_alloc(h, &M->lossacc, 2))) return rc;
  if ((rc = dev_alloc(h, &M->err, 1))) return rc;
  if ((rc = dev_alloc(h, &M->sig_d, 8))) return rc;
  // He-initialised hidden layers, output layer at zero with Ahat = I via b3
  std::vector<float> w(kNParam, 0.f);
  std::mt19937 gen(12345);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int i = 0; i < kH * kF; ++i) w[kOffW1 + i] = nd(gen) * std::sqrt(2.f / kF);
  for (int i = 0; i < kH * kH; ++i) w[kOffW2 + i] = nd(gen) * std::sqrt(2.f / kH);
  for (int i = 0; i < kO * kH; ++i) w[kOffW3 + i] = nd(gen) * 1e-3f;
  for (int i = 0; i < 4; ++i) w[kOffB3 + 5 * i] = 1.f;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(M->w, w.data(), 4 * kNParam, cudaMemcpyHostToDevice, h->stream));
  k_mlp_pack<<<64, 256, 0, h->stream>>>(M->w, M->wb);
  C3D_LAUNCH_CHECK(h);
  static bool attr = false;
  if (!attr) {
    C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem));
    C3D_CUDA_TRY(h, cudaFuncSetAttribute(k_mlp_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kBwdSmem));
    attr = true;
  }
  return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : C3D_ERR_CUDA;
}

static int upload_sig(Handle* h) {
  MlpState* S = h->mlp;
  float sig[8];
  for (int i = 0; i < 4; ++i) { sig[i] = S->sig_r[i]; sig[4 + i] = S->sig_e[i]; }
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S->sig_d, sig, 32, cudaMemcpyHostToDevice, h->stream));
  return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : C3D_ERR_CUDA;
}

void mlp_free(Handle* h) {
  delete h->mlp;   // device buffers are tracked by the handle
  h->mlp = nullptr;
}

static int check_mlp_err(Handle* h) {
  int e = 0;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(&e, h->mlp->err, 4, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (e) {
    h->last_error = "a tensor-core MLP kernel gave up waiting for its MMAs";
    return C3D_ERR_CUDA;
  }
  return 0;
}

static int mlp_forward(Handle* h, const __nv_bfloat16* X, int M, float* out, __nv_bfloat16* H1,
                       __nv_bfloat16* H2) {
  FwdArgs a{};
  a.X = X; a.wb = h->mlp->wb; a.w = h->mlp->w; a.out = out; a.H1 = H1; a.H2 = H2; a.M = M;
  a.err = h->mlp->err;
  k_mlp_fwd<<<(M + kTile - 1) / kTile, kTile, kFwdSmem, h->stream>>>(a);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

// one training pass over M rows: forward, loss and dO, backward into g
static int mlp_train_pass(Handle* h, const __nv_bfloat16* X, const float* mom, int M, const float* sig_d,
                          double* loss, double* norm) {
  MlpState* S = h->mlp;
  int rc;
  if ((rc = mlp_forward(h, X, M, S->out, S->H1, S->H2))) return rc;
  C3D_CUDA_TRY(h, cudaMemsetAsync(S->lossacc, 0, 16, h->stream));
  k_mlp_loss<<<std::min(1184, (M + 255) / 256), 256, 0, h->stream>>>(S->out, mom, M, sig_d, S->dO, S->lossacc);
  C3D_LAUNCH_CHECK(h);
  C3D_CUDA_TRY(h, cudaMemsetAsync(S->g, 0, 4 * kNParam, h->stream));
  BwdArgs b{};
  b.X = X; b.H1 = S->H1; b.H2 = S->H2; b.dO = S->dO; b.wb = S->wb; b.g = S->g; b.M = M; b.err = S->err;
  const int ntiles = (M + kTile - 1) / kTile;
  k_mlp_bwd<<<std::min(148, ntiles), kTile, kBwdSmem, h->stream>>>(b);
  C3D_LAUNCH_CHECK(h);
  double la[2];
  C3D_CUDA_TRY(h, cudaMemcpyAsync(la, S->lossacc, 16, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  *loss = la[0];
  *norm = la[1];
  return check_mlp_err(h);
}

static int ensure_rows(Handle* h, int rows) {
  MlpState* S = h->mlp;
  if (S->cap_rows >= rows) return 0;
  int rc;
  S->cap_rows = rows;
  if ((rc = dev_alloc(h, &S->H1, (int64_t)rows * kH))) return rc;
  if ((rc = dev_alloc(h, &S->H2, (int64_t)rows * kH))) return rc;
  if ((rc = dev_alloc(h, &S->dO, (int64_t)rows * kO))) return rc;
  if ((rc = dev_alloc(h, &S->out, (int64_t)rows * kO))) return rc;
  return 0;
}

static int compute_features(Handle* h, __nv_bfloat16* F, double dt) {
  IbState* s = h->ib;
  FeatArgs a{};
  a.xb = s->xb_d; a.yb = s->yb_d; a.zb = s->zb_d; a.nrm = s->nrm_d; a.sb = s->sb_d;
  a.yf = s->y_d; a.ny = (int)h->y.size(); a.nb = s->nb;
  a.dx = h->dx; a.dz = h->dz; a.dymin = h->dymin; a.Ly = h->p.Ly_channel; a.dtnu = dt * h->p.nu;
  a.F = F;
  k_mlp_features<<<(s->nb + 127) / 128, 128, 0, h->stream>>>(a);
  C3D_LAUNCH_CHECK(h);
  return 0;
}

int mlp_build_blocks(Handle* h, double dt) {
  IbState* s = h->ib;
  int rc;
  if ((rc = mlp_ensure(h))) return rc;
  MlpState* S = h->mlp;
  if (S->nb != s->nb || S->fq == nullptr) {
    if ((rc = dev_alloc(h, &S->fq, (int64_t)s->nb * kF))) return rc;
    if ((rc = dev_alloc(h, &S->oq, (int64_t)s->nb * kO))) return rc;
    S->nb = s->nb;
  }
  if ((rc = compute_features(h, S->fq, dt))) return rc;
  if ((rc = mlp_forward(h, S->fq, s->nb, S->oq, nullptr, nullptr))) return rc;
  if ((rc = upload_sig(h))) return rc;
  k_mlp_blocks<<<(s->nb + 255) / 256, 256, 0, h->stream>>>(S->oq, s->nb, S->sig_d, S->kind == 1 ? 1 : 0,
                                                           s->lrn_blk);
  C3D_LAUNCH_CHECK(h);
  if ((rc = check_mlp_err(h))) return rc;
  s->have_lrn = true;
  return 0;
}

bool mlp_collecting(const Handle* h) { return h->mlp != nullptr && h->mlp->collecting; }

int mlp_store_iterate(Handle* h, const double* x, const double* r, int k) {
  MlpState* S = h->mlp;
  if (k >= S->max_store) return 0;
  const int64_t n = 4 * (int64_t)h->ib->nb;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S->xs + (size_t)k * n, x, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S->rs + (size_t)k * n, r, 8 * n, cudaMemcpyDeviceToDevice, h->stream));
  return 0;
}

int mlp_collect_solve(Handle* h, int stored) {
  MlpState* S = h->mlp;
  IbState* s = h->ib;
  const int nk = std::min(stored, S->max_store);
  if (nk <= 0) return 0;
  const int64_t n = 4 * (int64_t)s->nb;
  k_mlp_rnorm<<<nk, 256, 0, h->stream>>>(S->rs, n, S->rn);
  C3D_LAUNCH_CHECK(h);
  const int set = S->next_set;
  // final residual of this solve: r is in IbState::r
  double* rfin = S->rn + S->max_store;
  k_mlp_rnorm<<<1, 256, 0, h->stream>>>(s->r, n, rfin);
  C3D_LAUNCH_CHECK(h);
  double rf = 0.0;
  std::vector<double> rn(nk);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(&rf, rfin, 8, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(rn.data(), S->rn, 8 * nk, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  int used = 0;
  for (int k = 0; k < nk; ++k) used += (rn[k] > 100.0 * rf && rn[k] > 0.0) ? 1 : 0;
  if (used == 0 || S->kind == 1) return 0;
  S->kind = 0;
  k_mlp_moments<<<(s->nb + 127) / 128, 128, 0, h->stream>>>(S->xs, S->rs, S->rn, s->fb, nk, rf, s->nb,
                                                           S->mom + (size_t)set * s->nb * kMom);
  C3D_LAUNCH_CHECK(h);
  const double dt = h->dt > 0 ? h->dt : (h->p.CFL < 0 ? -h->p.CFL : 1e-3);
  int rc = compute_features(h, S->feats + (size_t)set * s->nb * kF, dt);
  if (rc) return rc;
  S->next_set = (set + 1) % S->cap_sets;
  S->nsets = std::min(S->nsets + 1, S->cap_sets);
  S->pairs += used;
  return 0;
}

}  // namespace c3d

using namespace c3d;


namespace c3d {
Handle* lookup_handle(int id);
}

static int ensure_sets(Handle* h, int max_sets) {
  MlpState* S = h->mlp;
  const int nb = h->ib->nb;
  if (S->feats == nullptr || S->cap_sets != max_sets || S->nb != nb) {
    int rc;
    if ((rc = dev_alloc(h, &S->feats, (int64_t)max_sets * nb * kF))) return rc;
    if ((rc = dev_alloc(h, &S->mom, (int64_t)max_sets * nb * kMom))) return rc;
    S->cap_sets = max_sets;
    S->nsets = 0;
    S->next_set = 0;
    S->pairs = 0;
    S->kind = -1;
    S->nb = nb;
    S->fq = nullptr;
  }
  return 0;
}

extern "C" int c3d_precond_probe(int id) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  cudaSetDevice(h->device);
  if (!h->ib) { h->last_error = "no immersed body: the learned preconditioner acts on IB solves"; return C3D_ERR_UNSUPPORTED; }
  int rc;
  if ((rc = mlp_ensure(h))) return rc;
  MlpState* S = h->mlp;
  if (S->feats == nullptr && (rc = ensure_sets(h, 16))) return rc;
  if (S->kind == 0) { h->last_error = "the collected sets hold iterate pairs; probe pairs cannot be mixed in"; return C3D_ERR_PARAM; }
  const double dt = h->dt > 0 ? h->dt : (h->p.CFL < 0 ? -h->p.CFL : 1e-3);
  const int set = S->next_set;
  if ((rc = ib_probe(h, dt, S->mom + (size_t)set * S->nb * kMom))) return rc;
  if ((rc = compute_features(h, S->feats + (size_t)set * S->nb * kF, dt))) return rc;
  S->kind = 1;
  S->next_set = (set + 1) % S->cap_sets;
  S->nsets = std::min(S->nsets + 1, S->cap_sets);
  S->pairs += 4 * (int64_t)S->nb;
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

extern "C" int c3d_precond_collect(int id, int enable, int max_store, int max_sets) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  cudaSetDevice(h->device);
  if (!h->ib) { h->last_error = "no immersed body: the learned preconditioner acts on IB solves"; return C3D_ERR_UNSUPPORTED; }
  int rc;
  if ((rc = mlp_ensure(h))) return rc;
  MlpState* S = h->mlp;
  if (!enable) { S->collecting = false; return 0; }
  if (max_store < 1 || max_sets < 1) return C3D_ERR_PARAM;
  const int nb = h->ib->nb;
  const int64_t n = 4 * (int64_t)nb;
  if (S->xs == nullptr || S->max_store < max_store) {
    if ((rc = dev_alloc(h, &S->xs, (int64_t)max_store * n))) return rc;
    if ((rc = dev_alloc(h, &S->rs, (int64_t)max_store * n))) return rc;
    if ((rc = dev_alloc(h, &S->rn, (int64_t)max_store + 1))) return rc;
    S->max_store = max_store;
  }
  if ((rc = ensure_sets(h, max_sets))) return rc;
  S->collecting = true;
  return 0;
}

extern "C" int c3d_precond_train(int id, int epochs, double lr, double* final_loss) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  cudaSetDevice(h->device);
  MlpState* S = h->mlp;
  if (!S || S->nsets == 0) { if (h) h->last_error = "no training pairs collected"; return C3D_ERR_PARAM; }
  if (epochs < 1 || !(lr > 0)) return C3D_ERR_PARAM;
  const int M = S->nsets * S->nb;
  int rc;
  if ((rc = ensure_rows(h, M))) return rc;
  // normalisation: sig_r^2 = mean diag Crr, sig_e^2 = mean diag Cee over all markers
  std::vector<float> mom((size_t)M * kMom);
  C3D_CUDA_TRY(h, cudaMemcpyAsync(mom.data(), S->mom, 4 * mom.size(), cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  double sr[4] = {0}, se[4] = {0};
  for (int b = 0; b < M; ++b)
    for (int c = 0; c < 4; ++c) { sr[c] += mom[(size_t)b * kMom + 5 * c]; se[c] += mom[(size_t)b * kMom + 32 + c]; }
  for (int c = 0; c < 4; ++c) {
    S->sig_r[c] = (float)std::sqrt(std::max(sr[c] / M, 1e-30));
    S->sig_e[c] = (float)std::sqrt(std::max(se[c] / M, 1e-30));
  }
  if ((rc = upload_sig(h))) return rc;
  const float* sd = S->sig_d;
  double loss = 0, norm = 1;
  for (int ep = 0; ep < epochs; ++ep) {
    if ((rc = mlp_train_pass(h, S->feats, S->mom, M, sd, &loss, &norm))) return rc;
    ++S->adam_t;
    const float b1c = 1.f - std::pow(0.9f, (float)S->adam_t), b2c = 1.f - std::pow(0.999f, (float)S->adam_t);
    k_mlp_adam<<<(kNParam + 255) / 256, 256, 0, h->stream>>>(S->w, S->g, S->m, S->v, (float)lr, b1c, b2c,
                                                             (float)(1.0 / std::max(norm, 1e-300)));
    C3D_LAUNCH_CHECK(h);
    k_mlp_pack<<<64, 256, 0, h->stream>>>(S->w, S->wb);
    C3D_LAUNCH_CHECK(h);
    ++S->epochs;
  }
  // loss after the last update
  if ((rc = mlp_train_pass(h, S->feats, S->mom, M, sd, &loss, &norm))) return rc;
  S->last_loss = loss / std::max(norm, 1e-300);
  S->trained = true;
  if (h->ib) h->ib->have_lrn = false;
  if (final_loss) *final_loss = S->last_loss;
  return 0;
}

extern "C" int c3d_precond_info(int id, int64_t* pairs, int* sets, int* epochs, double* last_loss) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  MlpState* S = h->mlp;
  if (pairs) *pairs = S ? S->pairs : 0;
  if (sets) *sets = S ? S->nsets : 0;
  if (epochs) *epochs = S ? S->epochs : 0;
  if (last_loss) *last_loss = S ? S->last_loss : -1.0;
  return 0;
}

extern "C" int c3d_precond_get_params(int id, float* params, int n) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  cudaSetDevice(h->device);
  if (!params || n != kNParam + 8) return C3D_ERR_PARAM;
  int rc;
  if ((rc = mlp_ensure(h))) return rc;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(params, h->mlp->w, 4 * kNParam, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int i = 0; i < 4; ++i) { params[kNParam + i] = h->mlp->sig_r[i]; params[kNParam + 4 + i] = h->mlp->sig_e[i]; }
  return 0;
}

extern "C" int c3d_precond_set_params(int id, const float* params, int n, const float* sig) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  cudaSetDevice(h->device);
  if (!params || n != kNParam) return C3D_ERR_PARAM;
  int rc;
  if ((rc = mlp_ensure(h))) return rc;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(h->mlp->w, params, 4 * kNParam, cudaMemcpyHostToDevice, h->stream));
  k_mlp_pack<<<64, 256, 0, h->stream>>>(h->mlp->w, h->mlp->wb);
  C3D_LAUNCH_CHECK(h);
  if (sig)
    for (int i = 0; i < 4; ++i) { h->mlp->sig_r[i] = sig[i]; h->mlp->sig_e[i] = sig[4 + i]; }
  if ((rc = upload_sig(h))) return rc;
  h->mlp->trained = true;
  if (h->ib) h->ib->have_lrn = false;
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return 0;
}

// Forward, loss and gradient of the network on caller data (m rows of 32
// features and 36 moments): out[m][16], grad[kNParam], loss (unnormalised).
extern "C" int c3d_precond_eval(int id, const float* feats, const float* mom, int m, const float* sig,
                                float* out, float* grad, double* loss) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  cudaSetDevice(h->device);
  if (!feats || !mom || m < 1 || !sig) return C3D_ERR_PARAM;
  int rc;
  if ((rc = mlp_ensure(h))) return rc;
  if ((rc = ensure_rows(h, m))) return rc;
  MlpState* S = h->mlp;
  std::vector<__nv_bfloat16> fb((size_t)m * kF);
  for (size_t i = 0; i < fb.size(); ++i) fb[i] = __float2bfloat16_rn(feats[i]);
  if (S->eval_cap < m) {
    if ((rc = dev_alloc(h, &S->eval_f, (int64_t)m * kF))) return rc;
    if ((rc = dev_alloc(h, &S->eval_m, (int64_t)m * kMom))) return rc;
    S->eval_cap = m;
  }
  for (int i = 0; i < 4; ++i) { S->sig_r[i] = sig[i]; S->sig_e[i] = sig[4 + i]; }
  if ((rc = upload_sig(h))) return rc;
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S->eval_f, fb.data(), 2 * fb.size(), cudaMemcpyHostToDevice, h->stream));
  C3D_CUDA_TRY(h, cudaMemcpyAsync(S->eval_m, mom, 4 * (size_t)m * kMom, cudaMemcpyHostToDevice, h->stream));
  double l = 0, nrm = 0;
  if ((rc = mlp_train_pass(h, S->eval_f, S->eval_m, m, S->sig_d, &l, &nrm))) return rc;
  if (out) C3D_CUDA_TRY(h, cudaMemcpyAsync(out, h->mlp->out, 4 * (size_t)m * kO, cudaMemcpyDeviceToHost, h->stream));
  if (grad) C3D_CUDA_TRY(h, cudaMemcpyAsync(grad, h->mlp->g, 4 * kNParam, cudaMemcpyDeviceToHost, h->stream));
  C3D_CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (loss) *loss = l;
  return 0;
}
