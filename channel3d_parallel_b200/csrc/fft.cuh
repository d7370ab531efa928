// Batched shared-memory FFT for lengths N = 2^a 3^b (radix 4/2/3 passes).
//
// Stockham autosort formulation: pass p with radix R and current sub-length
// Ns maps butterfly j of every line to
//   in[j + r*N/R] * w^(r*(j mod Ns)),  w = exp(-+2 pi i / (Ns*R)),
//   out[(j div Ns)*Ns*R + (j mod Ns) + r*Ns] = DFT_R(...)[r]
// so the output is in natural order after the last pass.  Twiddles come from
// a table exp(-2 pi i m / N) built on the host in long double.
#pragma once
#include <cuda_runtime.h>

namespace c3d {

struct FftPasses {
  int n;
  int npass;
  int radix[8];
};

template <typename T> struct cplx;
template <> struct cplx<double> { using t = double2; };
template <> struct cplx<float> { using t = float2; };

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }

// Runs all passes on nl lines of length N stored contiguously in buf0.
// buf1 is scratch of the same size.  Returns the buffer holding the result.
// tw: N twiddles exp(-2 pi i m/N) (shared or global memory).
// Must be called by all threads of the block.
template <typename T, bool INV>
__device__ typename cplx<T>::t* fft_lines(typename cplx<T>::t* buf0, typename cplx<T>::t* buf1,
                                          int nl, const typename cplx<T>::t* tw, const FftPasses& P) {
  using C = typename cplx<T>::t;
  const int N = P.n;
  C* src = buf0;
  C* dst = buf1;
  int Ns = 1;
  const T s3 = (T)0.86602540378443864676;   // sqrt(3)/2
  for (int p = 0; p < P.npass; ++p) {
    const int R = P.radix[p];
    const int nb = N / R;
    const int tws = N / (Ns * R);
    for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
      const int line = t / nb;
      const int j = t - line * nb;
      const C* in = src + line * N;
      C* out = dst + line * N;
      const int kk = j % Ns;
      C v[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (r < R) {
          C a = in[j + r * nb];
          if (r > 0 && kk > 0) {
            C w = tw[kk * r * tws];
            if (INV) w.y = -w.y;
            a = cmul(a, w);
          }
          v[r] = a;
        }
      }
      if (R == 4) {
        C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        C a2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        C a3;
        if (INV) { a3.x = -d.y; a3.y = d.x; }     // +i*d
        else     { a3.x = d.y;  a3.y = -d.x; }    // -i*d
        v[0] = cadd(a0, a2);
        v[1] = cadd(a1, a3);
        v[2] = csub(a0, a2);
        v[3] = csub(a1, a3);
      } else if (R == 2) {
        C a0 = cadd(v[0], v[1]), a1 = csub(v[0], v[1]);
        v[0] = a0; v[1] = a1;
      } else {  // R == 3
        C s = cadd(v[1], v[2]);
        C d = csub(v[1], v[2]);
        C m;
        m.x = v[0].x - (T)0.5 * s.x;
        m.y = v[0].y - (T)0.5 * s.y;
        C id;   // (forward) -i*s3*d ; (inverse) +i*s3*d
        if (INV) { id.x = -s3 * d.y; id.y = s3 * d.x; }
        else     { id.x = s3 * d.y;  id.y = -s3 * d.x; }
        v[0] = cadd(v[0], s);
        v[1] = cadd(m, id);
        v[2] = csub(m, id);
      }
      const int base = (j / Ns) * Ns * R + kk;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (r < R) out[base + r * Ns] = v[r];
    }
    __syncthreads();
    C* tmp = src; src = dst; dst = tmp;
    Ns *= R;
  }
  return src;
}

// Radix-R butterfly on v[0..R-1] (R = 2, 3, 4), forward or inverse.
template <typename T, bool INV, int R>
__device__ __forceinline__ void butterfly(typename cplx<T>::t* v) {
  using C = typename cplx<T>::t;
  if (R == 4) {
    C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    C a2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    C a3;
    if (INV) { a3.x = -d.y; a3.y = d.x; }
    else     { a3.x = d.y;  a3.y = -d.x; }
    v[0] = cadd(a0, a2);
    v[1] = cadd(a1, a3);
    v[2] = csub(a0, a2);
    v[3] = csub(a1, a3);
  } else if (R == 2) {
    C a0 = cadd(v[0], v[1]), a1 = csub(v[0], v[1]);
    v[0] = a0; v[1] = a1;
  } else {
    const T s3 = (T)0.86602540378443864676;
    C s = cadd(v[1], v[2]);
    C d = csub(v[1], v[2]);
    C m;
    m.x = v[0].x - (T)0.5 * s.x;
    m.y = v[0].y - (T)0.5 * s.y;
    C id;
    if (INV) { id.x = -s3 * d.y; id.y = s3 * d.x; }
    else     { id.x = s3 * d.y;  id.y = -s3 * d.x; }
    v[0] = cadd(v[0], s);
    v[1] = cadd(m, id);
    v[2] = csub(m, id);
  }
}

// In-place mixed-radix FFT of shared-memory rows (Cooley-Tukey, no
// reordering pass).  With radices R_0..R_{P-1} and spans L_p = N/(R_0..R_{p-1}),
// stage p combines, in every block of L_p elements, the R_p elements
// q + r*M (M = L_p/R_p, q < M).
//   forward (decimation in frequency): DFT_R of the R inputs, output s scaled
//     by w_L^(q*s), w = exp(-2 pi i/L); stages p = 0..P-1; natural-order
//     input, X[k] left at the digit-reversed position dr(k);
//   inverse (decimation in time): input r scaled by conj(w_L^(q*r)), inverse
//     DFT_R; stages p = P-1..0; takes the digit-reversed spectrum back to
//     natural order, unnormalised.
// A butterfly reads and writes the same R addresses, so a stage needs one
// barrier and no staging.  Consecutive threads take consecutive q when runs
// of q are at least `run` long (conflict-free rows), else consecutive rows
// (conflict-free when the row stride is chosen for it).
template <typename T, bool INV, int R>
__device__ __forceinline__ void ct_stage(typename cplx<T>::t* data, int nrows, int rs,
                                         const typename cplx<T>::t* tw, int N, int L, int run) {
  using C = typename cplx<T>::t;
  const int M = L / R, nb = N / R, tws = N / L;
  const int total = nrows * nb;
  const bool rowmajor = M < run;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int l, bb;
    if (rowmajor) { bb = t / nrows; l = t - bb * nrows; }
    else { l = t / nb; bb = t - l * nb; }
    const int blk = bb / M, q = bb - blk * M;
    C* p = data + l * rs + blk * L + q;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = p[r * M];
    if (INV && q > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[q * r * tws];
        w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    butterfly<T, INV, R>(v);
    if (!INV && q > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[q * r * tws]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) p[r * M] = v[r];
  }
  __syncthreads();
}

// Same stage when blockDim.x is a multiple of N/R: every thread keeps one
// butterfly position (q fixed, twiddles in registers) and walks the rows
// l0, l0 + nt/(N/R), ..., kB rows per iteration.
template <typename T, bool INV, int R, int kB>
__device__ __forceinline__ void ct_stage_fixed(typename cplx<T>::t* data, int nrows, int rs,
                                               const typename cplx<T>::t* tw, int N, int L) {
  using C = typename cplx<T>::t;
  const int M = L / R, nb = N / R, tws = N / L;
  const int bb = threadIdx.x % nb;
  const int l0 = threadIdx.x / nb, ls = blockDim.x / nb;
  const int blk = bb / M, q = bb - blk * M;
  C w[R];
#pragma unroll
  for (int r = 1; r < R; ++r) {
    w[r] = tw[q * r * tws];
    if (INV) w[r].y = -w[r].y;
  }
  C* p0 = data + blk * L + q;
  // all loads of an iteration are issued before any store (the compiler
  // cannot reorder shared-memory loads across stores to a runtime stride)
  int l = l0;
  for (; l + (kB - 1) * ls < nrows; l += kB * ls) {
    C v[kB][R];
#pragma unroll
    for (int b = 0; b < kB; ++b)
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = p0[(l + b * ls) * rs + r * M];
#pragma unroll
    for (int b = 0; b < kB; ++b) {
      if (INV) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], w[r]);
      }
      butterfly<T, INV, R>(v[b]);
      if (!INV) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], w[r]);
      }
    }
#pragma unroll
    for (int b = 0; b < kB; ++b)
#pragma unroll
      for (int r = 0; r < R; ++r) p0[(l + b * ls) * rs + r * M] = v[b][r];
  }
  for (; l < nrows; l += ls) {
    C* p = p0 + l * rs;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = p[r * M];
    if (INV) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
    }
    butterfly<T, INV, R>(v);
    if (!INV) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) p[r * M] = v[r];
  }
  __syncthreads();
}

template <typename T, bool INV, int kB>
__device__ __forceinline__ void ct_stage_any(typename cplx<T>::t* data, int nrows, int rs,
                                             const typename cplx<T>::t* tw, int N, int L, int R,
                                             int run) {
  if (blockDim.x % (N / R) == 0) {
    if (R == 4) ct_stage_fixed<T, INV, 4, kB>(data, nrows, rs, tw, N, L);
    else if (R == 2) ct_stage_fixed<T, INV, 2, kB>(data, nrows, rs, tw, N, L);
    else ct_stage_fixed<T, INV, 3, kB>(data, nrows, rs, tw, N, L);
  } else {
    if (R == 4) ct_stage<T, INV, 4>(data, nrows, rs, tw, N, L, run);
    else if (R == 2) ct_stage<T, INV, 2>(data, nrows, rs, tw, N, L, run);
    else ct_stage<T, INV, 3>(data, nrows, rs, tw, N, L, run);
  }
}

// forward transform of nrows rows; output in digit-reversed order
template <typename T, int kB>
__device__ void fft_rows_dif(typename cplx<T>::t* data, int nrows, int rs,
                             const typename cplx<T>::t* tw, const FftPasses& P, int run) {
  int L = P.n;
  for (int p = 0; p < P.npass; ++p) {
    ct_stage_any<T, false, kB>(data, nrows, rs, tw, P.n, L, P.radix[p], run);
    L /= P.radix[p];
  }
}

// inverse transform of nrows digit-reversed rows; output in natural order
template <typename T, int kB>
__device__ void fft_rows_dit_inv(typename cplx<T>::t* data, int nrows, int rs,
                                 const typename cplx<T>::t* tw, const FftPasses& P, int run) {
  int L = 1;
  for (int p = P.npass - 1; p >= 0; --p) {
    L *= P.radix[p];
    ct_stage_any<T, true, kB>(data, nrows, rs, tw, P.n, L, P.radix[p], run);
  }
}

// position at which the forward transform leaves the coefficient of index k
__host__ __device__ inline int dif_k_to_position(int k, const FftPasses& P) {
  int pos = 0, rem = k, span = P.n;
  for (int p = 0; p < P.npass; ++p) {
    const int M = span / P.radix[p];
    const int s = rem % P.radix[p];
    rem /= P.radix[p];
    pos += s * M;
    span = M;
  }
  return pos;
}

// wavenumber index k whose coefficient the forward transform leaves at
// position pos (inverse of the digit reversal)
__host__ __device__ inline int dif_position_to_k(int pos, const FftPasses& P) {
  int k = 0, mult = 1, rem = pos, span = P.n;
  for (int p = 0; p < P.npass; ++p) {
    const int M = span / P.radix[p];
    const int s = rem / M;
    rem -= s * M;
    k += s * mult;
    mult *= P.radix[p];
    span = M;
  }
  return k;
}

}  // namespace c3d
