// Batched in-place shared-memory FFT for lengths N = 2^a 3^b.
//
// A transform of rows held in shared memory runs as a few Cooley-Tukey
// stages of large radix (16, 12, 8, 6, 4, 3, 2; N = 192 is 16 x 12): each
// stage reads the R points of a butterfly once, computes their R-point DFT
// in registers (itself split into 2-, 3- and 4-point DFTs with constant
// roots of unity) and writes them back to the same addresses, so a stage
// costs one read and one write of the row and one barrier.  Twiddles come
// from a table exp(-2 pi i m / N) built on the host in long double.
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

// cos and sin of 2 pi a / 48 (every root of unity of order 16 and 12 is one
// of these); a is a compile-time constant wherever this is called, so the
// switch folds to a literal
__host__ __device__ constexpr double cos48_base(int r) {
  switch (r) {
    case 0: return 1.0;
    case 1: return 0.991444861373810411157;
    case 2: return 0.965925826289068286750;
    case 3: return 0.923879532511286756128;   // cos(pi/8)
    case 4: return 0.866025403784438646764;   // sqrt(3)/2
    case 5: return 0.793353340291235164595;
    case 6: return 0.707106781186547524401;   // sqrt(2)/2
    case 7: return 0.608761429008720639416;
    case 8: return 0.5;
    case 9: return 0.382683432365089771728;   // sin(pi/8)
    case 10: return 0.258819045102520762349;
    case 11: return 0.130526192220051591549;
    default: return 0.0;                      // r = 12
  }
}
__host__ __device__ constexpr double cos48(int a) {
  a = ((a % 48) + 48) % 48;
  const int q = a / 12, r = a % 12;
  return q == 0 ? cos48_base(r) : q == 1 ? -cos48_base(12 - r) : q == 2 ? -cos48_base(r) : cos48_base(12 - r);
}
__host__ __device__ constexpr double sin48(int a) { return cos48(a - 12); }

// a * exp(-+2 pi i m / R) (forward: minus), m and R compile-time constants
// after unrolling; quarter turns are exact
template <typename T, bool INV>
__device__ __forceinline__ typename cplx<T>::t mul_root(typename cplx<T>::t a, int m, int R) {
  using C = typename cplx<T>::t;
  const int e = ((m % R) * (48 / R)) % 48;      // angle index over 48
  if (e == 0) return a;
  if (e == 24) return C{-a.x, -a.y};
  // forward exp(-i theta) = c - i s; inverse c + i s
  if (e == 12) return INV ? C{-a.y, a.x} : C{a.y, -a.x};
  if (e == 36) return INV ? C{a.y, -a.x} : C{-a.y, a.x};
  const T c = (T)cos48(e), s = INV ? (T)sin48(e) : (T)-sin48(e);
  return C{a.x * c - a.y * s, a.x * s + a.y * c};
}

// R-point DFT of v[0..R-1] in registers, output in natural order:
// v[s] = sum_r v[r] exp(-+2 pi i r s / R).
template <typename T, bool INV, int R>
struct Dft;

template <typename T, bool INV>
struct Dft<T, INV, 2> {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    const C a0 = cadd(v[0], v[1]), a1 = csub(v[0], v[1]);
    v[0] = a0; v[1] = a1;
  }
};

template <typename T, bool INV>
struct Dft<T, INV, 3> {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    const T s3 = (T)0.866025403784438646764;   // sqrt(3)/2
    const C s = cadd(v[1], v[2]);
    const C d = csub(v[1], v[2]);
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
};

template <typename T, bool INV>
struct Dft<T, INV, 4> {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    const C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const C a2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    C a3;
    if (INV) { a3.x = -d.y; a3.y = d.x; }     // +i*d
    else     { a3.x = d.y;  a3.y = -d.x; }    // -i*d
    v[0] = cadd(a0, a2);
    v[1] = cadd(a1, a3);
    v[2] = csub(a0, a2);
    v[3] = csub(a1, a3);
  }
};

// R = R1 * R2: with r = r1 + R1 r2 and s = s2 + R2 s1,
//   X[s2 + R2 s1] = sum_r1 w_R1^(r1 s1) [w_R^(r1 s2) sum_r2 v[r1 + R1 r2] w_R2^(r2 s2)]:
// R1 DFTs of length R2, the constant twiddles w_R^(r1 s2), R2 DFTs of length R1.
template <typename T, bool INV, int R1, int R2>
struct DftSplit {
  template <typename C>
  __device__ __forceinline__ static void run(C* v) {
    constexpr int R = R1 * R2;
    C y[R];
#pragma unroll
    for (int r1 = 0; r1 < R1; ++r1) {
      C t[R2];
#pragma unroll
      for (int r2 = 0; r2 < R2; ++r2) t[r2] = v[r1 + R1 * r2];
      Dft<T, INV, R2>::run(t);
#pragma unroll
      for (int s2 = 0; s2 < R2; ++s2) y[r1 * R2 + s2] = mul_root<T, INV>(t[s2], r1 * s2, R);
    }
#pragma unroll
    for (int s2 = 0; s2 < R2; ++s2) {
      C t[R1];
#pragma unroll
      for (int r1 = 0; r1 < R1; ++r1) t[r1] = y[r1 * R2 + s2];
      Dft<T, INV, R1>::run(t);
#pragma unroll
      for (int s1 = 0; s1 < R1; ++s1) v[s2 + R2 * s1] = t[s1];
    }
  }
};

template <typename T, bool INV> struct Dft<T, INV, 6> : DftSplit<T, INV, 2, 3> {};
template <typename T, bool INV> struct Dft<T, INV, 8> : DftSplit<T, INV, 2, 4> {};
template <typename T, bool INV> struct Dft<T, INV, 12> : DftSplit<T, INV, 4, 3> {};
template <typename T, bool INV> struct Dft<T, INV, 16> : DftSplit<T, INV, 4, 4> {};

// One in-place Cooley-Tukey stage of radix R on nrows rows (stride rs) of
// length N.  With spans L_p = N/(R_0..R_{p-1}), stage p combines, in every
// block of L_p elements, the R_p elements q + r*M (M = L_p/R_p, q < M).
//   forward (decimation in frequency): DFT_R of the R inputs, output s scaled
//     by w_L^(q*s), w = exp(-2 pi i/L); stages p = 0..P-1; natural-order
//     input, X[k] left at the digit-reversed position dr(k);
//   inverse (decimation in time): input r scaled by conj(w_L^(q*r)), inverse
//     DFT_R; stages p = P-1..0; takes the digit-reversed spectrum back to
//     natural order, unnormalised.
// Consecutive threads take consecutive rows of the same butterfly, so with
// an odd row stride (in complex values) eight threads of a quarter warp touch
// eight different 16-byte bank groups, and the twiddle reads of a warp are
// broadcasts.
template <typename T, bool INV, int R>
__device__ __forceinline__ void ct_stage(typename cplx<T>::t* data, int nrows, int rs,
                                         const typename cplx<T>::t* tw, int N, int L) {
  using C = typename cplx<T>::t;
  const int M = L / R, nb = N / R, tws = N / L;
  const int total = nrows * nb;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int bb = t / nrows, l = t - bb * nrows;
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
    Dft<T, INV, R>::run(v);
    if (!INV && q > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[q * r * tws]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) p[r * M] = v[r];
  }
  __syncthreads();
}

// radices above MAXR are not compiled in (a kernel's register budget)
template <typename T, bool INV, int MAXR>
__device__ __forceinline__ void ct_stage_any(typename cplx<T>::t* data, int nrows, int rs,
                                             const typename cplx<T>::t* tw, int N, int L, int R) {
  if (MAXR >= 16 && R == 16) ct_stage<T, INV, (MAXR >= 16 ? 16 : 2)>(data, nrows, rs, tw, N, L);
  else if (MAXR >= 12 && R == 12) ct_stage<T, INV, (MAXR >= 12 ? 12 : 2)>(data, nrows, rs, tw, N, L);
  else if (MAXR >= 8 && R == 8) ct_stage<T, INV, (MAXR >= 8 ? 8 : 2)>(data, nrows, rs, tw, N, L);
  else if (MAXR >= 6 && R == 6) ct_stage<T, INV, (MAXR >= 6 ? 6 : 2)>(data, nrows, rs, tw, N, L);
  else if (R == 4) ct_stage<T, INV, 4>(data, nrows, rs, tw, N, L);
  else if (R == 3) ct_stage<T, INV, 3>(data, nrows, rs, tw, N, L);
  else ct_stage<T, INV, 2>(data, nrows, rs, tw, N, L);
}

// forward transform of nrows rows; output in digit-reversed order.  The plan
// P must come from make_fft_passes with the same MAXR.
template <typename T, int MAXR>
__device__ void fft_rows_dif(typename cplx<T>::t* data, int nrows, int rs,
                             const typename cplx<T>::t* tw, const FftPasses& P) {
  int L = P.n;
  for (int p = 0; p < P.npass; ++p) {
    ct_stage_any<T, false, MAXR>(data, nrows, rs, tw, P.n, L, P.radix[p]);
    L /= P.radix[p];
  }
}

// inverse transform of nrows digit-reversed rows; output in natural order
template <typename T, int MAXR>
__device__ void fft_rows_dit_inv(typename cplx<T>::t* data, int nrows, int rs,
                                 const typename cplx<T>::t* tw, const FftPasses& P) {
  int L = 1;
  for (int p = P.npass - 1; p >= 0; --p) {
    L *= P.radix[p];
    ct_stage_any<T, true, MAXR>(data, nrows, rs, tw, P.n, L, P.radix[p]);
  }
}

// Stage plan of an N-point transform: the largest radix of 16, 12, 8, 6, 4,
// 3, 2 (not above maxr) that divides what is left, first.  False when N is
// not 2^a 3^b.
__host__ inline bool make_fft_passes(int n, FftPasses& P, int maxr) {
  static const int kRadices[] = {16, 12, 8, 6, 4, 3, 2};
  P.n = n;
  P.npass = 0;
  int m = n;
  while (m > 1 && P.npass < 8) {
    int r = 0;
    for (int c : kRadices)
      if (c <= maxr && m % c == 0) { r = c; break; }
    if (r == 0) break;
    P.radix[P.npass++] = r;
    m /= r;
  }
  return m == 1 && n >= 2;
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
