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

}  // namespace c3d
