// CPU check of the shared-memory FFT engine (channel3d_parallel_b200/csrc/fft.cuh):
// every stage plan of the radices 16, 12, 8, 6, 4, 3, 2 against a long-double
// DFT, the digit-reversal maps, and the forward/inverse round trip.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include "../../channel3d_parallel_b200/csrc/fft.cuh"

using namespace c3d;

template <int MAXR>
static double check(int n, int nrows) {
  FftPasses P;
  if (!make_fft_passes(n, P, MAXR)) return 1.0;
  const int rs = n + 3;
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<double2> tw(n), data((size_t)nrows * rs);
  for (int m = 0; m < n; ++m) {
    const long double a = -2.0L * pi * m / n;
    tw[m] = {(double)cosl(a), (double)sinl(a)};
  }
  std::mt19937_64 g(1000 + n);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<std::complex<double>> x((size_t)nrows * n);
  for (int l = 0; l < nrows; ++l)
    for (int i = 0; i < n; ++i) {
      x[(size_t)l * n + i] = {u(g), u(g)};
      data[(size_t)l * rs + i] = {x[(size_t)l * n + i].real(), x[(size_t)l * n + i].imag()};
    }
  fft_rows_dif<double, MAXR>(data.data(), nrows, rs, tw.data(), P);
  double err = 0.0, mx = 0.0;
  for (int l = 0; l < nrows; ++l)
    for (int k = 0; k < n; ++k) {
      std::complex<long double> s = 0.0L;
      for (int i = 0; i < n; ++i)
        s += std::complex<long double>(x[(size_t)l * n + i]) *
             std::polar(1.0L, -2.0L * pi * (long double)((long long)i * k % n) / n);
      const int pos = dif_k_to_position(k, P);
      if (dif_position_to_k(pos, P) != k) return 1.0;
      const double2 got = data[(size_t)l * rs + pos];
      err = std::max(err, (double)std::abs(std::complex<long double>(got.x, got.y) - s));
      mx = std::max(mx, (double)std::abs(s));
    }
  fft_rows_dit_inv<double, MAXR>(data.data(), nrows, rs, tw.data(), P);
  double err2 = 0.0;
  for (int l = 0; l < nrows; ++l)
    for (int i = 0; i < n; ++i) {
      const double2 v = data[(size_t)l * rs + i];
      err2 = std::max(err2, std::abs(std::complex<double>(v.x / n, v.y / n) - x[(size_t)l * n + i]));
    }
  printf("n=%4d maxr=%2d plan=", n, MAXR);
  for (int p = 0; p < P.npass; ++p) printf("%d ", P.radix[p]);
  printf(" forward %.2e round trip %.2e\n", err / mx, err2);
  return std::max(err / mx, err2);
}

int main() {
  double worst = 0.0;
  for (int n : {2, 3, 4, 6, 8, 12, 16, 18, 24, 32, 48, 54, 64, 96, 128, 192, 256, 384, 486}) {
    worst = std::max(worst, check<16>(n, 3));
    worst = std::max(worst, check<8>(n, 2));
    worst = std::max(worst, check<4>(n, 2));
  }
  printf("worst %.3e\n", worst);
  return worst < 1e-14 ? 0 : 1;
}
