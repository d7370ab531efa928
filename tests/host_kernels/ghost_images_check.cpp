// CPU check of the ghost-entry writers of the projection update
// (channel3d_parallel_b200/csrc/ghost_images.cuh): every interior point of a
// u-, v- or w-shaped field writes its value at itself and at every ghost
// entry whose boundary-condition source it is; the result must equal, entry
// for entry, apply_boundary_conditions (src/boundary_conditions.f90:20-252)
// as restated here: ghost = sign * F(fold(i), mapy(j), fold(k)), periodic
// folds 1 <- N+1, N+2 <- 2, N+3 <- 3 in x and z, odd y reflections for
// cell-centred y and zero wall values for the y faces of v.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../channel3d_parallel_b200/csrc/ghost_images.cuh"

using namespace c3d;

static int fold(int i, int N) { return i == 1 ? N + 1 : (i >= N + 2 ? i - N : i); }
static double value(int i, int j, int k) { return 1.0 + i + 1000.0 * j + 1.0e6 * k; }

// n1 x n2 x n3 field with Nx, Nz unique points in x and z; yface: v
static int check(int Nx, int Ny, int Nz, int n1, int n2, int n3, bool yface, const char* name) {
  std::vector<double> F((size_t)n1 * n2 * n3, NAN);
  for (int k = 2; k <= Nz + 1; ++k)
    for (int j = 2; j <= n2 - 1; ++j)
      for (int i = 2; i <= Nx + 1; ++i) {
        put_images_all(F.data(), n1, n2, n3, Nx, Nz, yface, i, j, k, value(i, j, k));
        // the zero wall values of v, written by the rows next to the walls
        if (yface && j == 2) put_images_all(F.data(), n1, n2, n3, Nx, Nz, true, i, 1, k, 0.0);
        if (yface && j == n2 - 1) put_images_all(F.data(), n1, n2, n3, Nx, Nz, true, i, n2, k, 0.0);
      }
  int bad = 0;
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) {
        double want;
        if (yface && (j == 1 || j == n2)) {
          want = 0.0;
        } else {
          int sj = j;
          double sg = 1.0;
          if (!yface && j == 1) { sj = 2; sg = -1.0; }
          if (!yface && j == n2) { sj = n2 - 1; sg = -1.0; }
          want = sg * value(fold(i, Nx), sj, fold(k, Nz));
        }
        const double got = F[(size_t)(i - 1) + (size_t)n1 * ((j - 1) + (size_t)n2 * (k - 1))];
        if (!(got == want)) {
          if (bad < 5) printf("%s (%d,%d,%d): got %g want %g\n", name, i, j, k, got, want);
          ++bad;
        }
      }
  printf("%s %dx%dx%d (field %dx%dx%d): %d mismatches\n", name, Nx, Ny, Nz, n1, n2, n3, bad);
  return bad;
}

int main() {
  int bad = 0;
  const int sizes[][3] = {{16, 16, 12}, {32, 64, 54}, {192, 17, 192}, {2, 3, 2}, {4, 2, 3}};
  for (const auto& s : sizes) {
    const int Nx = s[0], Ny = s[1], Nz = s[2];
    // extents of the single-domain arrays: nx = Nx+2, nxg = Nx+3, ny = Ny+1,
    // nyg = Ny+2, nz = Nz+2, nzg = Nz+3
    bad += check(Nx, Ny, Nz, Nx + 2, Ny + 2, Nz + 3, false, "u");
    bad += check(Nx, Ny, Nz, Nx + 3, Ny + 1, Nz + 3, true, "v");
    bad += check(Nx, Ny, Nz, Nx + 3, Ny + 2, Nz + 2, false, "w");
  }
  return bad == 0 ? 0 : 1;
}
