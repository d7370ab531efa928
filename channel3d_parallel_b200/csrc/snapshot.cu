// Binary snapshots: output_data (src/input_output.f90:498-728) and
// read_input_data (src/input_output.f90:335-489), one domain.
//
// Layout (big-endian stream, no record markers; tools/file_io.py reads it):
//   int32 nx, x(nx); int32 ny, y(ny); int32 nz, z(nz)
//   int32 nxm, xm; int32 nym, ym; int32 nzm, zm
//   for U, V, W, P: int32 n1, n2, n3 and the array in Fortran order
//   (the "original" format stops here)
//   for Hu_interior, Hv_interior, Hw_interior: the same
//   real8 t, dt, dPdx, nu
//   int32 nb, xb(nb); int32 nb, yb; int32 nb, zb; int32 nxb; int32 nzb
//   int32 4nb, fb; int32 3nb, ub; int32 nb, sb;
//   int32 3nb, normals; int32 3nb, tangents_1; int32 3nb, tangents_2
// Without a body the Heaviside fields are 1 (app/main.f90:80-85) and the
// marker arrays are empty.  The reader takes the mesh and U, V, W, checks
// every size against the handle, as the reference does before reading, and
// replaces the grid and the three fields.
#include <cstdio>
#include <cstring>
#include <vector>

#include "c3d_internal.cuh"
#include "ib_state.cuh"

namespace c3d {

Handle* lookup_handle(int id);

namespace {

struct BeOut {
  FILE* f = nullptr;
  bool ok = true;
  void bytes(const void* p, size_t n) {
    if (ok && std::fwrite(p, 1, n, f) != n) ok = false;
  }
  void i32(int32_t v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u = __builtin_bswap32(u);
    bytes(&u, 4);
  }
  void f64(const double* a, size_t n) {
    std::vector<uint64_t> buf(n < 65536 ? n : 65536);
    for (size_t o = 0; o < n; o += buf.size()) {
      const size_t m = (n - o < buf.size()) ? n - o : buf.size();
      for (size_t q = 0; q < m; ++q) {
        uint64_t u;
        std::memcpy(&u, a + o + q, 8);
        buf[q] = __builtin_bswap64(u);
      }
      bytes(buf.data(), 8 * m);
    }
  }
  void vec(const double* a, int32_t n) {   // Write(1) Shape(a), a
    i32(n);
    f64(a, (size_t)n);
  }
};

struct BeIn {
  FILE* f = nullptr;
  bool ok = true;
  void bytes(void* p, size_t n) {
    if (ok && std::fread(p, 1, n, f) != n) ok = false;
  }
  int32_t i32() {
    uint32_t u = 0;
    bytes(&u, 4);
    u = __builtin_bswap32(u);
    int32_t v;
    std::memcpy(&v, &u, 4);
    return v;
  }
  void f64(double* a, size_t n) {
    bytes(a, 8 * n);
    if (!ok) return;
    for (size_t q = 0; q < n; ++q) {
      uint64_t u;
      std::memcpy(&u, a + q, 8);
      u = __builtin_bswap64(u);
      std::memcpy(a + q, &u, 8);
    }
  }
};

int field_extents(const Dims& d, int field, int e[3]) {
  switch (field) {
    case C3D_FIELD_U: case C3D_FIELD_HU_INTERIOR: e[0] = d.nx; e[1] = d.nyg; e[2] = d.nzg; return 0;
    case C3D_FIELD_V: case C3D_FIELD_HV_INTERIOR: e[0] = d.nxg; e[1] = d.ny; e[2] = d.nzg; return 0;
    case C3D_FIELD_W: case C3D_FIELD_HW_INTERIOR: e[0] = d.nxg; e[1] = d.nyg; e[2] = d.nz; return 0;
    case C3D_FIELD_P: e[0] = d.nxg; e[1] = d.nyg; e[2] = d.nzg; return 0;
    default: return -1;
  }
}

}  // namespace
}  // namespace c3d

using namespace c3d;

extern "C" {

int c3d_write_snapshot(int id, const char* path, int original_format) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  if (!path) return C3D_ERR_PARAM;
  cudaSetDevice(h->device);
  const Dims& d = h->d;
  int rc;
  // every device read first, so a failure leaves no partial file
  const int fields[7] = {C3D_FIELD_U, C3D_FIELD_V, C3D_FIELD_W, C3D_FIELD_P,
                         C3D_FIELD_HU_INTERIOR, C3D_FIELD_HV_INTERIOR, C3D_FIELD_HW_INTERIOR};
  const int nf = original_format ? 4 : 7;
  std::vector<std::vector<double>> data(nf);
  for (int q = 0; q < nf; ++q) {
    int e[3];
    field_extents(d, fields[q], e);
    data[q].assign((size_t)e[0] * e[1] * e[2], 1.0);
    if (q >= 4 && !h->ib) continue;               // H = 1 without a body (app/main.f90:80-85)
    const int64_t lb[3] = {1, 1, 1}, ub[3] = {e[0], e[1], e[2]};
    if ((rc = c3d_download(id, fields[q], data[q].data(), lb, ub))) return rc;
  }
  const int nb = h->ib ? ib_nb(h) : 0;
  const int mk[6] = {C3D_MARKER_XB, C3D_MARKER_YB, C3D_MARKER_ZB, C3D_MARKER_FB, C3D_MARKER_UB, C3D_MARKER_SB};
  const int ml[6] = {nb, nb, nb, 4 * nb, 3 * nb, nb};
  std::vector<std::vector<double>> mdat(7);
  if (!original_format && nb > 0) {
    for (int q = 0; q < 6; ++q) {
      mdat[q].assign((size_t)ml[q], 0.0);
      const int64_t lb[3] = {1, 1, 1}, ub[3] = {ml[q], 1, 1};
      if ((rc = c3d_download(id, mk[q], mdat[q].data(), lb, ub))) return rc;
    }
    mdat[6].assign((size_t)3 * nb, 0.0);
    const int64_t lb[3] = {1, 1, 1}, ub[3] = {3 * nb, 1, 1};
    if ((rc = c3d_download(id, C3D_MARKER_NORMALS, mdat[6].data(), lb, ub))) return rc;
  }
  BeOut o;
  o.f = std::fopen(path, "wb");
  if (!o.f) {
    h->last_error = std::string("cannot open ") + path + " for writing";
    return C3D_ERR_IO;
  }
  o.vec(h->x.data() + 1, d.nx);
  o.vec(h->y.data() + 1, d.ny);
  o.vec(h->z.data() + 1, d.nz);
  o.vec(h->xm.data() + 1, d.nx - 1);
  o.vec(h->ym.data() + 1, d.ny - 1);
  o.vec(h->zm.data() + 1, d.nz - 1);
  for (int q = 0; q < nf; ++q) {
    int e[3];
    field_extents(d, fields[q], e);
    o.i32(e[0]); o.i32(e[1]); o.i32(e[2]);
    o.f64(data[q].data(), data[q].size());
  }
  if (!original_format) {
    const double sc[4] = {h->t, h->dt, h->dPdx, h->p.nu};
    o.f64(sc, 4);
    auto arr = [&](int q, int n) { o.vec(n > 0 ? mdat[q].data() : nullptr, n); };
    arr(0, nb); arr(1, nb); arr(2, nb);
    // double_cylinders_z recomputes nxb as the markers around both cylinders
    // (src/immersed_boundary_geometry.f90:131)
    const bool dc = h->ib && h->ib->kind == "double_cylinders_z";
    o.i32(dc ? h->ib->lat_nx : h->p.nxb);
    o.i32(h->p.nzb);
    arr(3, 4 * nb); arr(4, 3 * nb); arr(5, nb); arr(6, 3 * nb);
    o.vec(nb > 0 ? h->ib->tan1.data() : nullptr, 3 * nb);
    o.vec(nb > 0 ? h->ib->tan2.data() : nullptr, 3 * nb);
  }
  const bool ok = o.ok;
  if (std::fclose(o.f) != 0 || !ok) {
    h->last_error = std::string("write error on ") + path;
    return C3D_ERR_IO;
  }
  return 0;
}

int c3d_read_snapshot(int id, const char* path) {
  Handle* h = lookup_handle(id);
  if (!h) return C3D_ERR_HANDLE;
  if (!path) return C3D_ERR_PARAM;
  cudaSetDevice(h->device);
  const Dims& d = h->d;
  BeIn in;
  in.f = std::fopen(path, "rb");
  if (!in.f) {
    h->last_error = std::string("cannot open ") + path;
    return C3D_ERR_IO;
  }
  auto fail = [&](const std::string& msg, int code) {
    std::fclose(in.f);
    h->last_error = msg;
    return code;
  };
  // mesh (src/input_output.f90:347-370): sizes checked against the namelist
  std::vector<double> xyz[6];
  const int want[6] = {d.nx, d.ny, d.nz, d.nx - 1, d.ny - 1, d.nz - 1};
  const char* name[6] = {"nx", "ny", "nz", "nxm", "nym", "nzm"};
  for (int q = 0; q < 6; ++q) {
    const int n = in.i32();
    if (!in.ok) return fail(std::string("truncated snapshot ") + path, C3D_ERR_IO);
    if (n != want[q]) return fail(std::string("Error: ") + name[q] + "_f/=" + name[q], C3D_ERR_PARAM);
    xyz[q].resize((size_t)n);
    in.f64(xyz[q].data(), (size_t)n);
  }
  // U, V, W (:372-470), each preceded by its three extents
  const int fields[3] = {C3D_FIELD_U, C3D_FIELD_V, C3D_FIELD_W};
  const char* fname[3] = {"U", "V", "W"};
  std::vector<double> F[3];
  for (int q = 0; q < 3; ++q) {
    int e[3];
    field_extents(d, fields[q], e);
    const int n1 = in.i32(), n2 = in.i32(), n3 = in.i32();
    if (!in.ok) return fail(std::string("truncated snapshot ") + path, C3D_ERR_IO);
    if (n1 != e[0] || n2 != e[1] || n3 != e[2])
      return fail(std::string("Error! wrong size in input file (") + fname[q] + ")", C3D_ERR_PARAM);
    F[q].resize((size_t)n1 * n2 * n3);
    in.f64(F[q].data(), F[q].size());
    if (!in.ok) return fail(std::string("truncated snapshot ") + path, C3D_ERR_IO);
  }
  std::fclose(in.f);
  int rc = c3d_set_grid(id, xyz[0].data(), xyz[1].data(), xyz[2].data());
  if (rc) return rc;
  for (int q = 0; q < 3; ++q) {
    int e[3];
    field_extents(d, fields[q], e);
    const int64_t lb[3] = {1, 1, 1}, ub[3] = {e[0], e[1], e[2]};
    if ((rc = c3d_upload(id, fields[q], F[q].data(), lb, ub))) return rc;
  }
  return 0;
}

}  // extern "C"
