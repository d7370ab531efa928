// Immersed-boundary operators (placeholder until the IB kernels land).
#include "c3d_internal.cuh"

namespace c3d {

struct IbState {};

int ib_create(Handle* h) {
  h->last_error = "immersed boundary not available in this build";
  return C3D_ERR_UNSUPPORTED;
}
void ib_free(Handle* h) { (void)h; }
int ib_setup_geometry(Handle* h, double) { (void)h; return C3D_ERR_UNSUPPORTED; }
int ib_setup_operators(Handle* h) { (void)h; return C3D_ERR_UNSUPPORTED; }
int ib_heaviside(Handle* h) { (void)h; return C3D_ERR_UNSUPPORTED; }
int ib_projection(Handle* h, double, int) { (void)h; return C3D_ERR_UNSUPPORTED; }
int ib_regT(Handle*, const double*, const double*, const double*, double*) { return C3D_ERR_UNSUPPORTED; }
int ib_regTc_1n(Handle*, const double*, double*) { return C3D_ERR_UNSUPPORTED; }
int ib_regT_1n(Handle*, const double*, const double*, const double*, double*) { return C3D_ERR_UNSUPPORTED; }
int ib_reg(Handle*, int, const double*, double*) { return C3D_ERR_UNSUPPORTED; }
int ib_schur(Handle*, const double*, double*, double) { return C3D_ERR_UNSUPPORTED; }
int ib_bicgstab(Handle*, const double*, double) { return C3D_ERR_UNSUPPORTED; }
double* ib_marker_ptr(Handle*, int, int64_t*) { return nullptr; }
double* ib_field_ptr(Handle*, int) { return nullptr; }
double* ib_scratch(Handle*, int) { return nullptr; }
int ib_nb(Handle*) { return 0; }
const double* ib_hu(Handle*) { return nullptr; }
const double* ib_hv(Handle*) { return nullptr; }
const double* ib_hw(Handle*) { return nullptr; }
bool ib_moving(Handle*) { return false; }

}  // namespace c3d
