"""FP64 CPU restatement of channel3D's RK3 fractional-step path (test infrastructure).

Parity unpinned: the reference has no golden data and cannot be built here;
see ``oracle/__init__.py``.

Conventions
-----------
All 3-D arrays are *Fortran-indexed*: a reference array ``A(1:n1,1:n2,1:n3)``
is held as a NumPy array of shape ``(n1+1, n2+1, n3+1)`` whose index 0 in
every axis is unused padding, so ``A[i, j, k]`` here is ``A(i,j,k)`` there.
Arrays the reference declares with lower bound 2 (``rhs_p(2:nxg-1,2:nyg-1,2:nzg)``,
``Fu1(2:nx-1,...)``) are held with the same padding convention and shape
``(ub1+1, ub2+1, ub3+1)``.

The domain is the single-domain (one z slab) view of the reference's global
arrays: with ``nprocs = 1`` the reference's own extents are
``U(nx, nyg, nzg)`` with ``nz = nz_global`` and ``nzg = nz_global + 1``
(src/initialization.f90:60-94).  The z-periodic copies that the reference
performs between rank 0 and rank ``nprocs-1`` (src/boundary_conditions.f90:91-224,
src/poisson.f90:106-125) are restated as local copies within this one domain.
"""
import math

import numpy as np
from scipy.linalg import lapack

from .namelist import read_namelist, parse_namelist_text

PI = 4.0 * math.atan(1.0)  # src/global.f90:30

# RK3 tableau, src/initialization.f90:406-418
RK_T = (8.0 / 15.0, 2.0 / 3.0, 1.0)
RK_COEF = ((8.0 / 15.0, 0.0, 0.0),
           (1.0 / 4.0, 5.0 / 12.0, 0.0),
           (1.0 / 4.0, 0.0, 3.0 / 4.0))


def _f1(n):
    """Fortran-indexed 1-D array of length n (index 0 unused)."""
    return np.zeros(n + 1)


def create_grid(p):
    """Face grids x_global, y_global, z_global.  src/input_output.f90:140-206."""
    nxg_, nyg_, nzg_ = p["nx_global"], p["ny_global"], p["nz_global"]
    x = np.arange(nxg_, dtype=np.float64)
    x = p["lxp"] * x / x[nxg_ - 2]                       # :146-149
    z = np.arange(nzg_, dtype=np.float64)
    z = p["lzp"] * z / z[nzg_ - 2]                       # :151-154
    gt = p["grid_type"]
    if gt == 0:                                          # :157-162
        y = np.arange(nyg_, dtype=np.float64)
        y = p["ly_channel"] * y / y.max()
    elif gt == 1:                                        # :164-178
        y = np.arange(nyg_, dtype=np.float64)
        y = p["ly_channel"] * y / y.max() - 1.0
        if p["alpha_stretch"] > 0.0:
            y = np.tanh(p["alpha_stretch"] * y) / np.tanh(p["alpha_stretch"])
        y = y - y.min()
        y = y * p["ly_channel"] / y.max()
    elif gt == 2:                                        # :180-202
        y = _create_grid_type2(p)
    else:
        raise ValueError(f"grid_type {gt} not supported")
    return x, y, z


def _create_stretched_grid(L, n_total, n_uniform, alpha):
    """src/input_output.f90:208-247."""
    m = n_total - 2 * (n_uniform - 1)
    gu = np.arange(m, dtype=np.float64)
    gu = 2.0 * gu / gu.max() - 1.0
    if alpha > 0.0:
        gu = np.tanh(alpha * gu) / np.tanh(alpha)
    ds_un = gu[1] - gu[0]
    ds_sc = L * ds_un / (2.0 + (n_uniform - 1) * ds_un)
    g = np.zeros(n_total + 1)
    g[n_uniform:n_total - n_uniform + 2] = gu * ds_sc / ds_un
    for i in range(2, n_uniform + 1):
        g[n_total - n_uniform + i] = g[n_total - n_uniform + i - 1] + ds_sc
        g[n_uniform - i + 1] = g[n_uniform - i + 2] - ds_sc
    return g[1:]


def _create_grid_type2(p, suppy=2):
    """Grid type 2 loop, src/input_output.f90:180-202."""
    ny = p["ny_global"]
    n_uniform = 1
    while True:
        y = _create_stretched_grid(p["ly_channel"], ny, n_uniform, p["alpha_stretch"])
        dymin = y[1] - y[0]
        if n_uniform * dymin >= p["min_buffer_width"] + (2 * suppy + 2) * dymin:
            break
        n_uniform += 1
        if 2 * n_uniform >= ny - 1:
            raise ValueError("Number of buffer points exceeds the total number of grid points")
    return y + 1.0


class Grid:
    """Grid, metric and spectral set-up of ``initialize`` for nprocs = 1.

    src/initialization.f90:73-391.
    """

    def __init__(self, p, x=None, y=None, z=None):
        self.p = p
        nx = self.nx = p["nx_global"]
        ny = self.ny = p["ny_global"]
        nz = self.nz = p["nz_global"]
        if nx % 2 or nz % 2:
            raise ValueError("nx and nz must be even")       # :46-47
        if x is None:
            x, y, z = create_grid(p)
        self.nxm, self.nym, self.nzm = nx - 1, ny - 1, nz - 1  # :79-85 (nzm = nz_global-1)
        self.nxg, self.nyg, self.nzg = nx + 1, ny + 1, nz + 1  # :92-94
        nxm, nym, nzm = self.nxm, self.nym, self.nzm
        X = _f1(nx); X[1:] = x
        Y = _f1(ny); Y[1:] = y
        Z = _f1(nz); Z[1:] = z
        xm = _f1(nxm); xm[1:] = 0.5 * (X[1:nx] + X[2:nx + 1])   # :173-181
        ym = _f1(nym); ym[1:] = 0.5 * (Y[1:ny] + Y[2:ny + 1])
        zm = _f1(nzm); zm[1:] = 0.5 * (Z[1:nz] + Z[2:nz + 1])

        def ghost(cm, cf, nm, n):
            g = _f1(nm + 2)                                         # :189-199
            g[2:nm + 2] = cm[1:nm + 1]
            g[1] = cm[1] - 2.0 * (cm[1] - cf[1])
            g[nm + 2] = cm[nm] + 2.0 * (cf[n] - cm[nm])
            return g

        self.x, self.y, self.z = X, Y, Z
        self.xm, self.ym, self.zm = xm, ym, zm
        self.xg = ghost(xm, X, nxm, nx)
        self.yg = ghost(ym, Y, nym, ny)
        self.zg = ghost(zm, Z, nzm, nz)
        xg, yg, zg = self.xg, self.yg, self.zg
        nxg, nyg, nzg = self.nxg, self.nyg, self.nzg
        # :212-214
        self.dxmin = float(np.min(xg[2:nxg + 1] - xg[1:nxg]))
        self.dymin = float(np.min(yg[2:nyg + 1] - yg[1:nyg]))
        self.dzmin = float(np.min(zg[2:nzg + 1] - zg[1:nzg]))
        self.Lx = X[nx] - X[1]                                      # :217-219
        self.Ly = Y[ny] - Y[1]
        self.Lz = Z[nz] - Z[1]
        # Fourier set-up, :247-305
        self.dx = self.dxmin
        self.dz = self.dzmin
        self.Lxp = self.Lx - self.dx
        self.Lzp = self.Lz - self.dz
        self.nxp = nxm - 1
        self.nzp = nzm - 1
        nxp, nzp = self.nxp, self.nzp
        self.kxx = np.zeros(nxp)
        self.kzz = np.zeros(nzp)
        for i in range(0, math.ceil(nxp / 2.0) + 1):
            self.kxx[i] = 2.0 * (math.cos(2.0 * PI * float(i) / float(nxp)) - 1.0) / self.dx ** 2
        for i in range(math.ceil(nxp / 2.0) + 1, nxp):
            self.kxx[i] = 2.0 * (math.cos(2.0 * PI * float(-nxp + i) / float(nxp)) - 1.0) / self.dx ** 2
        for k in range(0, math.ceil(nzp / 2.0) + 1):
            self.kzz[k] = 2.0 * (math.cos(2.0 * PI * float(k) / float(nzp)) - 1.0) / self.dz ** 2
        for k in range(math.ceil(nzp / 2.0) + 1, nzp):
            self.kzz[k] = 2.0 * (math.cos(2.0 * PI * float(-nzp + k) / float(nzp)) - 1.0) / self.dz ** 2
        # Dyy tridiagonal with Neumann rows, :352-383; stored as 3 diagonals
        # over rows j = 2..nyg-1 (Fortran-indexed).
        self.Dd = _f1(nyg)   # Dyy(j,j)
        self.Dl = _f1(nyg)   # Dyy(j,j-1)
        self.Du = _f1(nyg)   # Dyy(j,j+1)
        Yf, ygf = Y, yg
        for j in range(3, nyg - 1):
            a = 1.0 / (Yf[j] - Yf[j - 1]) / (ygf[j + 1] - ygf[j])
            b = 1.0 / (Yf[j] - Yf[j - 1]) * (-1.0 / (ygf[j + 1] - ygf[j]) - 1.0 / (ygf[j] - ygf[j - 1]))
            c = 1.0 / (Yf[j] - Yf[j - 1]) / (ygf[j] - ygf[j - 1])
            self.Du[j], self.Dl[j], self.Dd[j] = a, c, b
        j = 2
        a = 1.0 / (Yf[j] - Yf[j - 1]) / (ygf[j + 1] - ygf[j])
        b = 1.0 / (Yf[j] - Yf[j - 1]) * (-1.0 / (ygf[j + 1] - ygf[j]) - 1.0 / (ygf[j] - ygf[j - 1]))
        c = 1.0 / (Yf[j] - Yf[j - 1]) / (ygf[j] - ygf[j - 1])
        self.Dd[2] = b + c
        self.Du[2] = a
        j = nyg - 1
        a = 1.0 / (Yf[j] - Yf[j - 1]) / (ygf[j + 1] - ygf[j])
        b = 1.0 / (Yf[j] - Yf[j - 1]) * (-1.0 / (ygf[j + 1] - ygf[j]) - 1.0 / (ygf[j] - ygf[j - 1]))
        c = 1.0 / (Yf[j] - Yf[j - 1]) / (ygf[j] - ygf[j - 1])
        self.Dd[nyg - 1] = a + b
        self.Dl[nyg - 1] = c

    # ---- array factories with the reference extents (src/initialization.f90:116-155)
    def u_array(self):
        return np.zeros((self.nx + 1, self.nyg + 1, self.nzg + 1))

    def v_array(self):
        return np.zeros((self.nxg + 1, self.ny + 1, self.nzg + 1))

    def w_array(self):
        return np.zeros((self.nxg + 1, self.nyg + 1, self.nz + 1))

    def p_array(self):
        return np.zeros((self.nxg + 1, self.nyg + 1, self.nzg + 1))

    def rhs_p_array(self):
        """rhs_p(2:nxg-1, 2:nyg-1, 2:nzg) -- one extra plane in z (:155)."""
        return np.zeros((self.nxg, self.nyg, self.nzg + 1))


# --------------------------------------------------------------------------
# boundary conditions, src/boundary_conditions.f90:20-252 (single domain)
# --------------------------------------------------------------------------
def apply_periodic_bc_x(g, F, face):
    """src/boundary_conditions.f90:67-86."""
    if face:
        F[1, :, :] = F[g.nx - 1, :, :]
        F[g.nx, :, :] = F[2, :, :]
    else:
        F[1, :, :] = F[g.nxg - 2, :, :]
        F[g.nxg - 1, :, :] = F[2, :, :]
        F[g.nxg, :, :] = F[3, :, :]


def apply_periodic_bc_z(g, F, face):
    """Single-domain form of src/boundary_conditions.f90:91-224.

    Faces (W, id=3): F(1)=F(nz-1), F(nz)=F(2).  Centres: F(1)=F(nzg-2),
    F(nzg-1)=F(2), F(nzg)=F(3).
    """
    if face:
        top = F[:, :, g.nz - 1].copy()
        bot = F[:, :, 2].copy()
        F[:, :, 1] = top
        F[:, :, g.nz] = bot
    else:
        top = F[:, :, g.nzg - 2].copy()
        b2 = F[:, :, 2].copy()
        b3 = F[:, :, 3].copy()
        F[:, :, 1] = top
        F[:, :, g.nzg - 1] = b2
        F[:, :, g.nzg] = b3


def apply_dirichlet_bc_y(g, F, face):
    """src/boundary_conditions.f90:237-252."""
    if face:
        F[:, 1, :] = 0.0
        F[:, g.ny, :] = 0.0
    else:
        F[:, 1, :] = -F[:, 2, :]
        F[:, g.nyg, :] = -F[:, g.nyg - 1, :]


def apply_boundary_conditions(g, U, V, W):
    """src/boundary_conditions.f90:20-55 (x, then z, then y)."""
    apply_periodic_bc_x(g, U, True)
    apply_periodic_bc_x(g, V, False)
    apply_periodic_bc_x(g, W, False)
    apply_periodic_bc_z(g, U, False)
    apply_periodic_bc_z(g, V, False)
    apply_periodic_bc_z(g, W, True)
    apply_dirichlet_bc_y(g, U, False)
    apply_dirichlet_bc_y(g, V, True)
    apply_dirichlet_bc_y(g, W, False)


# --------------------------------------------------------------------------
# right-hand sides, src/equations.f90
# --------------------------------------------------------------------------
def _col(a):
    return a[:, None, None]


def _row(a):
    return a[None, :, None]


def _dep(a):
    return a[None, None, :]


def compute_rhs_u(g, U, V, W, dPdx, Hu=None, exterior_pressure_gradient=True):
    """src/equations.f90:24-153.  Returns rhs_u(2:nx-1, 2:nyg-1, 2:nzg-1) as a
    dense array of shape (nx-2, nyg-2, nzg-2)."""
    nx, ny, nz, nyg, nzg = g.nx, g.ny, g.nz, g.nyg, g.nzg
    x, y, z, xg, yg, zg, nu = g.x, g.y, g.z, g.xg, g.yg, g.zg, g.p["nu"]
    I, J, K = slice(2, nx), slice(2, nyg), slice(2, nzg)
    # 1) -du^2/dx  (:43-57): centres i=2..nx
    a = 0.5 * (U[1:nx, J, K] + U[2:nx + 1, J, K])
    a = a * a
    rhs = -(a[1:] - a[:-1]) / _col(xg[3:nx + 1] - xg[2:nx])
    # 2) -duv/dy (:62-79): j = 1..ny
    b = (0.5 * (U[I, 1:ny + 1, K] + U[I, 2:ny + 2, K])) * \
        (0.5 * (V[2:nx, 1:ny + 1, K] + V[3:nx + 1, 1:ny + 1, K]))
    rhs = rhs + (-(b[:, 1:] - b[:, :-1]) / _row(y[2:ny + 1] - y[1:ny]))
    # 3) -duw/dz (:84-101): k = 1..nz
    c = (0.5 * (U[I, J, 1:nz + 1] + U[I, J, 2:nz + 2])) * \
        (0.5 * (W[2:nx, J, 1:nz + 1] + W[3:nx + 1, J, 1:nz + 1]))
    rhs = rhs + (-(c[:, :, 1:] - c[:, :, :-1]) / _dep(z[2:nz + 1] - z[1:nz]))
    # 4) viscous (:108-144)
    dUdy = (U[I, 2:nyg + 1, K] - U[I, 1:nyg, K]) / _row(yg[2:nyg + 1] - yg[1:nyg])  # j=1..nyg-1
    dx1 = _col(x[2:nx] - x[1:nx - 1]); dx2 = _col(x[3:nx + 1] - x[2:nx]); dx3 = _col(xg[3:nx + 1] - xg[2:nx])
    dy3 = _row(y[2:nyg] - y[1:nyg - 1])
    dz1 = _dep(zg[2:nzg] - zg[1:nzg - 1]); dz2 = _dep(zg[3:nzg + 1] - zg[2:nzg]); dz3 = _dep(z[2:nzg] - z[1:nzg - 1])
    Uc = U[I, J, K]
    visc = (1.0 / dx3 * (nu * 1.0 / dx2 * (U[3:nx + 1, J, K] - Uc) - nu * 1.0 / dx1 * (Uc - U[1:nx - 1, J, K]))
            + 1.0 / dy3 * (nu * dUdy[:, 1:] - nu * dUdy[:, :-1])
            + 1.0 / dz3 * (nu * 1.0 / dz2 * (U[I, J, 3:nzg + 1] - Uc) - nu * 1.0 / dz1 * (Uc - U[I, J, 1:nzg - 1])))
    rhs = rhs + visc
    # constant pressure gradient (:147-151)
    if exterior_pressure_gradient and Hu is not None:
        rhs = rhs + dPdx * Hu[I, J, K]
    else:
        rhs = rhs + dPdx
    return rhs


def compute_rhs_v(g, U, V, W, dPdy, Hv=None, exterior_pressure_gradient=True):
    """src/equations.f90:160-288.  Returns rhs_v(2:nxg-1, 2:ny-1, 2:nzg-1)."""
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    x, y, z, xg, yg, zg, nu = g.x, g.y, g.z, g.xg, g.yg, g.zg, g.p["nu"]
    I, J, K = slice(2, nxg), slice(2, ny), slice(2, nzg)
    # 1) -dv^2/dy (:179-193): centres j=2..ny
    a = 0.5 * (V[I, 1:ny, K] + V[I, 2:ny + 1, K])
    a = a * a
    rhs = -(a[:, 1:] - a[:, :-1]) / _row(yg[3:ny + 1] - yg[2:ny])
    # 2) -duv/dx (:198-215): i = 1..nx
    b = (0.5 * (U[1:nx + 1, J, K] + U[1:nx + 1, 3:ny + 1, K])) * \
        (0.5 * (V[1:nx + 1, J, K] + V[2:nx + 2, J, K]))
    rhs = rhs + (-(b[1:] - b[:-1]) / _col(x[2:nx + 1] - x[1:nx]))
    # 3) -dvw/dz (:220-237): k = 1..nz
    c = (0.5 * (V[I, J, 1:nz + 1] + V[I, J, 2:nz + 2])) * \
        (0.5 * (W[I, J, 1:nz + 1] + W[I, 3:ny + 1, 1:nz + 1]))
    rhs = rhs + (-(c[:, :, 1:] - c[:, :, :-1]) / _dep(z[2:nz + 1] - z[1:nz]))
    # 4) viscous (:246-279)
    dx1 = _col(xg[2:nxg] - xg[1:nxg - 1]); dx2 = _col(xg[3:nxg + 1] - xg[2:nxg]); dx3 = _col(x[2:nxg] - x[1:nxg - 1])
    dy1 = _row(y[2:ny] - y[1:ny - 1]); dy2 = _row(y[3:ny + 1] - y[2:ny]); dy3 = _row(yg[3:ny + 1] - yg[2:ny])
    dz1 = _dep(zg[2:nzg] - zg[1:nzg - 1]); dz2 = _dep(zg[3:nzg + 1] - zg[2:nzg]); dz3 = _dep(z[2:nzg] - z[1:nzg - 1])
    Vc = V[I, J, K]
    visc = (1.0 / dx3 * (nu * 1.0 / dx2 * (V[3:nxg + 1, J, K] - Vc) - nu * 1.0 / dx1 * (Vc - V[1:nxg - 1, J, K]))
            + 1.0 / dy3 * (nu * 1.0 / dy2 * (V[I, 3:ny + 1, K] - Vc) - nu * 1.0 / dy1 * (Vc - V[I, 1:ny - 1, K]))
            + 1.0 / dz3 * (nu * 1.0 / dz2 * (V[I, J, 3:nzg + 1] - Vc) - nu * 1.0 / dz1 * (Vc - V[I, J, 1:nzg - 1])))
    rhs = rhs + visc
    if exterior_pressure_gradient and Hv is not None:
        rhs = rhs + dPdy * Hv[I, J, K]
    else:
        rhs = rhs + dPdy
    return rhs


def compute_rhs_w(g, U, V, W, dPdz, Hw=None, exterior_pressure_gradient=True):
    """src/equations.f90:295-423.  Returns rhs_w(2:nxg-1, 2:nyg-1, 2:nz-1)."""
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    x, y, z, xg, yg, zg, nu = g.x, g.y, g.z, g.xg, g.yg, g.zg, g.p["nu"]
    I, J, K = slice(2, nxg), slice(2, nyg), slice(2, nz)
    # 1) -dw^2/dz (:314-328): centres k=2..nz
    a = 0.5 * (W[I, J, 1:nz] + W[I, J, 2:nz + 1])
    a = a * a
    rhs = -(a[:, :, 1:] - a[:, :, :-1]) / _dep(zg[3:nz + 1] - zg[2:nz])
    # 2) -duw/dx (:333-350): i = 1..nx
    b = (0.5 * (U[1:nx + 1, J, K] + U[1:nx + 1, J, 3:nz + 1])) * \
        (0.5 * (W[1:nx + 1, J, K] + W[2:nx + 2, J, K]))
    rhs = rhs + (-(b[1:] - b[:-1]) / _col(x[2:nx + 1] - x[1:nx]))
    # 3) -dvw/dy (:355-372): j = 1..ny
    c = (0.5 * (V[I, 1:ny + 1, K] + V[I, 1:ny + 1, 3:nz + 1])) * \
        (0.5 * (W[I, 1:ny + 1, K] + W[I, 2:ny + 2, K]))
    rhs = rhs + (-(c[:, 1:] - c[:, :-1]) / _row(y[2:ny + 1] - y[1:ny]))
    # 4) viscous (:378-414)
    dWdy = (W[I, 2:nyg + 1, K] - W[I, 1:nyg, K]) / _row(yg[2:nyg + 1] - yg[1:nyg])
    dx1 = _col(xg[2:nxg] - xg[1:nxg - 1]); dx2 = _col(xg[3:nxg + 1] - xg[2:nxg]); dx3 = _col(x[2:nxg] - x[1:nxg - 1])
    dy3 = _row(y[2:nyg] - y[1:nyg - 1])
    dz1 = _dep(z[2:nz] - z[1:nz - 1]); dz2 = _dep(z[3:nz + 1] - z[2:nz]); dz3 = _dep(zg[3:nz + 1] - zg[2:nz])
    Wc = W[I, J, K]
    visc = (1.0 / dx3 * (nu * 1.0 / dx2 * (W[3:nxg + 1, J, K] - Wc) - nu * 1.0 / dx1 * (Wc - W[1:nxg - 1, J, K]))
            + 1.0 / dy3 * (nu * dWdy[:, 1:] - nu * dWdy[:, :-1])
            + 1.0 / dz3 * (nu * 1.0 / dz2 * (W[I, J, 3:nz + 1] - Wc) - nu * 1.0 / dz1 * (Wc - W[I, J, 1:nz - 1])))
    rhs = rhs + visc
    if exterior_pressure_gradient and Hw is not None:
        rhs = rhs + dPdz * Hw[I, J, K]
    else:
        rhs = rhs + dPdz
    return rhs


# --------------------------------------------------------------------------
# differential operators, src/differential_operators.f90
# --------------------------------------------------------------------------
def divergence(g, U, V, W):
    """src/differential_operators.f90:54-74; returns a fresh rhs_p array."""
    d = g.rhs_p_array()
    nxg, nyg, nzg = g.nxg, g.nyg, g.nzg
    x, y, z = g.x, g.y, g.z
    I, J, K = slice(2, nxg), slice(2, nyg), slice(2, nzg)
    d[I, J, K] = ((U[I, J, K] - U[1:nxg - 1, J, K]) / _col(x[2:nxg] - x[1:nxg - 1])
                  + (V[I, J, K] - V[I, 1:nyg - 1, K]) / _row(y[2:nyg] - y[1:nyg - 1])
                  + (W[I, J, K] - W[I, J, 1:nzg - 1]) / _dep(z[2:nzg] - z[1:nzg - 1]))
    return d


def gradient(g, p_):
    """src/differential_operators.f90:16-52; p_ is an rhs_p-shaped array.
    Returns (Gpx, Gpy, Gpz) with U/V/W extents, zero outside the loops."""
    nx, ny, nz, nyg, nzg = g.nx, g.ny, g.nz, g.nyg, g.nzg
    xg, yg, zg = g.xg, g.yg, g.zg
    Gx, Gy, Gz = g.u_array(), g.v_array(), g.w_array()
    I = slice(2, nx)
    Gx[I, 2:nyg, 2:nzg] = (p_[3:nx + 1, 2:nyg, 2:nzg] - p_[I, 2:nyg, 2:nzg]) / _col(xg[3:nx + 1] - xg[2:nx])
    Gy[I, 2:ny, 2:nzg] = (p_[I, 3:ny + 1, 2:nzg] - p_[I, 2:ny, 2:nzg]) / _row(yg[3:ny + 1] - yg[2:ny])
    Gz[I, 2:nyg, 2:nz] = (p_[I, 2:nyg, 3:nz + 1] - p_[I, 2:nyg, 2:nz]) / _dep(zg[3:nz + 1] - zg[2:nz])
    return Gx, Gy, Gz


# --------------------------------------------------------------------------
# Poisson solve, src/poisson.f90:33-156
# --------------------------------------------------------------------------
def _zgtsv(dl, d, du, b):
    """LAPACK zgtsv (the reference's call, src/poisson.f90:72); b is (n, nrhs)."""
    _, _, _, xsol, info = lapack.zgtsv(dl.astype(np.complex128), d.astype(np.complex128),
                                        du.astype(np.complex128), b)
    if info != 0:
        raise FloatingPointError(f"zgtsv info={info}")
    return xsol


def solve_poisson_equation(g, rhs, state=None, rk_step=0, dt=None):
    """In-place solve of L_h phi = rhs on rhs(2:nxg-1, 2:nyg-1, 2:nzg).

    src/poisson.f90:33-101: per-y-plane 2-D complex DFT (:43-47), per-mode
    tridiagonal ``Zgtsv`` with the 00-mode pin D(2) *= 3/2 (:50-75), inverse
    DFT divided by nxp*nzp keeping the real part (:78-82), periodic copies
    (:85, :106-125) and, at ``rk_step == 1``, the ``P`` side effect (:91-99).
    Modes sharing a matrix (kxx(i)=kxx(nxp-i), kzz(k)=kzz(nzp-k)) are solved
    as one multi-right-hand-side ``zgtsv`` call; column-wise this is the same
    arithmetic as separate calls.
    """
    nxp, nzp, nyg = g.nxp, g.nzp, g.nyg
    J = slice(2, nyg)
    plane = rhs[2:nxp + 2, J, 2:nzp + 2]               # (nxp, nym, nzp)
    hat = np.fft.fft2(plane, axes=(0, 2))              # forward, unnormalised
    dd = g.Dd[2:nyg]
    dl = g.Dl[3:nyg]       # Dyy(j+1,j), j=2..nyg-2
    du = g.Du[2:nyg - 1]   # Dyy(j,j+1)
    for i in range(0, nxp // 2 + 1):
        ii = sorted({i, (nxp - i) % nxp})
        for k in range(0, nzp // 2 + 1):
            kk = sorted({k, (nzp - k) % nzp})
            D = (dd + g.kxx[i]) + g.kzz[k]
            if i == 0 and k == 0:
                D = D.copy()
                D[0] = 3.0 / 2.0 * D[0]
            cols = [(a, c) for a in ii for c in kk]
            B = np.stack([hat[a, :, c] for (a, c) in cols], axis=1)
            Xs = _zgtsv(dl, D, du, B)
            for n, (a, c) in enumerate(cols):
                hat[a, :, c] = Xs[:, n]
    out = np.fft.ifft2(hat, axes=(0, 2))               # includes 1/(nxp*nzp)
    rhs[2:nxp + 2, J, 2:nzp + 2] = out.real
    # apply_periodic_xz_centers (:106-125): x copy on every plane, then z copy
    rhs[g.nxg - 1, :, :] = rhs[2, :, :]
    rhs[2:g.nxg, :, nzp + 2] = rhs[2:g.nxg, :, 2]
    # update_ghost_interior_planes_centers (:130-156) is a no-op on one domain:
    # plane nzg is left as it was (zero after `divergence`).
    if rk_step == 1 and state is not None:
        _pressure_side_effect(g, state, rhs, dt)
    return rhs


def _pressure_side_effect(g, st, rhs, dt):
    """src/poisson.f90:91-99 (P = rhs/(dt*rk_coef(1,1)) and copies)."""
    P = st.P
    nxg, nyg, nzg = g.nxg, g.nyg, g.nzg
    P[2:nxg, 2:nyg, 2:nzg] = rhs[2:nxg, 2:nyg, 2:nzg] / (dt * RK_COEF[0][0])
    P[1, :, :] = P[2, :, :]
    P[nxg, :, :] = P[nxg - 1, :, :]
    P[:, 1, :] = P[:, 2, :]
    P[:, nyg, :] = P[:, nyg - 1, :]
    P[:, :, 1] = P[:, :, 2]
    P[:, :, nzg] = P[:, :, nzg - 1]


# --------------------------------------------------------------------------
# actual pressure, src/pressure.f90:21-341
# --------------------------------------------------------------------------
def compute_pressure_bc(g, V):
    """src/pressure.f90:270-341: bc_1, bc_2 = d/dy(nu dV/dy) at the walls by
    one-sided second-order differences in the grid index (dzeta = 1), as
    arrays over (i, k) = (2..nxg-1, 2..nzg-1) (shape (nxg+1, nzg+1), Fortran
    indexed)."""
    y, ny, nxg, nzg, nu = g.y, g.ny, g.nxg, g.nzg, g.p["nu"]
    dzeta = 1.0
    bc1 = np.zeros((nxg + 1, nzg + 1))
    bc2 = np.zeros((nxg + 1, nzg + 1))
    I, K = slice(2, nxg), slice(2, nzg)
    gm = (-3.0 * y[1] + 4.0 * y[2] - y[3]) / (2.0 * dzeta)
    g2 = (2.0 * y[1] - 5.0 * y[2] + 4.0 * y[3] - 1.0 * y[4]) / dzeta ** 2.0
    dV = (-3.0 * V[I, 1, K] + 4.0 * V[I, 2, K] - V[I, 3, K]) / (2.0 * dzeta) * 1.0 / gm
    ddV = (2.0 * V[I, 1, K] - 5.0 * V[I, 2, K] + 4.0 * V[I, 3, K] - 1.0 * V[I, 4, K]) / dzeta ** 2.0
    ddV = (ddV - dV * g2) / gm ** 2.0
    bc1[I, K] = 0.0 * dV + nu * ddV
    gm = (3.0 * y[ny] - 4.0 * y[ny - 1] + y[ny - 2]) / (2.0 * dzeta)
    g2 = (2.0 * y[ny] - 5.0 * y[ny - 1] + 4.0 * y[ny - 2] - 1.0 * y[ny - 3]) / dzeta ** 2.0
    dV = (3.0 * V[I, ny, K] - 4.0 * V[I, ny - 1, K] + V[I, ny - 2, K]) / (2.0 * dzeta) * 1.0 / gm
    ddV = (2.0 * V[I, ny, K] - 5.0 * V[I, ny - 1, K] + 4.0 * V[I, ny - 2, K]
           - 1.0 * V[I, ny - 3, K]) / dzeta ** 2.0
    ddV = (ddV - dV * g2) / gm ** 2.0
    bc2[I, K] = 0.0 * dV + nu * ddV
    return bc1, bc2


def compute_pressure_rhs(g, st, bc1, bc2, Hu=None, Hv=None, Hw=None):
    """src/pressure.f90:42-70: rhs_p = div(rhs_uf, rhs_vf, rhs_wf) with the
    periodic copies of rhs_uf in x and rhs_wf in z and bc_1/bc_2 as the wall
    values of rhs_vf."""
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    epg = g.p["exterior_pressure_gradient"]
    ruf, rvf, rwf = g.u_array(), g.v_array(), g.w_array()
    ruf[2:nx, 2:nyg, 2:nzg] = compute_rhs_u(g, st.U, st.V, st.W, st.dPdx, Hu, epg)
    rvf[2:nxg, 2:ny, 2:nzg] = compute_rhs_v(g, st.U, st.V, st.W, st.dPdy, Hv, epg)
    rwf[2:nxg, 2:nyg, 2:nz] = compute_rhs_w(g, st.U, st.V, st.W, st.dPdz, Hw, epg)
    apply_periodic_bc_x(g, ruf, True)                  # compute_rhs_v_boundary (:237-247)
    rvf[2:nxg, 1, 2:nzg] = bc1[2:nxg, 2:nzg]
    rvf[2:nxg, ny, 2:nzg] = bc2[2:nxg, 2:nzg]
    apply_periodic_bc_z(g, rwf, True)
    x, y, z = g.x, g.y, g.z
    rhs = g.rhs_p_array()
    I, J, K = slice(2, nxg), slice(2, nyg), slice(2, nzg)
    rhs[I, J, K] = ((ruf[I, J, K] - ruf[1:nxg - 1, J, K]) / _col(x[2:nxg] - x[1:nxg - 1])
                    + (rvf[I, J, K] - rvf[I, 1:nyg - 1, K]) / _row(y[2:nyg] - y[1:nyg - 1])
                    + (rwf[I, J, K] - rwf[I, J, 1:nzg - 1]) / _dep(z[2:nzg] - z[1:nzg - 1]))
    return rhs


def solve_poisson_equation_for_pressure(g, rhs, bc1, bc2, P):
    """src/pressure.f90:90-165: the Poisson solve of the projection with the
    inhomogeneous Neumann rows (coef_bc_1, coef_bc_2 of
    src/initialization.f90:374,383), then P(2:nxg-2, 2:nyg-1, 2:nzg-2), its
    y ghosts P(1) = P(2) - (yg(2)-yg(1)) bc_1 and P(nyg) = P(nyg-1) +
    (yg(nyg)-yg(nyg-1)) bc_2, and the periodic copies (:173-187).

    The y-ghost assignment of the reference (:160-161) takes a whole (nxg, nzg)
    section of P from bc_1, which is allocated (2:nxg-1, 2:nzg-1)
    (src/initialization.f90:385): the shapes do not conform.  It is applied
    here over bc_1's domain (i, k) = (2..nxg-1, 2..nzg-1); the x and z ghost
    planes of P (i = 1, nxg; k = 1, nzg) keep their values."""
    nxp, nzp, nyg, nxg, nzg = g.nxp, g.nzp, g.nyg, g.nxg, g.nzg
    y, yg = g.y, g.yg
    J = slice(2, nyg)
    hat = np.fft.fft2(rhs[2:nxp + 2, J, 2:nzp + 2], axes=(0, 2))
    b1 = np.fft.fft2(bc1[2:nxp + 2, 2:nzp + 2])
    b2 = np.fft.fft2(bc2[2:nxp + 2, 2:nzp + 2])
    j = 2
    coef_bc_1 = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1])
    j = nyg - 1
    coef_bc_2 = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j])
    dd, dl, du = g.Dd[2:nyg], g.Dl[3:nyg], g.Du[2:nyg - 1]
    for i in range(nxp):
        ia = min(i, nxp - i)
        for k in range(nzp):
            ka = min(k, nzp - k)
            D = (dd + g.kxx[ia]) + g.kzz[ka]
            if i == 0 and k == 0:
                D = D.copy()
                D[0] = 3.0 / 2.0 * D[0]
            r = hat[i, :, k].copy()
            r[0] = r[0] + coef_bc_1 * (yg[2] - yg[1]) * b1[i, k]
            r[-1] = r[-1] - coef_bc_2 * (yg[nyg] - yg[nyg - 1]) * b2[i, k]
            hat[i, :, k] = _zgtsv(dl, D, du, r.reshape(-1, 1))[:, 0]
    out = np.fft.ifft2(hat, axes=(0, 2))
    P[2:nxp + 2, J, 2:nzp + 2] = out.real
    I, K = slice(2, nxg), slice(2, nzg)
    P[I, 1, K] = P[I, 2, K] - (yg[2] - yg[1]) * bc1[I, K]
    P[I, nyg, K] = P[I, nyg - 1, K] + (yg[nyg] - yg[nyg - 1]) * bc2[I, K]
    P[nxg - 1, :, :] = P[2, :, :]                      # apply_periodic_xz_pressure
    P[2:nxg, :, nzp + 2] = P[2:nxg, :, 2]
    return P


def compute_pressure(g, st, Hu=None, Hv=None, Hw=None):
    """src/pressure.f90:21-29 on st.P (in place)."""
    bc1, bc2 = compute_pressure_bc(g, st.V)
    rhs = compute_pressure_rhs(g, st, bc1, bc2, Hu, Hv, Hw)
    solve_poisson_equation_for_pressure(g, rhs, bc1, bc2, st.P)
    return st.P


# --------------------------------------------------------------------------
# mass flow, src/mass_flow.f90
# --------------------------------------------------------------------------
def mean_mass_flow_u(g, U, Hu=None):
    """src/mass_flow.f90:24-53 (also the integral of :144-175)."""
    nx, nyg, nzg, yg = g.nx, g.nyg, g.nzg, g.yg
    if Hu is None:
        Hu = np.ones_like(U)
    I, K = slice(2, nx), slice(2, nzg)
    w = _row(0.5 * (yg[3:nyg] - yg[2:nyg - 1]))
    HU = Hu[I, 2:nyg, K] * U[I, 2:nyg, K]
    q = float(np.sum((HU[:, 1:] + HU[:, :-1]) * w))
    H = Hu[I, 2:nyg, K]
    norm = float(np.sum((H[:, 1:] + H[:, :-1]) * w))
    return q, norm


def compute_dPx_for_constant_mass_flow(g, U, Qflow_x_0, Hu=None):
    """src/mass_flow.f90:144-175: dPdx = Qflow_x_0 - Int_U/norm."""
    q, norm = mean_mass_flow_u(g, U, Hu)
    return Qflow_x_0 - q / norm


def mean_mass_flow_v(g, V, Hv=None):
    """src/mass_flow.f90:62-91 (also the integral of :190-221): trapezoid of
    H*V between y(1:ny) over i = 2..nxg-1, k = 2..nzg-1."""
    nxg, ny, nzg, y = g.nxg, g.ny, g.nzg, g.y
    if Hv is None:
        Hv = np.ones_like(V)
    I, K = slice(2, nxg), slice(2, nzg)
    w = _row(0.5 * (y[2:ny + 1] - y[1:ny]))
    HV = Hv[I, 1:ny + 1, K] * V[I, 1:ny + 1, K]
    q = float(np.sum((HV[:, 1:] + HV[:, :-1]) * w))
    H = Hv[I, 1:ny + 1, K]
    norm = float(np.sum((H[:, 1:] + H[:, :-1]) * w))
    return q, norm


def mean_mass_flow_w(g, W, Hw=None):
    """src/mass_flow.f90:100-129: trapezoid of H*W between yg(2:nyg-1) over
    i = 2..nxg-1, k = 2..nz-1."""
    nxg, nyg, nz, yg = g.nxg, g.nyg, g.nz, g.yg
    if Hw is None:
        Hw = np.ones_like(W)
    I, K = slice(2, nxg), slice(2, nz)
    w = _row(0.5 * (yg[3:nyg] - yg[2:nyg - 1]))
    HW = Hw[I, 2:nyg, K] * W[I, 2:nyg, K]
    q = float(np.sum((HW[:, 1:] + HW[:, :-1]) * w))
    H = Hw[I, 2:nyg, K]
    norm = float(np.sum((H[:, 1:] + H[:, :-1]) * w))
    return q, norm


def compute_dPy_for_constant_mass_flow(g, V, Qflow_y_0, Hv=None):
    """src/mass_flow.f90:190-221: dPdy = Qflow_y_0 - Int_V/norm."""
    q, norm = mean_mass_flow_v(g, V, Hv)
    return Qflow_y_0 - q / norm


def compute_dPz_for_constant_mass_flow(g, W, Qflow_z_0, Hw=None):
    """src/mass_flow.f90:236-267: dPdz = Qflow_z_0 - Int_W/norm.

    The routine declares its dummy W with the extents of U,
    ``Dimension(nx,nyg,nzg)`` (:238), while the actual argument is W(nxg,nyg,nz):
    its W(i,j,k) is the element at Fortran offset (i-1) + nx*((j-1) + nyg*(k-1))
    of the real W.  That is what is read here (every offset the loops reach
    lies inside W).  Hw_interior is the module array with its own extents."""
    nx, nxg, nyg, nz, yg = g.nx, g.nxg, g.nyg, g.nz, g.yg
    flat = np.asarray(W)[1:, 1:, 1:].ravel(order="F")
    if Hw is None:
        Hw = np.ones_like(W)
    i = np.arange(2, nxg)[:, None, None]
    j = np.arange(3, nyg)[None, :, None]
    k = np.arange(2, nz)[None, None, :]
    off = lambda ii, jj, kk: (ii - 1) + nx * ((jj - 1) + nyg * (kk - 1))
    Wa, Wb = flat[off(i, j, k)], flat[off(i, j - 1, k)]
    Ha, Hb = Hw[2:nxg, 3:nyg, 2:nz], Hw[2:nxg, 2:nyg - 1, 2:nz]
    w = _row(0.5 * (yg[3:nyg] - yg[2:nyg - 1]))
    q = float(np.sum((Ha * Wa + Hb * Wb) * w))
    norm = float(np.sum((Ha + Hb) * w))
    return Qflow_z_0 - q / norm


# --------------------------------------------------------------------------
# full state and the RK3 step
# --------------------------------------------------------------------------
class State:
    """Flow state of the reference's module globals used by the hot path."""

    def __init__(self, g):
        self.U, self.V, self.W, self.P = g.u_array(), g.v_array(), g.w_array(), g.p_array()
        self.P_interim = g.rhs_p_array()
        self.t = 0.0
        self.dPdx = 0.0
        self.dPdy = 0.0
        self.dPdz = 0.0
        self.Qflow_x_0 = 0.0
        self.Qflow_y_0 = 0.0
        self.Qflow_z_0 = 0.0

    def copy(self):
        s = State.__new__(State)
        for k, v in self.__dict__.items():
            s.__dict__[k] = v.copy() if isinstance(v, np.ndarray) else v
        return s


def compute_non_IB_projection(g, st, dt, rk_step=0):
    """src/projection.f90:22-46."""
    U_i, V_i, W_i = st.U.copy(), st.V.copy(), st.W.copy()
    rhs_p = divergence(g, st.U, st.V, st.W)
    solve_poisson_equation(g, rhs_p, st, rk_step, dt)
    rhs_p = rhs_p / dt
    st.P_interim = rhs_p.copy()
    rhs_p = dt * rhs_p
    Gx, Gy, Gz = gradient(g, rhs_p)
    st.U = U_i - Gx
    st.V = V_i - Gy
    st.W = W_i - Gz


def compute_time_step_RK3(g, st, dt):
    """src/time_integration.f90:86-213 for body_type='none'."""
    p = g.p
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    to = st.t
    Uo, Vo, Wo = st.U.copy(), st.V.copy(), st.W.copy()
    Iu, Ju, Ku = slice(2, nx), slice(2, nyg), slice(2, nzg)
    Iv, Jv, Kv = slice(2, nxg), slice(2, ny), slice(2, nzg)
    Iw, Jw, Kw = slice(2, nxg), slice(2, nyg), slice(2, nz)
    epg = p["exterior_pressure_gradient"]
    Fu, Fv, Fw = [], [], []
    for s in range(3):
        Fu.append(compute_rhs_u(g, st.U, st.V, st.W, st.dPdx, None, epg))
        Fv.append(compute_rhs_v(g, st.U, st.V, st.W, st.dPdy, None, epg))
        Fw.append(compute_rhs_w(g, st.U, st.V, st.W, st.dPdz, None, epg))
        c = RK_COEF[s]
        if s == 0:
            du, dv, dw = c[0] * Fu[0], c[0] * Fv[0], c[0] * Fw[0]
        elif s == 1:
            du = c[0] * Fu[0] + c[1] * Fu[1]
            dv = c[0] * Fv[0] + c[1] * Fv[1]
            dw = c[0] * Fw[0] + c[1] * Fw[1]
        else:
            du = c[0] * Fu[0] + c[1] * Fu[1] + c[2] * Fu[2]
            dv = c[0] * Fv[0] + c[1] * Fv[1] + c[2] * Fv[2]
            dw = c[0] * Fw[0] + c[1] * Fw[1] + c[2] * Fw[2]
        if s == 0:
            st.U[Iu, Ju, Ku] = Uo[Iu, Ju, Ku] + dt * c[0] * Fu[0]
            st.V[Iv, Jv, Kv] = Vo[Iv, Jv, Kv] + dt * c[0] * Fv[0]
            st.W[Iw, Jw, Kw] = Wo[Iw, Jw, Kw] + dt * c[0] * Fw[0]
        else:
            st.U[Iu, Ju, Ku] = Uo[Iu, Ju, Ku] + dt * du
            st.V[Iv, Jv, Kv] = Vo[Iv, Jv, Kv] + dt * dv
            st.W[Iw, Jw, Kw] = Wo[Iw, Jw, Kw] + dt * dw
        st.t = to + RK_T[s] * dt
        apply_boundary_conditions(g, st.U, st.V, st.W)
        compute_non_IB_projection(g, st, dt, rk_step=s + 1)
        apply_boundary_conditions(g, st.U, st.V, st.W)
    if p["x_mass_cte"] == 1:                             # :187-193
        dPdx_prev = st.dPdx
        shift = compute_dPx_for_constant_mass_flow(g, st.U, st.Qflow_x_0)
        st.U[Iu, Ju, Ku] = st.U[Iu, Ju, Ku] + shift
        st.dPdx = 0.5 * (dPdx_prev + shift / dt)
        apply_boundary_conditions(g, st.U, st.V, st.W)
    if p.get("y_mass_cte", 0) == 1:                      # :196-202
        dPdy_prev = st.dPdy
        shift = compute_dPy_for_constant_mass_flow(g, st.V, st.Qflow_y_0)
        st.V[Iv, Jv, Kv] = st.V[Iv, Jv, Kv] + shift
        st.dPdy = 0.5 * (dPdy_prev + shift / dt)
        apply_boundary_conditions(g, st.U, st.V, st.W)
    if p.get("z_mass_cte", 0) == 1:                      # :205-211
        dPdz_prev = st.dPdz
        shift = compute_dPz_for_constant_mass_flow(g, st.W, st.Qflow_z_0)
        st.W[Iw, Jw, Kw] = st.W[Iw, Jw, Kw] + shift
        st.dPdz = 0.5 * (dPdz_prev + shift / dt)
        apply_boundary_conditions(g, st.U, st.V, st.W)
    return st


def compute_time_step_Euler(g, st, dt, Hu=None, Hv=None, Hw=None):
    """src/time_integration.f90:25-81: explicit Euler with rk_step = 3 (no P
    side effect), the non-IB projection, and the x and y constant-flux
    corrections with dPd = shift/dt (no averaging; no z correction)."""
    p = g.p
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    Uo, Vo, Wo = st.U.copy(), st.V.copy(), st.W.copy()
    epg = p["exterior_pressure_gradient"]
    ru = compute_rhs_u(g, Uo, Vo, Wo, st.dPdx, Hu, epg)
    st.U[2:nx, 2:nyg, 2:nzg] = Uo[2:nx, 2:nyg, 2:nzg] + dt * ru
    rv = compute_rhs_v(g, Uo, Vo, Wo, st.dPdy, Hv, epg)
    st.V[2:nxg, 2:ny, 2:nzg] = Vo[2:nxg, 2:ny, 2:nzg] + dt * rv
    rw = compute_rhs_w(g, Uo, Vo, Wo, st.dPdz, Hw, epg)
    st.W[2:nxg, 2:nyg, 2:nz] = Wo[2:nxg, 2:nyg, 2:nz] + dt * rw
    st.t = st.t + dt
    apply_boundary_conditions(g, st.U, st.V, st.W)
    compute_non_IB_projection(g, st, dt, rk_step=3)
    apply_boundary_conditions(g, st.U, st.V, st.W)
    if p["x_mass_cte"] == 1:                             # :65-70
        shift = compute_dPx_for_constant_mass_flow(g, st.U, st.Qflow_x_0, Hu)
        st.U[2:nx, 2:nyg, 2:nzg] = st.U[2:nx, 2:nyg, 2:nzg] + shift
        st.dPdx = shift / dt
        apply_boundary_conditions(g, st.U, st.V, st.W)
    if p.get("y_mass_cte", 0) == 1:                      # :73-78 (walls included)
        shift = compute_dPy_for_constant_mass_flow(g, st.V, st.Qflow_y_0, Hv)
        st.V[2:nxg, 1:ny + 1, 2:nzg] = st.V[2:nxg, 1:ny + 1, 2:nzg] + shift
        st.dPdy = shift / dt
        apply_boundary_conditions(g, st.U, st.V, st.W)
    return st


def compute_dt(g, st):
    """src/time_integration.f90:219-267 (CFL < 0 gives dt = -CFL)."""
    p = g.p
    cfl = p["cfl"]
    if cfl < 0:
        return -cfl
    nxg, nyg, nzg = g.nxg, g.nyg, g.nzg
    I, J, K = slice(2, nxg), slice(2, nyg), slice(2, nzg)
    with np.errstate(divide="ignore"):
        lU = np.max(_col(g.xg[3:nxg + 1] - g.xg[2:nxg]) / np.abs(st.U[I, J, K]))
        lV = np.max(_row(g.yg[3:nyg + 1] - g.yg[2:nyg]) / np.abs(st.V[I, J, K]))
        lW = np.max(_dep(g.zg[3:nzg + 1] - g.zg[2:nzg]) / np.abs(st.W[I, J, K]))
    lU, lV, lW = max(0.0, lU), max(0.0, lV), max(0.0, lW)
    dt_conv = min(cfl * lU, cfl * lV, cfl * lW)
    nu = p["nu"]
    dt_vis = min(cfl * g.dxmin ** 2 / nu, cfl * g.dymin ** 2 / nu, cfl * g.dzmin ** 2 / nu)
    dt = min(dt_conv, dt_vis)
    return min(dt, 1e-1)


# --------------------------------------------------------------------------
# seeded initial state (replaces Intel rand() of src/input_output.f90:270-313)
# --------------------------------------------------------------------------
def seeded_initial_state(g, dPdx, amplitude=0.1, seed=0, project=True, dt=1e-3):
    """Laminar profile dPdx/(Ly*nu)*y*(Ly-y) (src/input_output.f90:275-280)
    plus uniform perturbations of peak ``amplitude`` (perturb_scale = 2*amplitude),
    drawn from NumPy PCG64(seed) in Fortran order for U, then V, then W;
    wall conditions as :288-313; all boundary conditions; one projection
    (dt cancels); boundary conditions again.  Qflow_x_0 from the result
    (app/main.f90:90)."""
    p = g.p
    st = State(g)
    rng = np.random.Generator(np.random.PCG64(seed))
    ps = 2.0 * amplitude
    Ly, nu = p["ly_channel"], p["nu"]
    U, V, W = st.U, st.V, st.W
    for jj in range(1, g.ny):
        ymv = 0.5 * (g.y[jj] + g.y[jj + 1])
        if 0.0 < ymv < Ly:
            U[1:, jj + 1, 1:] = dPdx / (Ly * nu) * ymv * (Ly - ymv)

    def draw(arr):
        shape = tuple(s - 1 for s in arr.shape)
        r = rng.random(shape[::-1]).T           # Fortran order, x fastest
        arr[1:, 1:, 1:] += ps * (r - 0.5)

    draw(U)
    U[:, 1, :] = -U[:, 2, :]
    U[:, g.ny + 1, :] = -U[:, g.ny, :]
    draw(V)
    V[:, 1, :] = 0.0
    V[:, g.ny, :] = 0.0
    draw(W)
    W[:, 1, :] = -W[:, 2, :]
    W[:, g.ny + 1, :] = -W[:, g.ny, :]
    apply_boundary_conditions(g, U, V, W)
    st.dPdx = dPdx
    if project:
        compute_non_IB_projection(g, st, dt)
        apply_boundary_conditions(g, st.U, st.V, st.W)
        st.P_interim[...] = 0.0
    q, norm = mean_mass_flow_u(g, st.U)
    st.Qflow_x_0 = q / norm
    q, norm = mean_mass_flow_w(g, st.W)                  # app/main.f90:91-92
    st.Qflow_z_0 = q / norm
    st.Qflow_y_0 = 0.0                                   # :93-94 (the V flux is
    st.dPdy = 0.0                                        # computed, then reset)
    return st


def channel_params(nx_global, ny_global, nz_global, Lxp, Lzp, nu, alpha=2.0,
                   dPdx=None, cfl=-1e-3, x_mass_cte=1, grid_type=1, **extra):
    """Parameter dict for a channel configuration of the benchmark workloads."""
    from .namelist import DEFAULTS
    p = dict(DEFAULTS)
    p.update(dict(nx_global=nx_global, ny_global=ny_global, nz_global=nz_global,
                  lxp=Lxp, lzp=Lzp, nu=nu, alpha_stretch=alpha,
                  dpdx=3.0 * nu if dPdx is None else dPdx, cfl=cfl,
                  x_mass_cte=x_mass_cte, grid_type=grid_type, ly_channel=2.0,
                  init_type=0))
    p.update(extra)
    return p
