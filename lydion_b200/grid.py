"""Host-side set-up of the spatial and frequency grids the Lyman-alpha step runs on.

This is the caller side of the drop-in boundary: in LYDION these arrays are built once by
Julia (SetupCylindricalGrid, GenerateLyaArrays) and handed to the step. The functions here
restate that set-up in numpy so the Python front end and the benchmarks can build the same
inputs:

* cylindrical geometry -- src/SpatialGrid.jl:26-170 (centroids, volumes, areas, <1/r>),
  src/SpatialGrid.jl:516-586 (PLM intervals with mirrored / extrapolated ghost centroids),
  src/SpatialGrid.jl:606-913 (uniform interfaces, and the logarithmic regions of N_r_log and
  N_Z_log_side cells whose widths grow by the ratio bisection finds);
* frequency grid -- src/SetupLymanAlphaArrays.jl:40-135 (symmetric, geometrically growing
  bins, core range), and the fixed-count variant used to inject a 48/64/128-bin grid
  through GenerateLyaArrays_FromSaved (src/SetupLymanAlphaArrays.jl:244-296).
"""
from dataclasses import dataclass, field

import numpy as np

from . import constants as K


def julia_linrange(a, b, n):
    """Julia LinRange(a, b, n) element values: (1 - i/d)*a + (i/d)*b with d = n-1."""
    d = n - 1
    t = np.arange(n, dtype=np.float64) / d
    return (1.0 - t) * a + t * b


@dataclass
class CylGeometry:
    """Mirror of the GeometryCylindrical fields the Lyman-alpha step reads."""
    r: np.ndarray
    Z: np.ndarray
    rCoM: np.ndarray
    ZCoM: np.ndarray
    dV: np.ndarray        # [j, i] (C order) == Julia ΔV[i, j]
    inv_dV: np.ndarray
    A_r: np.ndarray       # [j, f] f = 0..nr
    A_Z: np.ndarray       # [f, i] f = 0..nz
    inv_r_cell: np.ndarray
    dr_L: np.ndarray
    dr_R: np.ndarray
    inv_dr_i_im1: np.ndarray
    inv_dr_ip1_i: np.ndarray
    inv_dr_ip2_ip1: np.ndarray
    dr_b: np.ndarray      # 10: inner (L, R, i_im1, ip1_i, ip2_ip1), outer (same)
    dZ_L: np.ndarray
    dZ_R: np.ndarray
    inv_dZ_j_jm1: np.ndarray
    inv_dZ_jp1_j: np.ndarray
    inv_dZ_jp2_jp1: np.ndarray
    dZ_b: np.ndarray
    cartesian: bool = False   # GeometryCartesian: r, Z stand for X, Y

    @property
    def nr(self):
        return self.rCoM.size

    @property
    def nz(self):
        return self.ZCoM.size


def grid_differences(x, xc):
    """Compute_Grid_Differences!, src/SpatialGrid.jl:516-586.

    Returns (L, R, inv_i_im1, inv_ip1_i, inv_ip2_ip1, boundary[10])."""
    n = xc.size
    c0 = x[0] - (xc[0] - x[0])
    cm1 = x[0] - (xc[1] - x[0])
    cN1 = x[n] + (x[n] - xc[n - 1])
    cN2 = x[n] + (x[n] - xc[n - 2])
    bnd = np.empty(10)
    bnd[2] = 1.0 / (c0 - cm1)
    bnd[3] = 1.0 / (xc[0] - c0)
    bnd[4] = 1.0 / (xc[1] - xc[0])
    bnd[0] = x[0] - c0
    bnd[1] = xc[0] - x[0]
    L = np.empty(n); R = np.empty(n)
    a = np.empty(n); b = np.empty(n); c = np.empty(n)
    for i in range(n):
        cim1 = c0 if i == 0 else xc[i - 1]
        cip1 = cN1 if i == n - 1 else xc[i + 1]
        if i <= n - 3:
            cip2 = xc[i + 2]
        elif i == n - 2:
            cip2 = cN1
        else:
            cip2 = cN2
        a[i] = 1.0 / (xc[i] - cim1)
        b[i] = 1.0 / (cip1 - xc[i])
        c[i] = 1.0 / (cip2 - cip1)
        L[i] = x[i + 1] - xc[i]
        R[i] = cip1 - x[i + 1]
    bnd[7] = 1.0 / (xc[n - 1] - xc[n - 2])
    bnd[8] = 1.0 / (cN1 - xc[n - 1])
    bnd[9] = 1.0 / (cN2 - cN1)
    bnd[5] = x[n] - xc[n - 1]
    bnd[6] = cN1 - x[n]
    return L, R, a, b, c, bnd


def cylindrical_geometry(r, Z):
    """Geometry from interface coordinates, src/SpatialGrid.jl:26-170 and 842-891."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    Z = np.ascontiguousarray(Z, dtype=np.float64)
    nr, nz = r.size - 1, Z.size - 1
    if nr < 3 or nz < 3:
        raise ValueError("the M1 stencil needs N_r >= 3 and N_Z >= 3")
    if r[0] != 0.0:
        raise ValueError("innermost interface r[1] must be 0 in cylindrical coordinates")
    rp, rm = r[1:], r[:-1]
    rCoM = (2.0 / 3.0) * (rp * rp * rp - rm * rm * rm) / (rp * rp - rm * rm)
    ZCoM = 0.5 * (Z[:-1] + Z[1:])
    dZ = Z[1:] - Z[:-1]
    ring = np.pi * (rp * rp - rm * rm)
    dV = ring[None, :] * dZ[:, None]
    A_r = (2.0 * np.pi * r)[None, :] * dZ[:, None]
    A_Z = np.broadcast_to(ring[None, :], (nz + 1, nr)).copy()
    inv_r_cell = 2.0 / (rp + rm)
    rL, rR, ra, rb, rc, rbnd = grid_differences(r, rCoM)
    zL, zR, za, zb, zc, zbnd = grid_differences(Z, ZCoM)
    return CylGeometry(r=r, Z=Z, rCoM=rCoM, ZCoM=ZCoM, dV=dV, inv_dV=1.0 / dV, A_r=A_r, A_Z=A_Z,
                       inv_r_cell=inv_r_cell, dr_L=rL, dr_R=rR, inv_dr_i_im1=ra, inv_dr_ip1_i=rb,
                       inv_dr_ip2_ip1=rc, dr_b=rbnd, dZ_L=zL, dZ_R=zR, inv_dZ_j_jm1=za,
                       inv_dZ_jp1_j=zb, inv_dZ_jp2_jp1=zc, dZ_b=zbnd)


def cartesian_geometry(X, Y):
    """GeometryCartesian from interface coordinates (SetupCartesianGrid, src/SpatialGrid.jl:1349-1440):
    cell centres at the midpoints, dV = dX dY, A_X = dY and A_Y = dX per unit depth
    (src/SpatialGrid.jl:1061-1135), the same PLM intervals as the cylindrical Z coordinate
    (Compute_Grid_Differences!), and no <1/r>. Stored in the cylindrical field names (r = X,
    Z = Y)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    nx, ny = X.size - 1, Y.size - 1
    if nx < 3 or ny < 3:
        raise ValueError("the M1 stencil needs N_X >= 3 and N_Y >= 3")
    XC = 0.5 * (X[:-1] + X[1:])
    YC = 0.5 * (Y[:-1] + Y[1:])
    dX = X[1:] - X[:-1]
    dY = Y[1:] - Y[:-1]
    dV = dX[None, :] * dY[:, None]
    A_r = np.broadcast_to(dY[:, None], (ny, nx + 1)).copy()
    A_Z = np.broadcast_to(dX[None, :], (ny + 1, nx)).copy()
    rL, rR, ra, rb, rc, rbnd = grid_differences(X, XC)
    zL, zR, za, zb, zc, zbnd = grid_differences(Y, YC)
    return CylGeometry(r=X, Z=Y, rCoM=XC, ZCoM=YC, dV=dV, inv_dV=1.0 / dV, A_r=A_r, A_Z=A_Z,
                       inv_r_cell=np.zeros(nx), dr_L=rL, dr_R=rR, inv_dr_i_im1=ra, inv_dr_ip1_i=rb,
                       inv_dr_ip2_ip1=rc, dr_b=rbnd, dZ_L=zL, dZ_R=zR, inv_dZ_j_jm1=za,
                       inv_dZ_jp1_j=zb, inv_dZ_jp2_jp1=zc, dZ_b=zbnd, cartesian=True)


def uniform_cylindrical_geometry(rmax, zmax, nr, nz):
    """Uniform branch of SetupCylindricalGrid (N_r_log = N_Z_log_side = 0)."""
    return cylindrical_geometry(julia_linrange(0.0, rmax, nr + 1), julia_linrange(0.0, zmax, nz + 1))


def _isapprox(a, b, rtol):
    return abs(a - b) <= rtol * max(abs(a), abs(b))


def geometric_ratio(L, d, n):
    """The ratio q > 1 of n intervals d q, d q^2, ..., d q^n... that span L: the root of
    f(q) = L - d (q^n - 1) / (q - 1), found as SetupCylindricalGrid finds it
    (src/SpatialGrid.jl:693-716): a bracket [1 + 1e-14, 2] whose upper end doubles until
    f < 0, then bisection until the bracket cannot be split further in FP64."""
    f = lambda q: L - d * (q ** n - 1.0) / (q - 1.0)
    lo, hi = 1.0 + 1e-14, 2.0
    while f(hi) > 0.0:
        hi *= 2.0
        if hi > 1e12:
            raise ValueError("failed to bracket the ratio of the logarithmic grid")
    flo = f(lo)
    while True:
        mid = 0.5 * (lo + hi)
        if mid <= lo or mid >= hi:
            break
        fm = f(mid)
        if fm == 0.0:
            return mid
        if (fm > 0.0) == (flo > 0.0):
            lo, flo = mid, fm
        else:
            hi = mid
    return lo if abs(f(lo)) <= abs(f(hi)) else hi


def _log_tail(x0, d, L, n, sign=1.0):
    """The n - 1 interfaces beyond x0 (towards sign) of n cells spanning L that start at the
    uniform width d and grow geometrically (or stay uniform when n d already spans L)."""
    if _isapprox(L, n * d, 1e-12):
        return np.array([x0 + sign * k * d for k in range(1, n)])
    if L < n * d:
        raise ValueError("can't find a consistent logarithmic grid: use a larger range or a uniform grid")
    q = geometric_ratio(L, d, n)
    return np.array([x0 + sign * d * (q ** k - 1.0) / (q - 1.0) for k in range(1, n)])


def log_stretched_interfaces(rmax, rmax_lin, Zmax, LZ_uniform, N_r_lin, N_r_log, N_Z_lin, N_Z_log_side,
                             bc_z_bot="Reflect"):
    """Interfaces (r, Z) of SetupCylindricalGrid (src/SpatialGrid.jl:606-830): a uniform radial
    grid of N_r_lin cells up to rmax_lin, then N_r_log cells growing geometrically to rmax; in Z
    a uniform central region of N_Z_lin cells and length LZ_uniform with N_Z_log_side growing
    cells on each open side (above it for a reflecting bottom at Z = 0; above and below it,
    mirrored, for an outflowing bottom)."""
    if not (rmax > 0.0 and Zmax > 0.0 and LZ_uniform > 0.0 and rmax_lin > 0.0 and LZ_uniform <= Zmax):
        raise ValueError("SetupCylindricalGrid needs rmax, Zmax, LZ_uniform, rmax_lin > 0 and LZ_uniform <= Zmax")
    outflow = str(bc_z_bot).strip(":") == "Outflow"
    N_r = N_r_lin + N_r_log
    N_Z = N_Z_lin + (2 if outflow else 1) * N_Z_log_side
    if N_r < 3 or N_Z < 3:
        raise ValueError("the M1 stencil needs N_r >= 3 and N_Z >= 3")
    if outflow:
        zmin_lin, zmax_lin = 0.5 * (Zmax - LZ_uniform), 0.5 * (Zmax + LZ_uniform)
        Z_lin = julia_linrange(zmin_lin, zmax_lin, N_Z_lin + 1)
        dZ = Z_lin[1] - Z_lin[0]
        if N_Z_log_side >= 2:
            L_lower, L_upper = zmin_lin, Zmax - zmax_lin
            if not _isapprox(L_lower, L_upper, 1e-12):
                raise ValueError("the two logarithmic Z regions differ in length")
            up = _log_tail(zmax_lin, dZ, L_upper, N_Z_log_side)
            low = (zmin_lin - (up - zmax_lin))[::-1]
            Z = np.concatenate(([0.0], low, Z_lin, up, [Zmax]))
        else:
            Z = julia_linrange(0.0, Zmax, N_Z_lin + 1)
    else:
        Z_lin = julia_linrange(0.0, LZ_uniform, N_Z_lin + 1)
        dZ = Z_lin[1] - Z_lin[0]
        if N_Z_log_side >= 2:
            Z = np.concatenate((Z_lin, _log_tail(LZ_uniform, dZ, Zmax - LZ_uniform, N_Z_log_side), [Zmax]))
        else:
            Z = julia_linrange(0.0, Zmax, N_Z_lin + 1)
    r_lin = julia_linrange(0.0, rmax_lin, N_r_lin + 1)
    dr = r_lin[1] - r_lin[0]
    if N_r_log >= 2:
        r = np.concatenate((r_lin, _log_tail(rmax_lin, dr, rmax - rmax_lin, N_r_log), [rmax]))
    else:
        r = julia_linrange(0.0, rmax, N_r_lin + 1)
    if not (np.all(np.diff(r) > 0.0) and np.all(np.diff(Z) > 0.0)):
        raise ValueError("interfaces are not increasing")
    return r, Z


def log_stretched_cylindrical_geometry(rmax, rmax_lin, Zmax, LZ_uniform, N_r_lin, N_r_log, N_Z_lin, N_Z_log_side,
                                       bc_z_bot="Reflect"):
    """SetupCylindricalGrid (src/SpatialGrid.jl:606-915) with its logarithmic regions: the
    interfaces of log_stretched_interfaces and the geometry of cylindrical_geometry."""
    return cylindrical_geometry(*log_stretched_interfaces(rmax, rmax_lin, Zmax, LZ_uniform, N_r_lin, N_r_log,
                                                          N_Z_lin, N_Z_log_side, bc_z_bot))


@dataclass
class FreqGrid:
    nu: np.ndarray        # n_nu + 1 interfaces
    nuC: np.ndarray
    dnu: np.ndarray
    inv_dnu: np.ndarray
    inv_nuC: np.ndarray
    kcore_min: int        # 0-based inclusive
    kcore_max: int

    @property
    def n_nu(self):
        return self.nuC.size

    @property
    def dnu_c(self):
        return self.nuC - K.nu_lya


def _finish_freq_grid(nu):
    nu = np.ascontiguousarray(nu, dtype=np.float64)
    if not (np.all(nu > 0) and np.all(np.diff(nu) > 0)):
        raise ValueError("frequency interfaces must be positive and increasing")
    dnu = np.diff(nu)
    nuC = nu[:-1] + 0.5 * dnu
    dnuD3e4 = (K.compute_b(3e4) / K.c) * K.nu_lya
    ge = np.nonzero(nuC >= K.nu_lya - 4 * dnuD3e4)[0]
    le = np.nonzero(nuC <= K.nu_lya + 4 * dnuD3e4)[0]
    if ge.size == 0 or le.size == 0:
        raise ValueError("frequency grid has no bin centre inside the line core")
    return FreqGrid(nu=nu, nuC=nuC, dnu=dnu, inv_dnu=1.0 / dnu, inv_nuC=1.0 / nuC,
                    kcore_min=int(ge[0]), kcore_max=int(le[-1]))


def reference_frequency_grid(Tmin=30.0, q_fine=1.1, q_wing=None):
    """The default grid of GenerateLyaArrays, src/SetupLymanAlphaArrays.jl:40-135."""
    q_wing = q_fine if q_wing is None else q_wing
    x_fine_max_3e4 = 5.0
    x_max = 1e5
    dnu_min = (K.compute_b(Tmin) / K.c) * K.nu_lya
    x_max = min(x_max, 0.99 * K.nu_lya / dnu_min)
    x_max = min(x_max, (K.nu_lyc - K.nu_lya) / dnu_min)
    x_fine = x_fine_max_3e4 * K.compute_b(3e4) / K.compute_b(Tmin)
    x_pos = [0.0]
    dx = 1.0
    while x_pos[-1] < x_max:
        x = x_pos[-1]
        y = (x - x_fine) / (0.1 * x_fine)
        S = 0.0 if y < 0.0 else (1.0 if y > 1.0 else y)
        q = q_fine + (q_wing - q_fine) * S
        x_pos.append(x_pos[-1] + dx)
        dx *= q
    if x_pos[-1] > x_max:
        x_pos[-1] = x_max
    elif x_pos[-1] < x_max:
        x_pos.append(x_max)
    x_pos = np.array(x_pos)
    x_all = np.concatenate([-x_pos[1:][::-1], x_pos])
    return _finish_freq_grid(K.nu_lya + x_all * dnu_min)


def symmetric_frequency_grid(n_bins, x_max=600.0, T_ref=1e4, Tmin=30.0):
    """A grid of exactly n_bins (even) bins, symmetric about line centre, built with the
    reference's geometric scheme (first bin one Doppler width at Tmin, widths growing by a
    constant q) with q solved so that n_bins/2 bins per side reach |x| = x_max in units of
    the Doppler width at T_ref. Used for the 48/64/128-bin workloads, which the reference
    takes through GenerateLyaArrays_FromSaved."""
    if n_bins % 2 or n_bins < 4:
        raise ValueError("n_bins must be even and >= 4")
    n_side = n_bins // 2
    dnu_min = (K.compute_b(Tmin) / K.c) * K.nu_lya
    X = x_max * K.compute_dnuD(T_ref) / dnu_min

    def total(q):
        return n_side if q == 1.0 else (q ** n_side - 1.0) / (q - 1.0)

    if total(1.0) >= X:
        raise ValueError("x_max too small for this many bins")
    lo, hi = 1.0 + 1e-14, 2.0
    while total(hi) < X:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if total(mid) < X:
            lo = mid
        else:
            hi = mid
    q = 0.5 * (lo + hi)
    x_pos = [0.0]
    dx = 1.0
    for _ in range(n_side):
        x_pos.append(x_pos[-1] + dx)
        dx *= q
    x_pos[-1] = X
    x_pos = np.array(x_pos)
    x_all = np.concatenate([-x_pos[1:][::-1], x_pos])
    return _finish_freq_grid(K.nu_lya + x_all * dnu_min)


def alpha_floor(geom):
    """alpha_Lya_floor, src/SetupLymanAlphaArrays.jl:199."""
    return K.tau_alpha_floor * 1 / max(geom.r.max(), geom.Z.max())
