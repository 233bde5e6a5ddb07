"""Synthetic static-cloud workloads for the Lyman-alpha step.

The cloud set-up restates SetupStaticCloudTest (src/StaticCloudTest.jl:117-306): a uniform
cylindrical (r, Z) box of side 1.1 R_cl with R_cl = 1 pc, a uniform sphere of H I at
temperature T0 with line-centre optical depth tau0, gray continuum absorption tau_abs,
constant destruction probability, a Hubble-like outflow inside the cloud
(GetHubbleFlow, src/StaticCloudTest.jl:34-59), and either a uniform-sphere source of radius
rs*R_cl or (rs = 0) a point source in the axis cell at the cloud centre. The time step is
the CFL step of GetRHDCFLTimeStep (src/AdvectJandH.jl:29-68) with CFL = 0.4 and c~ = c.

Arrays use the reference's memory order: a Julia array A[k, i, j] (column-major) is the
numpy C-order array A[j, i, k]; a per-cell array A[i, j] is numpy A[j, i].

No public dataset is involved: every input is generated here from seeded parameters.
"""
from dataclasses import dataclass

import numpy as np

from . import constants as K
from .grid import FreqGrid, CylGeometry, symmetric_frequency_grid, uniform_cylindrical_geometry, alpha_floor

BC_REFLECT, BC_OUTFLOW = 0, 1
FLUX_GLF, FLUX_HLL = 0, 1


@dataclass
class StaticCloud:
    """All inputs of one static-cloud run (everything the step reads except H_voigt)."""
    name: str
    geom: CylGeometry
    freq: FreqGrid
    T: np.ndarray            # [j, i]
    alpha: np.ndarray        # line-centre opacity n_HI sigma0
    alpha_c: np.ndarray      # continuum absorption opacity (J)
    alpha_cF: np.ndarray     # continuum flux opacity added to alpha*H_voigt (0 for static clouds)
    pd: np.ndarray
    js: np.ndarray           # frequency-integrated emissivity
    u_r: np.ndarray          # cell-centred velocities (for the CFL step)
    u_Z: np.ndarray
    u_r_star: np.ndarray     # [j, f] f = 0..nr
    u_Z_star: np.ndarray     # [f, i] f = 0..nz
    dur_dr: np.ndarray
    dur_dZ: np.ndarray
    duZ_dr: np.ndarray
    duZ_dZ: np.ndarray
    ur_over_r: np.ndarray
    c_tilde: float
    dt: float
    z_center: float
    bc_r_right: int
    bc_z_bot: int
    bc_z_top: int
    recoil: bool
    flux_method: int
    alpha_floor: float
    tau0: float
    L_source: float
    n_H: np.ndarray = None       # hydrogen density behind alpha (x_HI = 1), when the cloud is built from one
    kappa_d: float = 0.0         # gray dust opacity per gram of dust behind alpha_c = kappa_d * 0.01 n_H m_H
    species: dict = None         # n_HII, n_e, n_HI, n_HeI, n_H2 per cell: pd is then computed on the device
    bc_r_left: int = BC_REFLECT  # first r (X) interface: the axis (cylindrical) or either rule (Cartesian)

    @property
    def n_nu(self):
        return self.freq.n_nu

    @property
    def nr(self):
        return self.geom.nr

    @property
    def nz(self):
        return self.geom.nz

    @property
    def cell_bins(self):
        return self.n_nu * self.nr * self.nz


def hubble_flow(r, Z, umax, Rcl, Zc):
    """GetHubbleFlow, src/StaticCloudTest.jl:34-59 (vectorised)."""
    R = np.hypot(r, Z - Zc)
    inside = R <= Rcl
    H = umax / Rcl
    u_r = np.where(inside, H * r, 0.0)
    u_Z = np.where(inside, H * (Z - Zc), 0.0)
    g = np.where(inside, H, 0.0)
    return u_r, u_Z, g


def cfl_dt(geom, c_tilde, u_r, u_Z, cfl):
    """GetRHDCFLTimeStep, src/AdvectJandH.jl:29-68."""
    dr = geom.r[1:] - geom.r[:-1]
    dZ = geom.Z[1:] - geom.Z[:-1]
    u = np.hypot(u_r, u_Z)
    dt = 0.5 * np.minimum(dr[None, :], dZ[:, None]) / (c_tilde + u)
    return cfl * float(dt.min())


def static_cloud(nr, nz, n_nu, tau0, T0=1e4, tau_abs=0.0, pd0=0.0, rs=0.0, umax_kms=0.0,
                 recoil=True, bc_z_bot=BC_REFLECT, flux_method=FLUX_GLF, freq=None, name="cloud",
                 cfl=0.4, x_max=600.0, geom=None):
    """Fields of SetupStaticCloudTest (src/StaticCloudTest.jl:117-306), no cone; on a uniform
    grid of nr x nz cells over 1.1 R_cl, or on `geom` (whose sizes then replace nr, nz)."""
    L = 1e5 * K.Lsun
    Rcl = K.pc
    Rmax = 1.1 * Rcl if geom is None else float(geom.r[-1])
    Zmax = 1.1 * Rcl if geom is None else float(geom.Z[-1])
    Zc = 0.0 if bc_z_bot == BC_REFLECT else 0.5 * Zmax
    c_tilde = K.c
    if geom is None:
        geom = uniform_cylindrical_geometry(Rmax, Zmax, nr, nz)
    nr, nz = geom.r.size - 1, geom.Z.size - 1
    if freq is None:
        freq = symmetric_frequency_grid(n_nu, x_max=x_max, T_ref=T0)
    rC, ZC = np.meshgrid(geom.rCoM, geom.ZCoM)            # [j, i]
    T = np.full((nz, nr), float(T0))
    Rs = rs * Rcl
    dL = Rcl
    sigma0 = K.compute_sigma0(T0)
    nHI0 = tau0 / (sigma0 * dL)
    ac0 = tau_abs / Rcl
    RCoM = np.sqrt(rC ** 2 + (ZC - Zc) ** 2)
    inside_cloud = RCoM < Rcl
    inside_source = RCoM < Rs
    alpha = np.where(inside_cloud, nHI0 * sigma0, 0.0)
    alpha_c = np.where(inside_cloud, ac0, 0.0)
    pd = np.where(inside_cloud, pd0, 0.0)
    js = np.where(inside_cloud & inside_source, 3 * L / ((4 * np.pi) * (4 * np.pi) * (Rs * Rs * Rs)) if Rs > 0 else 0.0, 0.0)
    umax = umax_kms * K.kms
    u_r, u_Z, g = hubble_flow(rC, ZC, umax, Rcl, Zc)
    rf, Zrow = np.meshgrid(geom.r, geom.ZCoM)             # [j, f]
    u_r_star, _, _ = hubble_flow(rf, Zrow, umax, Rcl, Zc)
    rcol, Zf = np.meshgrid(geom.rCoM, geom.Z)             # [f, i]
    _, u_Z_star, _ = hubble_flow(rcol, Zf, umax, Rcl, Zc)
    if js.max() <= 0.0:
        i0 = int(np.argmin(np.abs(geom.rCoM - 0.0)))
        j0 = int(np.argmin(np.abs(geom.ZCoM - Zc)))
        js[j0, i0] = L / (4 * np.pi * geom.dV[j0, i0])
    zeros = np.zeros((nz, nr))
    dt = cfl_dt(geom, c_tilde, u_r, u_Z, cfl)
    return StaticCloud(name=name, geom=geom, freq=freq, T=T, alpha=alpha, alpha_c=alpha_c,
                       alpha_cF=zeros.copy(), pd=pd, js=js, u_r=u_r, u_Z=u_Z,
                       u_r_star=np.ascontiguousarray(u_r_star), u_Z_star=np.ascontiguousarray(u_Z_star),
                       dur_dr=g.copy(), dur_dZ=zeros.copy(), duZ_dr=zeros.copy(), duZ_dZ=g.copy(),
                       ur_over_r=g.copy(), c_tilde=c_tilde, dt=dt, z_center=Zc,
                       bc_r_right=BC_OUTFLOW, bc_z_bot=bc_z_bot, bc_z_top=BC_OUTFLOW,
                       recoil=bool(recoil), flux_method=flux_method, alpha_floor=alpha_floor(geom),
                       tau0=tau0, L_source=L)


def config_c1(scale=1):
    """Plain FP64, 64x64 cells x 64 bins, tau0 = 1e6, T = 1e4 K, no dust, static, point source."""
    n = 64 // scale
    return static_cloud(n, n, 64 if scale == 1 else max(8, 64 // scale), tau0=1e6, T0=1e4, rs=0.0,
                        name="c1_static_point_64x64x64")


def config_c2(scale=1):
    """256x256 cells x 64 bins, tau0 = 1e8, T = 1e4 K, gray dust tau_abs = 1, uniform source of
    radius 0.5 R_cl, Hubble outflow with v_max = 200 km/s."""
    n = 256 // scale
    return static_cloud(n, n, 64 if scale == 1 else max(8, 64 // scale), tau0=1e8, T0=1e4, tau_abs=1.0,
                        rs=0.5, umax_kms=200.0, name="c2_dusty_outflow_256x256x64")


C3_SIDES = (32, 48, 64, 96, 128, 192, 256)


def batch_clouds(n_clouds=512, n_nu=48, sides=C3_SIDES, seed=20261203, tau0_range=(1e4, 1e8),
                 T_range=(1e2, 1e4), tau_abs_range=(0.0, 2.0), vmax_range=(0.0, 100.0), rs=0.5, x_max=600.0):
    """The ragged batch of independent static clouds: per cloud, drawn from
    numpy.random.default_rng(seed) in this order, the radial side and the vertical side
    (independently, uniform over `sides`), log-uniform tau0, log-uniform T, uniform tau_abs,
    uniform v_max. Every cloud has a uniform source of radius rs*R_cl, a reflecting bottom
    boundary and its own CFL time step; all share one symmetric frequency grid of n_nu bins
    reaching |x| = x_max Doppler widths at 1e4 K (a context holds one frequency grid)."""
    rng = np.random.default_rng(seed)
    fq = symmetric_frequency_grid(n_nu, x_max=x_max, T_ref=1e4)
    out = []
    for q in range(n_clouds):
        nr = int(rng.choice(sides))
        nz = int(rng.choice(sides))
        tau0 = float(np.exp(rng.uniform(np.log(tau0_range[0]), np.log(tau0_range[1]))))
        T0 = float(np.exp(rng.uniform(np.log(T_range[0]), np.log(T_range[1]))))
        tau_abs = float(rng.uniform(*tau_abs_range))
        vmax = float(rng.uniform(*vmax_range))
        out.append(static_cloud(nr, nz, n_nu, tau0=tau0, T0=T0, tau_abs=tau_abs, rs=rs, umax_kms=vmax, freq=fq,
                                name=f"batch{q}"))
    return out


def config_c3(n_clouds=512, seed=20261203):
    """512 ragged static clouds x 48 bins, sides from {32, ..., 256} drawn independently in r and Z."""
    return batch_clouds(n_clouds=n_clouds, seed=seed)


def gaussian_random_field(nr, nz, slope=-11.0 / 3.0, seed=20261207):
    """Unit-variance Gaussian random field on an (n_z, n_r) grid with isotropic 2-D power
    spectrum P(k) ~ k^slope, made by filtering seeded white noise in Fourier space."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((nz, nr))
    kz = np.fft.fftfreq(nz)[:, None]
    kr = np.fft.rfftfreq(nr)[None, :]
    k = np.hypot(kz, kr)
    amp = np.zeros_like(k)
    amp[k > 0] = k[k > 0] ** (0.5 * slope)
    g = np.fft.irfft2(np.fft.rfft2(white) * amp, s=(nz, nr))
    g -= g.mean()
    return g / g.std()


def turbulent_cloud(nr=128, nz=128, n_nu=48, n_mean=100.0, sigma_ln=1.0, T0=1e4, vmax_kms=50.0,
                    dust_to_gas=0.01, tau_abs_mean=1.0, rs=0.5, seed=20261207, x_max=600.0, name="turbulent"):
    """A static cloud with a lognormal turbulent density n_H = n_mean exp(sigma g - sigma^2/2)
    (g a unit-variance Gaussian random field with P(k) ~ k^-11/3) inside R_cl, x_HI = 1 so
    alpha = n_H sigma0(T), gray dust alpha_c = kappa_d dust_to_gas n_H m_H with kappa_d fixed so
    that the mean density gives a dust optical depth tau_abs_mean across R_cl, a Hubble-like
    radial outflow of v_max, and the uniform source of radius rs R_cl. The reference builds no
    such field (its turbulence module perturbs velocities only); this generator is the
    project's own."""
    base = static_cloud(nr, nz, n_nu, tau0=1.0, T0=T0, rs=rs, umax_kms=vmax_kms, x_max=x_max, name=name)
    g = gaussian_random_field(nr, nz, seed=seed)
    nH = n_mean * np.exp(sigma_ln * g - 0.5 * sigma_ln ** 2)
    inside = base.alpha > 0.0
    kappa = tau_abs_mean / (dust_to_gas * n_mean * K.mH * K.pc)
    sigma0 = K.compute_sigma0(T0)
    base.alpha = np.where(inside, nH * sigma0, 0.0)
    base.alpha_c = np.where(inside, kappa * dust_to_gas * nH * K.mH, 0.0)
    base.n_H = np.where(inside, nH, 0.0)
    base.kappa_d = kappa
    base.tau0 = float(n_mean * sigma0 * K.pc)
    return base


def config_c4(scale=1):
    """The adjoint configuration: 128 x 128 cells x 48 bins, lognormal turbulent n_H (sigma_ln = 1,
    mean 100 cm^-3), T = 1e4 K, gray dust at 0.01 n_H, radial outflow v_max = 50 km/s."""
    n = 128 // scale
    return turbulent_cloud(nr=n, nz=n, n_nu=48 if scale == 1 else max(8, 48 // scale), name="c4_turbulent_128x128x48")


def radial_flow(r, Z, Zc, v_of_R, dv_of_R):
    """u = v(R) R_hat about (0, Zc) and its gradient in (r, Z): u_i = v x_i / R gives
    du_i/dx_j = (v/R) delta_ij + (v' - v/R) x_i x_j / R^2, and u_r / r = v / R."""
    dz = Z - Zc
    R = np.hypot(r, dz)
    Rs = np.where(R > 0, R, 1.0)
    v = v_of_R(R)
    dv = dv_of_R(R)
    q = np.where(R > 0, v / Rs, dv)                 # v/R -> v'(0) at the centre
    s = np.where(R > 0, (dv - q) / (Rs * Rs), 0.0)
    return dict(u_r=q * r, u_Z=q * dz, dur_dr=q + s * r * r, dur_dZ=s * r * dz, duZ_dr=s * r * dz,
                duZ_dZ=q + s * dz * dz, ur_over_r=q)


def rhd_snapshot_cloud(n=1024, n_nu=128, sigma_ln=1.5, n_mean=100.0, bubble=0.2, x_HI_bubble=1e-4, T_in=1e4,
                       T_out=100.0, v_shell_kms=30.0, shell_width=0.05, dust_to_gas=0.01, tau_abs_mean=1.0,
                       seed=20261208, x_max=600.0, name="rhd_snapshot"):
    """One synthetic RHD snapshot on an n x n (r, Z) grid, frequency bins to |x| = x_max at 1e4 K:
    a lognormal turbulent n_H (sigma_ln) with P(k) ~ k^-11/3; a photoionised bubble of radius
    `bubble` R_cl (x_HI = 1e-4, T = 1e4 K, n_HII = n_e = (1 - x_HI) n_H, p_d from pd_Lya) with a
    uniform Lyman-alpha source inside it; neutral gas at T_out outside; a radial shell velocity
    v(R) = v_shell exp(-(R - R_b)^2 / (2 w^2)) about the bubble edge (w = shell_width R_cl);
    gray dust at dust_to_gas n_H (kappa_d as in turbulent_cloud). The reference has no such
    snapshot generator; this one is the project's own."""
    base = static_cloud(n, n, n_nu, tau0=1.0, T0=1e4, rs=bubble, umax_kms=0.0, x_max=x_max, name=name)
    g = base.geom
    rC, ZC = np.meshgrid(g.rCoM, g.ZCoM)
    Zc, Rcl = base.z_center, K.pc
    R = np.hypot(rC, ZC - Zc)
    inside = R < Rcl
    nH = n_mean * np.exp(sigma_ln * gaussian_random_field(n, n, seed=seed) - 0.5 * sigma_ln ** 2)
    nH = np.where(inside, nH, 0.0)
    ion = R < bubble * Rcl
    x_HI = np.where(ion, x_HI_bubble, 1.0)
    T = np.where(ion, T_in, T_out)
    nHI = x_HI * nH
    nHII = (1.0 - x_HI) * nH
    sigma0 = K.sigma0_prefact / (K.b_prefact * np.sqrt(T))
    kappa = tau_abs_mean / (dust_to_gas * n_mean * K.mH * K.pc)
    base.T = T
    base.alpha = nHI * sigma0
    base.alpha_c = kappa * dust_to_gas * nH * K.mH
    base.n_H = nH
    base.kappa_d = kappa
    base.species = dict(nHII=nHII, ne=nHII.copy(), nHI=nHI, nHeI=np.zeros_like(nH), nH2=np.zeros_like(nH))
    Rb, w, vs = bubble * Rcl, shell_width * Rcl, v_shell_kms * K.kms
    v_of = lambda x: vs * np.exp(-0.5 * ((x - Rb) / w) ** 2)
    dv_of = lambda x: -vs * (x - Rb) / (w * w) * np.exp(-0.5 * ((x - Rb) / w) ** 2)
    fl = radial_flow(rC, ZC, Zc, v_of, dv_of)
    for k in ("dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ", "ur_over_r"):
        setattr(base, k, fl[k])
    base.u_r, base.u_Z = fl["u_r"], fl["u_Z"]
    rf, Zrow = np.meshgrid(g.r, g.ZCoM)
    base.u_r_star = np.ascontiguousarray(radial_flow(rf, Zrow, Zc, v_of, dv_of)["u_r"])
    rcol, Zf = np.meshgrid(g.rCoM, g.Z)
    base.u_Z_star = np.ascontiguousarray(radial_flow(rcol, Zf, Zc, v_of, dv_of)["u_Z"])
    base.dt = cfl_dt(g, base.c_tilde, base.u_r, base.u_Z, 0.4)
    base.tau0 = float(n_mean * K.compute_sigma0(T_out) * K.pc)
    return base


def config_c5(scale=1):
    """The largest field: 1024 x 1024 cells x 128 bins of one synthetic RHD snapshot."""
    n = 1024 // scale
    return rhd_snapshot_cloud(n=n, n_nu=128 if scale == 1 else max(16, 128 // scale),
                              name="c5_rhd_snapshot_1024x1024x128")


def small_cloud(nr=12, nz=10, n_nu=16, **kw):
    """A cheap cloud for parity tests (the oracle finishes it in milliseconds)."""
    kw.setdefault("tau0", 1e5)
    kw.setdefault("rs", 0.5)
    kw.setdefault("umax_kms", 150.0)
    kw.setdefault("tau_abs", 0.5)
    kw.setdefault("x_max", 60.0)
    return static_cloud(nr, nz, n_nu, name="small", **kw)


# ---- gas and dust state for the RHD-side Lyman-alpha block ----------------------------------
DUST_KAPPA_ABS = (3.0e4, 5.0e4, 8.0e4)    # Lya absorption opacity per dust mass, Sil / C / PAH (cm^2 g^-1)
DUST_KAPPA_F = (6.0e4, 9.0e4, 1.2e5)      # Lya flux opacity per dust mass
DUST_RHO_IGNORE = 1.1e-13 * K.mH          # 1.1 rho_d_floor with rho_d_floor = 1e-13 m_H (src/Hydrodynamics.jl:53-54)


def rhd_gas_state(cloud, seed):
    """A seeded per-cell gas and dust state for lyd_rhd_lya_prepare: T log-uniform over 30 K ..
    4e4 K (both edges of the recombination tables and their interior), n_H log-uniform over
    0.1 .. 1e3 cm^-3, ionised fraction 1e-4 .. 1, molecular, He, OH and CH fractions, and dust
    at 1e-4 .. 1e-2 of the gas mass in three kinds, a fifth of the silicate below the ignore
    level. The dust opacities are this project's choice. Returns (species dict, rho_d (3, n_z, n_r))."""
    rng = np.random.default_rng(seed)
    shape = (cloud.nz, cloud.nr)
    lg = lambda lo, hi: 10.0 ** rng.uniform(lo, hi, size=shape)
    T = lg(1.5, 4.6)
    nH = lg(-1.0, 3.0)
    xHII = lg(-4.0, 0.0)
    sp = {"T": T, "nHI": nH * (1.0 - xHII), "nHII": nH * xHII, "ne": nH * xHII * 1.1,
          "nH2": nH * lg(-6.0, -1.0), "nHeI": 0.08 * nH, "nOHx": nH * lg(-9.0, -6.0), "nCHx": nH * lg(-9.0, -6.0)}
    rho = 0.01 * nH * K.mH * lg(-2.0, 0.0)
    rho_d = np.stack([rho, 0.5 * rho, 0.05 * rho])
    rho_d[0][rng.uniform(size=shape) < 0.2] = 0.5 * DUST_RHO_IGNORE
    return sp, rho_d


def cartesian_cloud(nx=12, ny=10, n_nu=16, bc_left=BC_OUTFLOW, seed=3, **kw):
    """A small cloud on a Cartesian (X, Y) grid: the fields of small_cloud moved onto a uniform
    Cartesian grid over the same extent, with seeded velocity gradients, no u_r / r term, and the
    chosen boundary at the first X interface. For parity tests of the Cartesian advection."""
    from .grid import cartesian_geometry, julia_linrange
    cl = small_cloud(nr=nx, nz=ny, n_nu=n_nu, **kw)
    g = cl.geom
    geom = cartesian_geometry(julia_linrange(-g.r[-1], g.r[-1], nx + 1), julia_linrange(0.0, g.Z[-1], ny + 1))
    rng = np.random.default_rng(seed)
    shape = (ny, nx)
    scale = 1e5 / K.pc
    cl.geom = geom
    cl.bc_r_left = bc_left
    cl.ur_over_r = np.zeros(shape)
    for name in ("dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ"):
        setattr(cl, name, scale * rng.normal(size=shape))
    cl.u_r_star = 1e6 * rng.normal(size=(ny, nx + 1))
    cl.u_Z_star = 1e6 * rng.normal(size=(ny + 1, nx))
    cl.name = "cartesian"
    return cl
