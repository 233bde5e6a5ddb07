"""Physical and numerical constants of the Lyman-alpha M1 path.

Values restate src/ConstantsAndFunctions.jl:46-170 (physical constants and units),
src/M1Closure.jl:36-41 (closure floors), src/FreqFactors.jl:16-18 (Peclet limits),
src/UpdateLyaJandH.jl:43 (active-bin threshold) and src/SetupLymanAlphaArrays.jl:12
(opacity-floor optical depth). The CUDA sources hold the same numbers in
lydion_b200/csrc/lyd_physics.cuh.
"""
import math

# units
Lsun = 3.839e33
pc = 3.085677581467192e18
kms = 1e5
yr = 365.24 * 86400.0

# physical constants (cgs)
c = 2.99792458e10
h = 6.626069573e-27
kB = 1.380648813e-16
mu = 1.660539069e-24
mH = 1.0080 * mu
mD = 2.014 * mu
# pristine-gas mass fractions, src/ConstantsAndFunctions.jl:124-127
Y_He = 0.247
D_H_ratio = 2.53e-5
X_D = D_H_ratio * (1 - Y_He) * mD / mH
X_H = 1 - Y_He - X_D
me = 9.109382917e-28
e = 4.80320451e-10
nu_lya = 2.466068e15
nu_lyc = 3.289842e15
A_lya = 6.265e8
f_lu_lya = 0.41641

four_pi = 4 * math.pi
inv_c = 1 / c

# M1 closure floors
fmin = 1e-10
fmax = 1.0 - 1e-10
Jeps = 1e-60
Heps = 1e-100

# frequency leakage coefficients
Pmin = 1e-3
Pmax = 40.0

eps_active = 1e-10
tau_alpha_floor = 1e-5

b_prefact = math.sqrt(2 * kB / mH)
a_prefact = A_lya / (four_pi * nu_lya * 1 / c)
sigma0_prefact = math.sqrt(math.pi) * (e * e) * f_lu_lya / (me * nu_lya)


def compute_b(T):
    """Thermal velocity b(T), src/ConstantsAndFunctions.jl:286-288."""
    return b_prefact * math.sqrt(T)


def compute_dnuD(T):
    """Doppler width, src/ConstantsAndFunctions.jl:294-296."""
    return compute_b(T) * (nu_lya / c)


def compute_a(T):
    """Voigt parameter, src/ConstantsAndFunctions.jl:303-305."""
    return a_prefact / compute_b(T)


def compute_sigma0(T):
    """Line-centre cross-section, src/ConstantsAndFunctions.jl:312-314."""
    return sigma0_prefact / compute_b(T)
