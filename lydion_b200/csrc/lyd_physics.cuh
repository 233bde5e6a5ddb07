// lyd_physics.cuh -- device arithmetic of the Lyman-alpha M1 step, templated on the
// arithmetic type R (double for the FP64 step, float for the bulk of the mixed step).
//
// Each function restates one piece of the LYDION reference (paths inside its source tree):
// the M1 closure (src/M1Closure.jl), PLM reconstruction and the GLF/HLL fluxes
// (src/AdvectJandH.jl), and the exponentially fitted frequency leakage coefficients
// (src/FreqFactors.jl). Thresholds that depend on the storage scale of J (the floors
// Jeps, Heps^2) are passed in at run time.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace lyd {

// ---- constants (src/ConstantsAndFunctions.jl:46-170) -------------------------------------
constexpr double kC = 2.99792458e10;
constexpr double kInvC = 1.0 / kC;
constexpr double kPi = 3.14159265358979323846;
constexpr double kFourPi = 4.0 * kPi;
constexpr double kFourPiOverC = kFourPi / kC;
constexpr double kHPlanck = 6.626069573e-27;
constexpr double kKBoltz = 1.380648813e-16;
constexpr double kHOverKB = kHPlanck / kKBoltz;
constexpr double kNuLya = 2.466068e15;
constexpr double kMH = 1.0080 * 1.660539069e-24;
constexpr double kALya = 6.265e8;
constexpr double kA2g = 8.2206;
constexpr double kA2p2s = 8.78e-7;
constexpr double kA2s2p = 1.597e-9;
// src/M1Closure.jl:36-41
constexpr double kFmin = 1e-10;
constexpr double kFmax = 1.0 - 1e-10;
constexpr double kJeps = 1e-60;
constexpr double kHeps = 1e-100;
// src/FreqFactors.jl:16-18
constexpr double kPmin = 1e-3;
constexpr double kPmax = 40.0;
// src/UpdateLyaJandH.jl:43
constexpr double kEpsActive = 1e-10;

template <typename R> struct Num;
template <> struct Num<double> {
    static __device__ __forceinline__ double third() { return 1.0 / 3.0; }
    static __device__ __forceinline__ double fmin() { return kFmin; }
    static __device__ __forceinline__ double fmax() { return kFmax; }
    static __device__ __forceinline__ double tiny() { return 1e-300; }
};
template <> struct Num<float> {
    static __device__ __forceinline__ float third() { return 1.0f / 3.0f; }
    static __device__ __forceinline__ float fmin() { return 1e-10f; }
    static __device__ __forceinline__ float fmax() { return 1.0f - 1e-7f; }
    static __device__ __forceinline__ float tiny() { return 1e-37f; }
};

// Square root. FP64: the IEEE square root. FP32: the hardware's approximate square root alone
// (PTX sqrt.approx.ftz.f32, relative error within 2^-23 over the normal range); the IEEE-rounded
// FP32 root costs a refinement sequence with special-case branches on the transcendental unit,
// which the FP32 advection keeps 40 % busy (mixed advection at 256^2 x 64, 32 rows per tile:
// 0.225 -> 0.207 ms; after 2000 steps the mixed form's M_F, edge spectrum and J differ from
// FP64 by 6.1e-7, 2.6e-7 and 1.5e-6 against 5.9e-7, 2.6e-7 and 1.7e-6 with the IEEE root).
// A subnormal argument is flushed, so its root is 0: the callers that divide by a root treat
// a zero root as a zero vector (the non-flushing form, sqrt.approx.f32, costs more than the
// IEEE root here).
__device__ __forceinline__ double rsq(double x) { return sqrt(x); }
__device__ __forceinline__ float rsq(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Reciprocal 1 / y. FP64: the hardware's approximate reciprocal (PTX rcp.approx.ftz.f64)
// refined by one third-order step of the Newton-Raphson family for 1/y: with e = 1 - y x,
// 1/y = x / (1 - e) = x (1 + e + e^2 + ...), so x <- x + x (e + e^2) cubes the relative error
// (Markstein, IBM J. Res. Dev. 34 (1990) 111-119), in three fused multiply-adds where two
// quadratic steps take four. No special-case branches: the callers divide by positive normal
// numbers whose reciprocals are normal. FP32: the hardware's approximate reciprocal alone (PTX
// rcp.approx.ftz.f32, relative error within 2^-23 over the normal range, subnormals flushed),
// one instruction in place of the IEEE division's refinement sequence; the FP32 arithmetic of
// the mixed and FP32-storage forms already carries a 2^-24 rounding per operation.
template <typename R> __device__ __forceinline__ R rcp(R y);
template <> __device__ __forceinline__ double rcp<double>(double y) {
    double x;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(y));
    const double e = fma(-y, x, 1.0);
    return fma(x, fma(e, e, e), x);
}
template <> __device__ __forceinline__ float rcp<float>(float y) {
    float x;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(x) : "f"(y));
    return x;
}

// Reciprocal square root 1 / sqrt(x) for FP64 arithmetic and x >= DBL_MIN: the hardware's
// approximate reciprocal square root (PTX rsqrt.approx.ftz.f64) refined by one third-order
// step: with e = 1 - x y^2, 1/sqrt(x) = y (1 - e)^(-1/2) = y (1 + e/2 + 3 e^2/8 + ...), so
// y <- y + y e (1/2 + 3 e / 8) cubes the relative error (Markstein, IBM J. Res. Dev. 34 (1990)
// 111-119), in two multiplies and three fused multiply-adds where two quadratic steps take
// seven operations. x * rsqrt_nr(x) is then sqrt(x) to about an ulp, and one such root gives both a
// length and its reciprocal where the IEEE root needs a root and a reciprocal.
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-(x * y), y, 1.0);
    return fma(y, e * fma(e, 0.375, 0.5), y);
}
constexpr double kDblMinNormal = 2.2250738585072014e-308;

// Reciprocal square root 1 / sqrt(x) for FP32 arithmetic: the hardware's approximation alone
// (PTX rsqrt.approx.ftz.f32, relative error within 2^-22.9 over the normal range; a subnormal
// or zero argument gives +inf, so callers check x against FLT_MIN first). One transcendental
// operation gives both a length, x * rsqf(x), and its reciprocal.
__device__ __forceinline__ float rsqf(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kFltMinNormal = 1.17549435e-38f;

// MinMod, src/ConstantsAndFunctions.jl:1571-1582
template <typename R>
__device__ __forceinline__ R minmod(R a, R b) {
    return (a * b <= R(0)) ? R(0) : (fabs(a) < fabs(b) ? a : b);
}

// Levermore closure chi(f), src/M1Closure.jl:28-33, evaluated as (5 - 2 sqrt(4 - 3 f^2)) / 3,
// the same function (multiply numerator and denominator by 5 - 2 sqrt(4 - 3 f^2): the
// denominator becomes 3 (3 + 4 f^2)), with one square root and no reciprocal; 5 - 2 sqrt(..)
// >= 1 for f <= 1, so at most a factor 4 cancels (f = 0: 5 - 4). In FP64 the root of
// t = 4 - 3 f^2, in [1, 4], is t * rsqrt_nr(t), folded into 5 - 2 s by one fused multiply-add.
template <typename R>
__device__ __forceinline__ R chi_L84(R f) {
    R f2 = f * f;
    R t = R(4) - R(3) * f2;
    if constexpr (sizeof(R) == 4)
        return (R(5) - R(2) * rsq(t)) * R(1.0f / 3.0f);
    else
        return fma(-2.0 * t, rsqrt_nr(t), 5.0) * (1.0 / 3.0);
}

// Compute_D_Edd_from_f_n, src/M1Closure.jl:91-119
template <typename R>
__device__ __forceinline__ void D_from_f_n(R f, R nr, R nZ, R &Drr, R &DZZ, R &DrZ) {
    if (f > Num<R>::fmin()) {
        f = f < Num<R>::fmax() ? f : Num<R>::fmax();
        R chi = chi_L84(f);
        R a = (R(1) - chi) * R(0.5);
        R b = (R(3) * chi - R(1)) * R(0.5);
        R b_nr = b * nr;
        Drr = a + b_nr * nr;
        DZZ = a + b * nZ * nZ;
        DrZ = b_nr * nZ;
    } else {
        Drr = Num<R>::third(); DZZ = Num<R>::third(); DrZ = R(0);
    }
}

// Compute_D_Edd, src/M1Closure.jl:46-83. jeps / heps2 are the floors in storage units.
template <typename R>
__device__ __forceinline__ void D_edd(R Hr, R HZ, R J, R jeps, R heps2, R &Drr, R &DZZ, R &DrZ) {
    R H2 = Hr * Hr + HZ * HZ;
    const R fmin2 = Num<R>::fmin() * Num<R>::fmin();
    if (J <= jeps || H2 <= heps2 || H2 <= fmin2 * J * J) {
        Drr = Num<R>::third(); DZZ = Num<R>::third(); DrZ = R(0);
        return;
    }
    R Hmag, inv_H;
    // one reciprocal square root gives |H| and 1/|H|; |H|^2 below the type's normal range
    // counts as no direction
    if constexpr (sizeof(R) == 4) {
        if (!(H2 >= kFltMinNormal)) {
            Drr = Num<R>::third(); DZZ = Num<R>::third(); DrZ = R(0);
            return;
        }
        inv_H = rsqf(H2);
    } else {
        if (!(H2 >= kDblMinNormal)) {
            Drr = Num<R>::third(); DZZ = Num<R>::third(); DrZ = R(0);
            return;
        }
        inv_H = rsqrt_nr(H2);
    }
    Hmag = H2 * inv_H;
    R f = Hmag * rcp<R>(J);
    f = f < Num<R>::fmin() ? Num<R>::fmin() : (f > Num<R>::fmax() ? Num<R>::fmax() : f);
    R chi = chi_L84(f);
    R a = (R(1) - chi) * R(0.5);
    R b = (R(3) * chi - R(1)) * R(0.5);
    R nr = Hr * inv_H, nZ = HZ * inv_H;
    R b_nr = b * nr;
    Drr = a + b_nr * nr;
    DZZ = a + b * nZ * nZ;
    DrZ = b_nr * nZ;
}

// HLL_Eigenvalues, src/M1Closure.jl:273-296
template <typename R>
__device__ __forceinline__ void hll_eigen(R f, R mu, R &l1, R &l3) {
    f = f < Num<R>::fmin() ? Num<R>::fmin() : (f > Num<R>::fmax() ? Num<R>::fmax() : f);
    mu = mu < R(-1) ? R(-1) : (mu > R(1) ? R(1) : mu);
    R f2 = f * f, mu2 = mu * mu, muf = mu * f;
    R t = R(4) - R(3) * f2;
    // t >= 1 (f <= fmax < 1): one reciprocal square root gives the root and its reciprocal
    R inv_sq;
    if constexpr (sizeof(R) == 4) inv_sq = rsqf(t);
    else inv_sq = rsqrt_nr(t);
    const R sq = t * inv_sq;
    R g = R(2) / R(3) * (R(4) - R(3) * f2 - sq) + R(2) * mu2 * (R(2) - f2 - sq);
    R fac = rsq(g > R(0) ? g : R(0));
    R x1 = (muf - fac) * inv_sq, x3 = (muf + fac) * inv_sq;
    l1 = x1 < R(-1) ? R(-1) : (x1 > R(1) ? R(1) : x1);
    l3 = x3 < R(-1) ? R(-1) : (x3 > R(1) ? R(1) : x3);
}

// One cell of the reconstruction stencil.
template <typename R> struct Cell { R J, Hr, HZ; };

// ReconstructInterface output, src/AdvectJandH.jl:359-473
template <typename R> struct Recon {
    R J_L, J_R, Hr_L, Hr_R, HZ_L, HZ_R, tau_L, tau_R, f_L, f_R, nr_L, nr_R, nZ_L, nZ_R;
};

// A stencil cell in the form ReconstructInterface works on: J and the reduced flux
// f = H / max(J, Jeps) (src/AdvectJandH.jl:373-386). Computing it once per cell lets every
// face that uses the cell share one reciprocal.
template <typename R> struct CellF { R J, fr, fZ; };

template <typename R>
__device__ __forceinline__ CellF<R> cell_f(R J, R Hr, R HZ, R jeps) {
    R iJ = rcp<R>(J > jeps ? J : jeps);
    CellF<R> c;
    c.J = J; c.fr = Hr * iJ; c.fZ = HZ * iJ;
    return c;
}

// ReconstructInterface, src/AdvectJandH.jl:359-473, on prepared cells im1, i, ip1, ip2
// around the interface between i and ip1; iv = {dL, dR, inv_i_im1, inv_ip1_i, inv_ip2_ip1}.
template <typename R>
__device__ __forceinline__ Recon<R> reconstruct_f(const CellF<R> &cm1, const CellF<R> &ci, const CellF<R> &cp1,
                                                  const CellF<R> &cp2, const R iv[5], R aF_i, R aF_ip1, R jeps) {
    Recon<R> o;
    const R dL = iv[0], dR = iv[1];
    o.tau_L = aF_i * dL;
    o.tau_R = aF_ip1 * dR;
    R dJc = (cp1.J - ci.J) * iv[3];
    R dJL = minmod((ci.J - cm1.J) * iv[2], dJc);
    R dJR = minmod((cp2.J - cp1.J) * iv[4], dJc);
    R dfrc = (cp1.fr - ci.fr) * iv[3];
    R dfrL = minmod((ci.fr - cm1.fr) * iv[2], dfrc);
    R dfrR = minmod((cp2.fr - cp1.fr) * iv[4], dfrc);
    R dfZc = (cp1.fZ - ci.fZ) * iv[3];
    R dfZL = minmod((ci.fZ - cm1.fZ) * iv[2], dfZc);
    R dfZR = minmod((cp2.fZ - cp1.fZ) * iv[4], dfZc);

    R JL = ci.J + dJL * dL;
    R JR = cp1.J - dJR * dR;
    o.J_L = JL > jeps ? JL : jeps;
    o.J_R = JR > jeps ? JR : jeps;
    R frL = ci.fr + dfrL * dL, frR = cp1.fr - dfrR * dR;
    R fZL = ci.fZ + dfZL * dL, fZR = cp1.fZ - dfZR * dR;

    // one reciprocal square root gives |f| and 1/|f|; |f|^2 below the type's normal range
    // counts as no flux (no direction)
    const R sL = frL * frL + fZL * fZL, sR = frR * frR + fZR * fZR;
    R iL, iR;
    if constexpr (sizeof(R) == 4) {
        iL = sL >= kFltMinNormal ? rsqf(sL) : R(0);
        iR = sR >= kFltMinNormal ? rsqf(sR) : R(0);
    } else {
        iL = sL >= kDblMinNormal ? rsqrt_nr(sL) : R(0);
        iR = sR >= kDblMinNormal ? rsqrt_nr(sR) : R(0);
    }
    R fL = sL * iL, fR = sR * iR;
    if (fL > R(1)) { frL *= iL; fZL *= iL; fL = R(1); iL = R(1); }
    if (fR > R(1)) { frR *= iR; fZR *= iR; fR = R(1); iR = R(1); }
    o.Hr_L = frL * o.J_L; o.Hr_R = frR * o.J_R;
    o.HZ_L = fZL * o.J_L; o.HZ_R = fZR * o.J_R;
    o.nr_L = frL * iL; o.nZ_L = fZL * iL;
    o.nr_R = frR * iR; o.nZ_R = fZR * iR;
    o.f_L = fL; o.f_R = fR;
    return o;
}

// ReconstructInterface from raw cells (J, H_r, H_Z).
template <typename R>
__device__ __forceinline__ Recon<R> reconstruct(const Cell<R> &cm1, const Cell<R> &ci, const Cell<R> &cp1,
                                                const Cell<R> &cp2, const R iv[5], R aF_i, R aF_ip1, R jeps) {
    return reconstruct_f<R>(cell_f<R>(cm1.J, cm1.Hr, cm1.HZ, jeps), cell_f<R>(ci.J, ci.Hr, ci.HZ, jeps),
                            cell_f<R>(cp1.J, cp1.Hr, cp1.HZ, jeps), cell_f<R>(cp2.J, cp2.Hr, cp2.HZ, jeps), iv,
                            aF_i, aF_ip1, jeps);
}

// GetFluxGLF / GetFluxHLL, src/AdvectJandH.jl:81-118, 155-204, with the wave speeds of
// M1WaveSpeeds_r/Z (src/M1Closure.jl:301-326). F{J,Hr,HZ}_{L,R} are the physical fluxes of
// the three conserved quantities on either side; Ji/Jip1 the cell values for the
// diffusion-limit term. ZDIR selects n_Z (true) or n_r (false) for the HLL eigenvalues.
template <typename R, int FLUX, bool ZDIR>
__device__ __forceinline__ void m1_flux(R FJ_L, R FJ_R, R FHr_L, R FHr_R, R FHZ_L, R FHZ_R,
                                        const Recon<R> &q, R Ji, R Jip1, R &FJ, R &FHr, R &FHZ) {
    R tau = q.tau_L + q.tau_R;
    R num = R(0.2) + tau;
    R eps = num * rcp<R>(num + tau * tau);
    R ome = R(1) - eps;
    R tau_eff = tau > Num<R>::tiny() ? tau : Num<R>::tiny();
    R FJ_diff = -Num<R>::third() * (Jip1 - Ji) * rcp<R>(tau_eff);
    if (FLUX == 0) {
        R FJ_glf = R(0.5) * (FJ_L + FJ_R) - R(0.5) * (q.J_R - q.J_L);
        FJ = eps * FJ_glf + ome * FJ_diff;
        R he = R(0.5) * eps;
        FHr = R(0.5) * (FHr_L + FHr_R) - he * (q.Hr_R - q.Hr_L);
        FHZ = R(0.5) * (FHZ_L + FHZ_R) - he * (q.HZ_R - q.HZ_L);
    } else {
        R l1L, l3L, l1R, l3R;
        hll_eigen<R>(q.f_L, ZDIR ? q.nZ_L : q.nr_L, l1L, l3L);
        hll_eigen<R>(q.f_R, ZDIR ? q.nZ_R : q.nr_R, l1R, l3R);
        R SR = fmax(fmax(l3L, l3R), R(0));
        R SL = fmin(fmin(l1L, l1R), R(0));
        R dS = SR - SL;
        R inv_dS = rcp<R>(dS > Num<R>::tiny() ? dS : Num<R>::tiny());
        R SRSL = SR * SL;
        R FJh = (SR * FJ_L - SL * FJ_R + SRSL * (q.J_R - q.J_L)) * inv_dS;
        R FHrh = (SR * FHr_L - SL * FHr_R + SRSL * (q.Hr_R - q.Hr_L)) * inv_dS;
        R FHZh = (SR * FHZ_L - SL * FHZ_R + SRSL * (q.HZ_R - q.HZ_L)) * inv_dS;
        R hom = R(0.5) * ome;
        FJ = eps * FJh + ome * FJ_diff;
        FHr = eps * FHrh + hom * (FHr_L + FHr_R);
        FHZ = eps * FHZh + hom * (FHZ_L + FHZ_R);
    }
}

// GetAdvectionFlux, src/AdvectJandH.jl:276-282
template <typename R>
__device__ __forceinline__ R adv_flux(R uc, R L, R Rv) { return uc * (uc < R(0) ? Rv : L); }

// Compute_K_phiphi_InnerAxis, src/AdvectJandH.jl:499-522
template <typename R>
__device__ __forceinline__ R k_phiphi_axis(R J, R HZ, R jeps) {
    J = J > jeps ? J : jeps;
    R fZ = HZ * rcp<R>(J);
    fZ = fZ < R(-1) ? R(-1) : (fZ > R(1) ? R(1) : fZ);
    R f = fabs(fZ);
    R nZ = f > R(0) ? (fZ > R(0) ? R(1) : R(-1)) : R(0);
    R Drr, DZZ, DrZ;
    D_from_f_n<R>(f, R(0), nZ, Drr, DZZ, DrZ);
    R k = R(1) - Drr - DZZ;
    k = k < R(0) ? R(0) : (k > R(1) ? R(1) : k);
    return k * J;
}

template <typename R>
__device__ __forceinline__ R clamp01(R x) { return x < R(0) ? R(0) : (x > R(1) ? R(1) : x); }

// D_colon_grad_u_Cylindrical, src/ConstantsAndFunctions.jl:883-895
template <typename R>
__device__ __forceinline__ R d_colon_grad_u(R Drr, R DrZ, R DZZ, R a, R b, R c, R d, R e) {
    R Dpp = R(1) - Drr - DZZ;
    Dpp = Dpp > R(0) ? Dpp : R(0);
    return Drr * a + DrZ * (b + c) + DZZ * d + Dpp * e;
}

// exp(x) for |x| <= 40 in FP64 by the table-driven method of P. T. P. Tang (ACM Trans. Math.
// Softw. 15 (1989) 144-157): x = (32 m + j) ln2/32 + r with |r| <= ln2/64, exp(x) = 2^m 2^(j/32)
// e^r. The 32 values 2^(j/32) are correctly rounded (generated in 80-digit decimal arithmetic),
// e^r - 1 is its Taylor polynomial to degree 6 (truncation below 4e-18 relative) and the
// result is 2^m (T + T (e^r - 1)) with one rounding: within about an ulp. round(32 x / ln2)
// comes out of one fused multiply-add with 1.5 * 2^52 (its low bits then hold the integer);
// ln2/32 is split in a 40-bit head, whose products with |32 x / ln2| < 2^13 are exact, and a
// tail. `tab` is kExp2Tab, or a copy of it in shared memory.
static __constant__ double kExp2Tab[32] = {
    0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0,
    0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0,
    0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0,
    0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0,
    0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0,
    0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0,
    0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0,
    0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0};
__device__ __forceinline__ double exp_tab(double x, const double *tab) {
    constexpr double kShift = 0x1.8p52, kInvL = 0x1.71547652b82fep+5;
    constexpr double kLhi = 0x1.62e42fefa2000p-6, kLlo = 0x1.9ef35793c7673p-46;
    const double t = fma(x, kInvL, kShift);
    const int N = __double2loint(t);
    const double Nd = t - kShift;
    double r = fma(-Nd, kLhi, x);
    r = fma(-Nd, kLlo, r);
    double q = fma(r, 1.0 / 720.0, 1.0 / 120.0);
    q = fma(q, r, 1.0 / 24.0);
    q = fma(q, r, 1.0 / 6.0);
    q = fma(q, r, 0.5);
    q = fma(q, r, 1.0);
    q *= r;
    const double T = tab[N & 31];
    const double s = __hiloint2double(((N >> 5) + 1023) << 20, 0);
    return fma(T, q, T) * s;
}

// OneMinusphi_L_and_chi_L / OneMinusphi_R_and_chi_R, src/FreqFactors.jl:54-133, in FP64.
// Every caller clamps P to [-Pmax, Pmax] first (src/FreqFactors.jl:248-250), so the reference's
// |P| >= Pmax branches only ever see P = +-Pmax, where they return exp(-+Pmax) and
// (1 - exp(-+Pmax)) / +-Pmax: the general expression at that P. What remains is the choice
// between the exponential and the second-order Taylor form below |P| = Pmin, taken here by a
// select on values the warp computes for every lane, so lanes of one warp never take
// different paths (at P = 0 the unused general value is not finite; the select drops it).
// The exponentials are exp_tab's (|P| <= Pmax = 40) with the table at `tab`.
__device__ __forceinline__ void omphi_L(double P, double &omp, double &chi, const double *tab) {
    const double e = exp_tab(-P, tab);
    const double x = (1.0 - e) * rcp<double>(P);
    const bool tay = fabs(P) < kPmin;
    omp = tay ? 1.0 - P + 0.5 * (P * P) : e;
    chi = tay ? 1.0 - 0.5 * P : x;
}
__device__ __forceinline__ void omphi_R(double P, double &omp, double &chi, const double *tab) {
    const double e = exp_tab(P, tab);
    const double x = (1.0 - e) * rcp<double>(P);
    const bool tay = fabs(P) < kPmin;
    omp = tay ? 1.0 + P + 0.5 * (P * P) : e;
    chi = tay ? -1.0 - 0.5 * P : x;
}
// Both of the above at once for the same P (used for P_k, which needs phi^L and phi^R):
// one exponential and one reciprocal of P serve the two.
__device__ __forceinline__ void omphi_LR(double P, double &oL, double &xL, double &oR, double &xR,
                                         const double *tab) {
    const double e = exp_tab(-P, tab);
    const double ie = rcp<double>(e);
    const double iP = rcp<double>(P);
    const bool tay = fabs(P) < kPmin;
    const double h = 0.5 * (P * P);
    oL = tay ? 1.0 - P + h : e;
    xL = tay ? 1.0 - 0.5 * P : (1.0 - e) * iP;
    oR = tay ? 1.0 + P + h : ie;
    xR = tay ? -1.0 - 0.5 * P : (1.0 - ie) * iP;
}
// Thermal velocity, Doppler width, Voigt parameter (src/ConstantsAndFunctions.jl:282-314)
__host__ __device__ __forceinline__ double compute_b(double T) { return sqrt(2.0 * kKBoltz / kMH) * sqrt(T); }
__host__ __device__ __forceinline__ double compute_dnuD(double T) { return compute_b(T) * (kNuLya / kC); }
__host__ __device__ __forceinline__ double compute_a(double T) {
    return (kALya / (kFourPi * kNuLya * 1.0 / kC)) / compute_b(T);
}

}  // namespace lyd
