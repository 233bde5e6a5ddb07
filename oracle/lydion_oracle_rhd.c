/*
 * lydion_oracle_rhd.c -- CPU FP64 restatement of the Lyman-alpha block of LYDION's per-cell
 * photo-thermochemistry sub-cycle, used ONLY as test infrastructure (the checker of the CUDA
 * path). Nothing in the product library links or calls this code.
 *
 * Follows (paths inside the LYDION source tree):
 *   PrepareLyaSubCycling!           src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:2087-2155
 *   Update_Hvoigt_And_phinu_cell!   src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:2039-2080
 *   AbsorptionStep, Lyman-alpha     src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:1580-1680
 *   SplitRadPressure                src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:1017-1046
 *   emissivities                    src/LymanAlphaEmission.jl:36-175
 *   krecHII_A / krecHII_B           src/PhotoChemistryAndCooling/GasChemistryRates.jl:166-204
 * PARITY: unpinned against the reference (no Julia here). Pinned points: the Storey & Hummer
 * (1995) table nodes and the Case B recombination rate at 1e4 K (tests/test_oracle.py).
 */
#include <math.h>
#include <stddef.h>

#include "lydion_oracle.h"

#define R_C_LIGHT   2.99792458e10
#define R_H_PLANCK  6.626069573e-27
#define R_K_BOLTZ   1.380648813e-16
#define R_NU_LYA    2.466068e15
#define R_NU_LYC    3.289842e15
#define R_FOUR_PI   (4.0 * M_PI)
#define SIG_T       6.6524587321e-25
#define SIG_OH_LYA  4.07e-18
#define SIG_CH_LYA  0.05e-18
#define SIG_RAMAN   2.1e-25
#define TOL_ABS     0.1
#define J_FLOOR_ABS 1e-15

/* Storey & Hummer (1995) probability of Lyman-alpha emission after a recombination, the
 * grids and tables of src/LymanAlphaEmission.jl:36-65 (rows: T, columns: n_e). */
static const double sh_T[10] = {5e2, 1e3, 3e3, 5e3, 7.5e3, 1e4, 1.25e4, 1.5e4, 2e4, 3e4};
static const double sh_neB[13] = {1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11, 1e12, 1e13, 1e14};
static const double sh_neA[9] = {1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10};
static const double sh_B[10][13] = {
    {0.80793637, 0.90215197, 0.98157401, 0.9970534, 0.99933853, 0.99934845, 0.99967896, 0.99948547, 0.99931146, 0.99951894, 0.9997498, 0.99864818, 0.99372263},
    {0.78439303, 0.87743841, 0.97423464, 0.99680114, 0.99960243, 0.99967816, 0.9997671, 0.99939133, 0.99922946, 0.99960973, 0.99937386, 0.99906812, 0.9954834},
    {0.74159266, 0.82809599, 0.95734434, 0.99359891, 0.99892162, 0.99927343, 0.99979471, 0.99938909, 0.99899055, 0.99925979, 0.99957955, 0.99923525, 0.99703571},
    {0.71946081, 0.80133228, 0.94581237, 0.99246182, 0.99848958, 0.99940329, 0.99949246, 0.99952048, 0.99981447, 0.99956726, 0.9993515, 0.99952024, 0.99692499},
    {0.70117195, 0.7788453, 0.93441344, 0.99075058, 0.99831301, 0.99960223, 0.99940949, 0.99946884, 0.99948297, 0.99947146, 0.99965311, 0.99918254, 0.99690311},
    {0.68808416, 0.76220739, 0.92503048, 0.9891268, 0.99828523, 0.9994074, 0.99944339, 0.99952601, 0.99932358, 0.99927528, 0.99938987, 0.99904232, 0.9949615},
    {0.6775581, 0.74868826, 0.9176273, 0.98784252, 0.99835238, 0.99903921, 0.99977064, 0.99954296, 0.99930529, 0.99954743, 0.99944997, 0.99874439, 0.9916493},
    {0.66862468, 0.73785038, 0.91033402, 0.98701405, 0.99817046, 0.99892625, 0.99953078, 0.99960556, 0.9993362, 0.99941558, 0.99944365, 0.99828039, 0.98817287},
    {0.65534642, 0.72080463, 0.89823705, 0.98497224, 0.99798854, 0.9988133, 0.99929092, 0.99909416, 0.99933199, 0.9995549, 0.99924446, 0.99764512, 0.97960152},
    {0.63566376, 0.69600394, 0.87952243, 0.98121463, 0.99716593, 0.99896144, 0.99905958, 0.9996252, 0.99953649, 0.99931002, 0.99872497, 0.99561256, 0.96391965}};
static const double sh_A[10][9] = {
    {0.58042473, 0.59595911, 0.60335363, 0.58990186, 0.56623927, 0.53426043, 0.492528, 0.44534414, 0.40955195},
    {0.54712958, 0.56465163, 0.57999443, 0.57241623, 0.5541246, 0.5276139, 0.49052298, 0.44606687, 0.4101595},
    {0.48320245, 0.50151448, 0.52818381, 0.53008608, 0.52008701, 0.50298698, 0.47625175, 0.43924427, 0.40696841},
    {0.44933274, 0.46714191, 0.49852558, 0.50475148, 0.49815515, 0.48505756, 0.46319941, 0.43069186, 0.40125666},
    {0.42087234, 0.43810743, 0.47280049, 0.48268151, 0.47821493, 0.46794659, 0.4497736, 0.42097532, 0.39442497},
    {0.40023971, 0.41675887, 0.45373431, 0.46591319, 0.46300415, 0.45454038, 0.43876097, 0.41249415, 0.38810578},
    {0.3840314, 0.40007514, 0.43832241, 0.45257107, 0.45064954, 0.4434932, 0.42939783, 0.40511911, 0.38230403},
    {0.37046215, 0.38617473, 0.42546609, 0.44143608, 0.44049428, 0.43394168, 0.42127472, 0.39854551, 0.37684759},
    {0.34937867, 0.36397106, 0.40484801, 0.42349201, 0.42367822, 0.41860328, 0.40761256, 0.38699493, 0.36739625},
    {0.31960139, 0.33302781, 0.37528203, 0.39805701, 0.39984039, 0.39602958, 0.38718651, 0.36963656, 0.3518518}};

/* index i with g[i] <= x <= g[i+1] on an increasing grid of n nodes (x inside [g0, g_{n-1}]) */
static int bracket(const double *g, int n, double x) {
    int i = 0;
    while (i < n - 2 && x > g[i + 1]) i++;
    return i;
}

/* Prob_Lya_SH95, src/LymanAlphaEmission.jl:71-90: bilinear in (log10 T, log10 n_e) on the
 * tables, the arguments clamped to the grids. */
double orc_prob_lya_sh95(double T, double ne, int caseB) {
    double lT[10], lne[13];
    const int nne = caseB ? 13 : 9;
    const double *gne = caseB ? sh_neB : sh_neA;
    for (int i = 0; i < 10; i++) lT[i] = log10(sh_T[i]);
    for (int i = 0; i < nne; i++) lne[i] = log10(gne[i]);
    double x = log10(T), y = log10(ne);
    x = x < lT[0] ? lT[0] : (x > lT[9] ? lT[9] : x);
    y = y < lne[0] ? lne[0] : (y > lne[nne - 1] ? lne[nne - 1] : y);
    const int i = bracket(lT, 10, x), j = bracket(lne, nne, y);
    const double t = (x - lT[i]) / (lT[i + 1] - lT[i]), u = (y - lne[j]) / (lne[j + 1] - lne[j]);
    double v00, v10, v01, v11;
    if (caseB) { v00 = sh_B[i][j]; v10 = sh_B[i + 1][j]; v01 = sh_B[i][j + 1]; v11 = sh_B[i + 1][j + 1]; }
    else { v00 = sh_A[i][j]; v10 = sh_A[i + 1][j]; v01 = sh_A[i][j + 1]; v11 = sh_A[i + 1][j + 1]; }
    return (1.0 - t) * ((1.0 - u) * v00 + u * v01) + t * ((1.0 - u) * v10 + u * v11);
}

/* krecHII (Case B with the on-the-spot approximation, else Case A),
 * src/PhotoChemistryAndCooling/GasChemistryRates.jl:166-204 */
double orc_krec_hii(double T, int ots) {
    T = T < 1.0 ? 1.0 : (T > 1e9 ? 1e9 : T);
    const double lam = 315614.0 / T;
    if (ots) return 2.753e-14 * pow(lam, 1.5) / pow(1.0 + pow(lam / 2.74, 0.407), 2.242);
    return 1.269e-13 * pow(lam, 1.503) / pow(1.0 + pow(lam / 0.522, 0.47), 1.923);
}

/* int dnu js_recLya, src/LymanAlphaEmission.jl:106-131 */
double orc_js_rec_lya(double T, double nHII, double ne, int ots) {
    const double E = R_H_PLANCK * R_NU_LYA / R_FOUR_PI;
    return orc_prob_lya_sh95(T, ne, ots) * orc_krec_hii(T, ots) * nHII * ne * E;
}

/* int dnu js_collLya, src/LymanAlphaEmission.jl:148-175 (Smith et al. 2022 fits) */
double orc_js_coll_lya(double T, double nHI, double ne) {
    const double Tryd = R_H_PLANCK * R_NU_LYC / R_K_BOLTZ;
    const double T12 = (1.0 - 1.0 / 4.0) * Tryd, T13 = (1.0 - 1.0 / 9.0) * Tryd;
    const double T14 = (1.0 - 1.0 / 16.0) * Tryd, T15 = (1.0 - 1.0 / 25.0) * Tryd;
    T = T > 1.0 ? T : 1.0;
    const double iT = 1.0 / T;
    const double T6 = (T < 3e5 ? T : 3e5) * 1e-6, T62 = T6 * T6, T63 = T62 * T6;
    const double Y12 = 0.267486 + 1.57257 * T6 - 6.44026 * T62 + 11.5401 * T63;
    const double Y13 = 0.0940821 + 2.90748 * T6 - 6.69528 * T62 + 7.86419 * T63;
    const double Y14 = 0.0415028 + 1.13673 * T6 - 3.97454 * T62 + 6.05941 * T63;
    const double Y15 = 0.032277 + 0.40856 * T6 - 1.34604 * T62 + 2.07558 * T63;
    const double q = (8.63e-6 / (2.0 * sqrt(T))) *
                     (Y12 * exp(-T12 * iT) + Y13 * exp(-T13 * iT) + Y14 * exp(-T14 * iT) + Y15 * exp(-T15 * iT));
    return q * nHI * ne * (R_H_PLANCK * R_NU_LYA / R_FOUR_PI);
}

/* PrepareLyaSubCycling! without the profile part: sp = {T, nHI, nH2, nHII, nHeI, ne, nOHx, nCHx,
 * rho_Sil, rho_C, rho_PAH}; out = {alpha, alpha_c, alpha_cF, pd, js, aF_Sil, aF_C, aF_PAH}. */
void orc_rhd_lya_prepare_cell(const double sp[11], const orc_dust_lya *d, double z, int ots, int destruction,
                              double out[8]) {
    const double T = sp[0], nHI = sp[1], nH2 = sp[2], nHII = sp[3], nHeI = sp[4], ne = sp[5];
    const double nOHx = sp[6], nCHx = sp[7];
    double rho[3];
    for (int q = 0; q < 3; q++) rho[q] = sp[8 + q] > d->rho_ignore ? sp[8 + q] : 0.0;
    const double abs_gas = nH2 * SIG_RAMAN + nOHx * SIG_OH_LYA + nCHx * SIG_CH_LYA;
    const double F_gas = abs_gas + ne * SIG_T;
    out[0] = nHI * orc_compute_sigma0(T);
    out[1] = d->kappa_abs[0] * rho[0] + d->kappa_abs[1] * rho[1] + d->kappa_abs[2] * rho[2] + abs_gas;
    out[2] = d->kappa_F[0] * rho[0] + d->kappa_F[1] * rho[1] + d->kappa_F[2] * rho[2] + F_gas;
    out[3] = destruction ? orc_pd_lya(nHII, ne, nHI, nHeI, nH2, T, z) : 0.0;
    out[4] = orc_js_rec_lya(T, nHII, ne, ots) + orc_js_coll_lya(T, nHI, ne);
    for (int q = 0; q < 3; q++) out[5 + q] = d->kappa_F[q] * rho[q];
}

/* The Lyman-alpha block of AbsorptionStep for one cell over the sub-step dt. cell = the
 * prepare outputs; Hv, phi, J_old, H_old of the cell's n_nu bins; writes J, H. out = {e_new,
 * de, dru_r, dru_Z, gas_r, gas_Z, Sil_r, Sil_Z, C_r, C_Z, PAH_r, PAH_Z, dt_Lya}; returns 1 when
 * the step is rejected (the relative change of e_Lya exceeds tol_Abs while dt exceeds tol_Abs
 * times the absorption time, or is not finite). */
int orc_rhd_lya_absorb_cell(int nnu, const double *dnu, const double *Hv, const double *phi, const double *J_old,
                            const double *Hr_old, const double *HZ_old, double *J, double *Hr, double *HZ,
                            const double cell[8], double dt, double c_tilde, double e_old, double jeps,
                            double out[13]) {
    const double alpha = cell[0], ac = cell[1], acF = cell[2], pd = cell[3], js = cell[4];
    const double dS = cell[5], dC = cell[6], dP = cell[7];
    const double ic = 1.0 / c_tilde, ct_js = c_tilde * js, pd_a = pd * alpha;
    const double dt_lya = ic / (ac + pd_a);
    double intJ = 0.0, dr = 0.0, dz = 0.0, split[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < nnu; k++) {
        const double dJdt = ct_js * phi[k];
        const double a_abs = ac + pd_a * Hv[k];
        double Jn = (J_old[k] + dJdt * dt) / (1.0 + a_abs * c_tilde * dt);
        J[k] = Jn > jeps ? Jn : jeps;
        const double aF = alpha * Hv[k] + acF;
        Hr[k] = Hr_old[k] / (1.0 + aF * c_tilde * dt);
        HZ[k] = HZ_old[k] / (1.0 + aF * c_tilde * dt);
        const double w = dnu[k] * (R_FOUR_PI / R_C_LIGHT);
        const double mr = w * (ic * (Hr_old[k] - Hr[k])), mz = w * (ic * (HZ_old[k] - HZ[k]));
        dr += mr;
        dz += mz;
        double ag = aF - dS - dC - dP;
        ag = ag > 0.0 ? ag : 0.0;
        const double tot = ag + dS + dC + dP;
        double f[4] = {1.0, 0.0, 0.0, 0.0};
        if (tot > 0.0) {
            const double it = 1.0 / tot;
            f[0] = ag * it; f[1] = dS * it; f[2] = dC * it; f[3] = dP * it;
        }
        for (int q = 0; q < 4; q++) { split[2 * q] += f[q] * mr; split[2 * q + 1] += f[q] * mz; }
        intJ += dnu[k] * J[k];
    }
    const double e_new = (R_FOUR_PI / R_C_LIGHT) * intJ;
    const double de = fabs(e_new - e_old) / (e_old + (R_FOUR_PI / R_C_LIGHT) * J_FLOOR_ABS);
    out[0] = e_new; out[1] = de; out[2] = dr; out[3] = dz;
    for (int q = 0; q < 8; q++) out[4 + q] = split[q];
    out[12] = dt_lya;
    return ((de > TOL_ABS && dt > TOL_ABS * dt_lya) || !isfinite(de)) ? 1 : 0;
}

/* FindRSL_LyaRT, src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:614-711, on a single
 * cloud: cell arrays of nr*nz (i fastest), rho_d [3][nr*nz], interfaces r (nr+1) and Z (nz+1). */
double orc_find_rsl_lya(int nr, int nz, const double *r, const double *Z, const double *u_r, const double *u_Z,
                        const double *P, const double *rho, const double *gamma_ad, const double *T,
                        const double *xHII, const double *xH2, const double *rho_d, const double *pd,
                        const double kappa_abs[3], double eps_rsl, double X_over_mH, double ct_old,
                        double ct_min) {
    const size_t n = (size_t)nr * nz;
    double ct = 0.0;
    for (int j = 0; j < nz; j++) {
        const double dZ = Z[j + 1] - Z[j];
        for (int i = 0; i < nr; i++) {
            const size_t c = (size_t)i + (size_t)nr * j;
            const double dr = r[i + 1] - r[i];
            const double cs = sqrt(gamma_ad[c] * P[c] / rho[c]);
            double xHI = 1.0 - xHII[c] - 2.0 * xH2[c];
            xHI = xHI > 0.0 ? xHI : 0.0;
            const double nHI = xHI * X_over_mH * rho[c];
            const double alpha = nHI * orc_compute_sigma0(T[c]);
            const double dX = dr > dZ ? dr : dZ;
            const double tau = alpha * dX;
            const double tauc = (kappa_abs[0] * rho_d[c] + kappa_abs[1] * rho_d[n + c] + kappa_abs[2] * rho_d[2 * n + c]) * dX;
            const double at = orc_compute_a(T[c]) * tau;
            const double at13 = pow(at, 1.0 / 3.0);
            const double fabs_ = 1.0 / (1.0 + at13 * tauc + 0.6 * pd[c] * tau);
            const double u = hypot(u_r[c], u_Z[c]);
            const double f = at13 * fabs_;
            const double v = eps_rsl * (f > 1.0 ? f : 1.0) * (u > cs ? u : cs);
            ct = v > ct ? v : ct;
        }
    }
    ct = ct < ct_min ? ct_min : ct;
    ct = ct < R_C_LIGHT ? ct : R_C_LIGHT;
    if (ct < ct_old) ct = ct > 0.75 * ct_old ? ct : 0.75 * ct_old;
    if (ct > ct_old) ct = ct < 4.0 * ct_old ? ct : 4.0 * ct_old;
    return ct;
}
