/*
 * lydion_oracle.c -- CPU FP64 restatement of the LYDION Lyman-alpha M1 step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA library and the CPU
 * baseline timed beside it; the product never links it. Parity status: the step is
 * "parity unpinned" (the Julia reference cannot run here and ships no J/H golden
 * vectors); its LAPACK dgtsv and the erf/Dawson Voigt tables are pinned by committed
 * scipy fixtures. See lydion_oracle.h.
 *
 * Each function names the reference file:line it restates. The code follows the
 * reference's loop structure and operation order where that affects rounding (face by
 * face in AdvectJandH_Cylindrical!, serial reductions), but it is written from the
 * algorithm, in C, 0-based. Compiled without fast-math and without FMA contraction.
 */
#include "lydion_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- constants: src/ConstantsAndFunctions.jl:46-170, src/M1Closure.jl:36-41,
 *      src/FreqFactors.jl:16-18, src/UpdateLyaJandH.jl:43 ----------------------- */
#define C_LIGHT     2.99792458e10
#define H_PLANCK    6.626069573e-27
#define K_BOLTZ     1.380648813e-16
#define M_U         1.660539069e-24
#define M_H         (1.0080 * M_U)
#define M_ELEC         9.109382917e-28
#define E_CHARGE    4.80320451e-10
#define NU_LYA      2.466068e15
#define A_LYA       6.265e8
#define A_2GAM      8.2206
#define A_2P2S      8.78e-7
#define A_2S2P      1.597e-9
#define F_LU_LYA    0.41641

static const double ONE_THIRD  = 1.0 / 3.0;
static const double TWO_THIRDS = 2.0 / 3.0;
#define FOUR_PI (4.0 * M_PI)

static const double FMIN = 1e-10;
static const double FMAX = 1.0 - 1e-10;
static const double JEPS = 1e-60;
static const double HEPS = 1e-100;
static const double PMIN = 1e-3;
static const double PMAX = 40.0;
static const double EPS_ACTIVE = 1e-10;

static inline size_t ix3(int nnu, int nr, int k, int i, int j) {
    return (size_t)k + (size_t)nnu * ((size_t)i + (size_t)nr * (size_t)j);
}
static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline double dclamp(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* MinMod: src/ConstantsAndFunctions.jl:1571-1582 */
double orc_minmod(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    return fabs(a) < fabs(b) ? a : b;
}

/* Levermore (1984) Eddington factor: src/M1Closure.jl:28-33 */
double orc_chi_L84(double f) {
    double f2 = f * f;
    return (3.0 + 4.0 * f2) / (5.0 + 2.0 * sqrt(4.0 - 3.0 * f2));
}

/* Compute_D_Edd: src/M1Closure.jl:46-83 */
void orc_D_edd(double Hr, double HZ, double J, double out[3]) {
    double H2 = Hr * Hr + HZ * HZ;
    if (J <= JEPS || H2 <= HEPS * HEPS || H2 <= (FMIN * FMIN) * J * J) {
        out[0] = ONE_THIRD; out[1] = ONE_THIRD; out[2] = 0.0;
        return;
    }
    double Hmag = sqrt(H2);
    double f = dclamp(Hmag / J, FMIN, FMAX);
    double chi = orc_chi_L84(f);
    double inv_H = 1.0 / Hmag;
    double a = (1.0 - chi) * 0.5;
    double b = (3.0 * chi - 1.0) * 0.5;
    double nr = Hr * inv_H, nZ = HZ * inv_H;
    double b_nr = b * nr;
    out[0] = a + b_nr * nr;
    out[1] = a + b * nZ * nZ;
    out[2] = b_nr * nZ;
}

/* Compute_D_Edd_from_f_n: src/M1Closure.jl:91-119 */
void orc_D_edd_from_f_n(double f, double nr, double nZ, double out[3]) {
    if (f > FMIN) {
        f = dmin(f, FMAX);
        double chi = orc_chi_L84(f);
        double a = (1.0 - chi) * 0.5;
        double b = (3.0 * chi - 1.0) * 0.5;
        double b_nr = b * nr;
        out[0] = a + b_nr * nr;
        out[1] = a + b * nZ * nZ;
        out[2] = b_nr * nZ;
    } else {
        out[0] = ONE_THIRD; out[1] = ONE_THIRD; out[2] = 0.0;
    }
}

/* HLL_Eigenvalues: src/M1Closure.jl:273-296 */
void orc_hll_eigenvalues(double f, double mu, double out[2]) {
    f = dclamp(f, FMIN, FMAX);
    mu = dclamp(mu, -1.0, 1.0);
    double f2 = f * f, mu2 = mu * mu, muf = mu * f;
    double sq = sqrt(dmax(4.0 - 3.0 * f2, 0.0));
    double inv_sq = 1.0 / sq;
    double fac = sqrt(dmax(TWO_THIRDS * (4.0 - 3.0 * f2 - sq) + 2.0 * mu2 * (2.0 - f2 - sq), 0.0));
    out[0] = dclamp((muf - fac) * inv_sq, -1.0, 1.0);
    out[1] = dclamp((muf + fac) * inv_sq, -1.0, 1.0);
}

/* ---- interface reconstruction and fluxes: src/AdvectJandH.jl:81-522 ---------- */
typedef struct recon {
    double J_L, J_R, Hr_L, Hr_R, HZ_L, HZ_R, tau_L, tau_R, f_L, f_R, nr_L, nr_R, nZ_L, nZ_R;
} recon;

/* ReconstructInterface: src/AdvectJandH.jl:359-473 */
static recon reconstruct(double J_i, double J_ip1, double J_ip2, double J_im1,
                         double Hr_i, double Hr_ip1, double Hr_ip2, double Hr_im1,
                         double HZ_i, double HZ_ip1, double HZ_ip2, double HZ_im1,
                         double dL, double dR, double inv_i_im1, double inv_ip1_i, double inv_ip2_ip1,
                         double aF_i, double aF_ip1) {
    recon o;
    o.tau_L = aF_i * dL;
    o.tau_R = aF_ip1 * dR;
    double iJ_i = 1.0 / dmax(J_i, JEPS), iJ_ip1 = 1.0 / dmax(J_ip1, JEPS);
    double iJ_ip2 = 1.0 / dmax(J_ip2, JEPS), iJ_im1 = 1.0 / dmax(J_im1, JEPS);
    double fr_i = Hr_i * iJ_i, fr_ip1 = Hr_ip1 * iJ_ip1, fr_ip2 = Hr_ip2 * iJ_ip2, fr_im1 = Hr_im1 * iJ_im1;
    double fZ_i = HZ_i * iJ_i, fZ_ip1 = HZ_ip1 * iJ_ip1, fZ_ip2 = HZ_ip2 * iJ_ip2, fZ_im1 = HZ_im1 * iJ_im1;

    double dJ_c = (J_ip1 - J_i) * inv_ip1_i;
    double dJ_L = orc_minmod((J_i - J_im1) * inv_i_im1, dJ_c);
    double dJ_R = orc_minmod((J_ip2 - J_ip1) * inv_ip2_ip1, dJ_c);
    double dfr_c = (fr_ip1 - fr_i) * inv_ip1_i;
    double dfr_L = orc_minmod((fr_i - fr_im1) * inv_i_im1, dfr_c);
    double dfr_R = orc_minmod((fr_ip2 - fr_ip1) * inv_ip2_ip1, dfr_c);
    double dfZ_c = (fZ_ip1 - fZ_i) * inv_ip1_i;
    double dfZ_L = orc_minmod((fZ_i - fZ_im1) * inv_i_im1, dfZ_c);
    double dfZ_R = orc_minmod((fZ_ip2 - fZ_ip1) * inv_ip2_ip1, dfZ_c);

    o.J_L = dmax(J_i + dJ_L * dL, JEPS);
    o.J_R = dmax(J_ip1 - dJ_R * dR, JEPS);
    double fr_L = fr_i + dfr_L * dL, fr_R = fr_ip1 - dfr_R * dR;
    double fZ_L = fZ_i + dfZ_L * dL, fZ_R = fZ_ip1 - dfZ_R * dR;

    double f_L = sqrt(fr_L * fr_L + fZ_L * fZ_L);
    if (f_L > 1.0) { double inv = 1.0 / f_L; fr_L *= inv; fZ_L *= inv; f_L = 1.0; }
    double f_R = sqrt(fr_R * fr_R + fZ_R * fZ_R);
    if (f_R > 1.0) { double inv = 1.0 / f_R; fr_R *= inv; fZ_R *= inv; f_R = 1.0; }

    o.Hr_L = fr_L * o.J_L; o.Hr_R = fr_R * o.J_R;
    o.HZ_L = fZ_L * o.J_L; o.HZ_R = fZ_R * o.J_R;
    if (f_L > 0.0) { double inv = 1.0 / f_L; o.nr_L = fr_L * inv; o.nZ_L = fZ_L * inv; }
    else { o.nr_L = 0.0; o.nZ_L = 0.0; }
    if (f_R > 0.0) { double inv = 1.0 / f_R; o.nr_R = fr_R * inv; o.nZ_R = fZ_R * inv; }
    else { o.nr_R = 0.0; o.nZ_R = 0.0; }
    o.f_L = f_L; o.f_R = f_R;
    return o;
}

/* GetFluxGLF: src/AdvectJandH.jl:81-118 */
static void flux_glf(double FJ_L, double FJ_R, double FHr_L, double FHr_R, double FHZ_L, double FHZ_R,
                     const recon *q, double J_i, double J_ip1, double out[3]) {
    double tau = q->tau_L + q->tau_R;
    double num = 0.2 + tau;
    double eps = num / (num + tau * tau);
    double ome = 1.0 - eps;
    double tau_eff = dmax(tau, 1e-300);
    double FJ_diff = -ONE_THIRD * (J_ip1 - J_i) / tau_eff;
    double FJ_glf = 0.5 * (FJ_L + FJ_R) - 0.5 * (q->J_R - q->J_L);
    out[0] = eps * FJ_glf + ome * FJ_diff;
    double he = 0.5 * eps;
    out[1] = 0.5 * (FHr_L + FHr_R) - he * (q->Hr_R - q->Hr_L);
    out[2] = 0.5 * (FHZ_L + FHZ_R) - he * (q->HZ_R - q->HZ_L);
}

/* GetFluxHLL: src/AdvectJandH.jl:155-204 with M1WaveSpeeds_r/Z: src/M1Closure.jl:301-326 */
static void flux_hll(double FJ_L, double FJ_R, double FHr_L, double FHr_R, double FHZ_L, double FHZ_R,
                     const recon *q, double J_i, double J_ip1, int zdir, double out[3]) {
    double eL[2], eR[2];
    orc_hll_eigenvalues(q->f_L, zdir ? q->nZ_L : q->nr_L, eL);
    orc_hll_eigenvalues(q->f_R, zdir ? q->nZ_R : q->nr_R, eR);
    double tau = q->tau_L + q->tau_R;
    double num = 0.2 + tau;
    double eps = num / (num + tau * tau);
    double ome = 1.0 - eps;
    double hom = 0.5 * ome;
    double tau_eff = dmax(tau, 1e-300);
    double FJ_diff = -ONE_THIRD * (J_ip1 - J_i) / tau_eff;
    double S_R = dmax(dmax(eL[1], eR[1]), 0.0);
    double S_L = dmin(dmin(eL[0], eR[0]), 0.0);
    double inv_dS = 1.0 / dmax(S_R - S_L, 1e-300);
    double SRSL = S_R * S_L;
    double FJ = (S_R * FJ_L - S_L * FJ_R + SRSL * (q->J_R - q->J_L)) * inv_dS;
    double FHr = (S_R * FHr_L - S_L * FHr_R + SRSL * (q->Hr_R - q->Hr_L)) * inv_dS;
    double FHZ = (S_R * FHZ_L - S_L * FHZ_R + SRSL * (q->HZ_R - q->HZ_L)) * inv_dS;
    out[0] = eps * FJ + ome * FJ_diff;
    out[1] = eps * FHr + hom * (FHr_L + FHr_R);
    out[2] = eps * FHZ + hom * (FHZ_L + FHZ_R);
}

/* GetAdvectionFlux: src/AdvectJandH.jl:276-282 */
static inline double adv_flux(double u_over_c, double L, double R) {
    return u_over_c * (u_over_c < 0.0 ? R : L);
}

/* Compute_K_phiphi_InnerAxis: src/AdvectJandH.jl:499-522 */
static double k_phiphi_axis(double J_axis, double HZ_axis) {
    J_axis = dmax(J_axis, JEPS);
    double fZ = dclamp(HZ_axis / J_axis, -1.0, 1.0);
    double f = fabs(fZ);
    double nZ = (f > 0.0) ? (fZ > 0.0 ? 1.0 : -1.0) : 0.0;
    double D[3];
    orc_D_edd_from_f_n(f, 0.0, nZ, D);
    return dclamp(1.0 - D[0] - D[1], 0.0, 1.0) * J_axis;
}

/* One r-interface (GetFluxM1 with Val(:r)) plus the advection flux, as done at each
 * face inside src/AdvectJandH.jl:641-968. Writes the three fluxes and, through kL/kR,
 * the generic K_phiphi values clamp(1-Drr-DZZ,0,1)*J of both sides. */
static void face_r(int flux_method, double uc, const recon *q, double J_i, double J_ip1,
                   double F[3], double *kL, double *kR) {
    double DL[3], DR[3];
    orc_D_edd_from_f_n(q->f_L, q->nr_L, q->nZ_L, DL);
    orc_D_edd_from_f_n(q->f_R, q->nr_R, q->nZ_R, DR);
    double Krr_L = DL[0] * q->J_L, Krr_R = DR[0] * q->J_R;
    double KrZ_L = DL[2] * q->J_L, KrZ_R = DR[2] * q->J_R;
    double o[3];
    if (flux_method == ORC_FLUX_HLL)
        flux_hll(q->Hr_L, q->Hr_R, Krr_L, Krr_R, KrZ_L, KrZ_R, q, J_i, J_ip1, 0, o);
    else
        flux_glf(q->Hr_L, q->Hr_R, Krr_L, Krr_R, KrZ_L, KrZ_R, q, J_i, J_ip1, o);
    F[0] = o[0] + adv_flux(uc, q->J_L, q->J_R);
    F[1] = o[1] + adv_flux(uc, q->Hr_L, q->Hr_R);
    F[2] = o[2] + adv_flux(uc, q->HZ_L, q->HZ_R);
    *kL = dclamp(1.0 - DL[0] - DL[1], 0.0, 1.0) * q->J_L;
    *kR = dclamp(1.0 - DR[0] - DR[1], 0.0, 1.0) * q->J_R;
}

/* One Z-interface (GetFluxM1 with Val(:Z)), src/AdvectJandH.jl:978-1289 */
static void face_z(int flux_method, double uc, const recon *q, double J_i, double J_ip1, double F[3]) {
    double DL[3], DR[3];
    orc_D_edd_from_f_n(q->f_L, q->nr_L, q->nZ_L, DL);
    orc_D_edd_from_f_n(q->f_R, q->nr_R, q->nZ_R, DR);
    double KZZ_L = DL[1] * q->J_L, KZZ_R = DR[1] * q->J_R;
    double KrZ_L = DL[2] * q->J_L, KrZ_R = DR[2] * q->J_R;
    double o[3];
    if (flux_method == ORC_FLUX_HLL)
        flux_hll(q->HZ_L, q->HZ_R, KrZ_L, KrZ_R, KZZ_L, KZZ_R, q, J_i, J_ip1, 1, o);
    else
        flux_glf(q->HZ_L, q->HZ_R, KrZ_L, KrZ_R, KZZ_L, KZZ_R, q, J_i, J_ip1, o);
    F[0] = o[0] + adv_flux(uc, q->J_L, q->J_R);
    F[1] = o[1] + adv_flux(uc, q->Hr_L, q->Hr_R);
    F[2] = o[2] + adv_flux(uc, q->HZ_L, q->HZ_R);
}

/* D_colon_grad_u_Cylindrical: src/ConstantsAndFunctions.jl:883-895 */
static inline double d_colon_grad_u(double Drr, double DrZ, double DZZ, double a, double b,
                                    double c, double d, double e) {
    double Dpp = dmax(1.0 - Drr - DZZ, 0.0);
    return Drr * a + DrZ * (b + c) + DZZ * d + Dpp * e;
}

/* FindActiveBins: src/UpdateLyaJandH.jl:47-97 (serial, k-outer second pass) */
void orc_find_active_bins(const orc_lya *s, const orc_geom *g, int *kmin_out, int *kmax_out) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    double Etot = 0.0;
    for (int j = 0; j < nz; j++)
        for (int i = 0; i < nr; i++) {
            double dV = g->dV[i + nr * j];
            for (int k = 0; k < nnu; k++)
                Etot += s->dnu[k] * dmax(s->J[ix3(nnu, nr, k, i, j)] - JEPS, 0.0) * dV;
        }
    int kmin = nnu - 1, kmax = 0;
    for (int k = 0; k < nnu; k++) {
        double Ebin = 0.0;
        for (int j = 0; j < nz; j++)
            for (int i = 0; i < nr; i++)
                Ebin += s->dnu[k] * dmax(s->J[ix3(nnu, nr, k, i, j)] - 10.0 * JEPS, 0.0) * g->dV[i + nr * j];
        if (Ebin > EPS_ACTIVE * Etot) {
            if (k < kmin) kmin = k;
            if (k > kmax) kmax = k;
        }
    }
    if (s->kcore_max > kmax) kmax = s->kcore_max;
    if (s->kcore_min < kmin) kmin = s->kcore_min;
    *kmin_out = kmin;
    *kmax_out = kmax;
}

/* AdvectJandH_Cylindrical!: src/AdvectJandH.jl:526-1390 */
void orc_advect_jh(orc_lya *s, const orc_geom *g, const orc_vel *v, double ctdt, int update_jold,
                   int bc_r_right, int bc_z_bot, int bc_z_top, int kmin, int kmax) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    const int fm = s->flux_method;
    const int k0 = kmin < 0 ? 0 : kmin;
    const int k1 = kmax > nnu - 1 ? nnu - 1 : kmax;
    const double inv_c = 1.0 / C_LIGHT;
    const double ctdt_c = ctdt * inv_c;
    double *J = s->J, *Hr = s->H_r, *HZ = s->H_Z;
    const double *aF = s->alpha_F;
#define IR(k, f, j) ((size_t)(k) + (size_t)nnu * ((size_t)(f) + (size_t)(nr + 1) * (size_t)(j)))
#define IZ(k, i, f) ((size_t)(k) + (size_t)nnu * ((size_t)(i) + (size_t)nr * (size_t)(f)))
#define I3(k, i, j) ix3(nnu, nr, k, i, j)

    /* r-direction fluxes, src/AdvectJandH.jl:641-968 */
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nz; j++) {
        double uc0 = v->u_r_star[0 + (nr + 1) * j] * inv_c;
        double uc1 = v->u_r_star[1 + (nr + 1) * j] * inv_c;
        for (int k = k0; k <= k1; k++) {
            double J1 = J[I3(k, 0, j)], J2 = J[I3(k, 1, j)];
            double Hr1 = Hr[I3(k, 0, j)], Hr2 = Hr[I3(k, 1, j)];
            double HZ1 = HZ[I3(k, 0, j)], HZ2 = HZ[I3(k, 1, j)];
            double aF1 = aF[I3(k, 0, j)];
            /* axis ghost cells (always reflecting), src/AdvectJandH.jl:662-673; on a Cartesian
             * grid the first interface may let flow out instead (:1537-1545) */
            double J0 = J1, Hr0 = -Hr1, HZ0 = HZ1;
            double Jm1 = J2, Hrm1 = -Hr2, HZm1 = HZ2;
            if (g->bc_r_left == ORC_BC_OUTFLOW) {
                Hr0 = dmin(Hr1, 0.0);
                Jm1 = J0; Hrm1 = Hr0; HZm1 = HZ0;
            }
            recon q = reconstruct(J0, J1, J2, Jm1, Hr0, Hr1, Hr2, Hrm1, HZ0, HZ1, HZ2, HZm1,
                                  g->dr_b[0], g->dr_b[1], g->dr_b[2], g->dr_b[3], g->dr_b[4], aF1, aF1);
            double Fo[3], kL, kR;
            face_r(fm, uc0, &q, J0, J1, Fo, &kL, &kR);
            s->F_r[IR(k, 0, j)] = Fo[0]; s->F_r_Hr[IR(k, 0, j)] = Fo[1]; s->F_r_HZ[IR(k, 0, j)] = Fo[2];
            s->K_imh[I3(k, 0, j)] = k_phiphi_axis(q.J_R, q.HZ_R);
            /* interface i = 3/2 */
            q = reconstruct(J1, J2, J[I3(k, 2, j)], J0, Hr1, Hr2, Hr[I3(k, 2, j)], Hr0,
                            HZ1, HZ2, HZ[I3(k, 2, j)], HZ0, g->dr_L[0], g->dr_R[0],
                            g->inv_dr_i_im1[0], g->inv_dr_ip1_i[0], g->inv_dr_ip2_ip1[0],
                            aF1, aF[I3(k, 1, j)]);
            face_r(fm, uc1, &q, J1, J2, Fo, &kL, &kR);
            s->F_r[IR(k, 1, j)] = Fo[0]; s->F_r_Hr[IR(k, 1, j)] = Fo[1]; s->F_r_HZ[IR(k, 1, j)] = Fo[2];
            s->K_iph[I3(k, 0, j)] = kL;
            s->K_imh[I3(k, 1, j)] = kR;
        }
        /* interior interfaces, src/AdvectJandH.jl:770-834 (1-based i = 2..N_r-2) */
        for (int i = 1; i <= nr - 3; i++) {
            double uc = v->u_r_star[(i + 1) + (nr + 1) * j] * inv_c;
            for (int k = k0; k <= k1; k++) {
                double Ji = J[I3(k, i, j)], Jip1 = J[I3(k, i + 1, j)];
                recon q = reconstruct(Ji, Jip1, J[I3(k, i + 2, j)], J[I3(k, i - 1, j)],
                                      Hr[I3(k, i, j)], Hr[I3(k, i + 1, j)], Hr[I3(k, i + 2, j)], Hr[I3(k, i - 1, j)],
                                      HZ[I3(k, i, j)], HZ[I3(k, i + 1, j)], HZ[I3(k, i + 2, j)], HZ[I3(k, i - 1, j)],
                                      g->dr_L[i], g->dr_R[i], g->inv_dr_i_im1[i], g->inv_dr_ip1_i[i],
                                      g->inv_dr_ip2_ip1[i], aF[I3(k, i, j)], aF[I3(k, i + 1, j)]);
                double Fo[3], kL, kR;
                face_r(fm, uc, &q, Ji, Jip1, Fo, &kL, &kR);
                s->F_r[IR(k, i + 1, j)] = Fo[0]; s->F_r_Hr[IR(k, i + 1, j)] = Fo[1];
                s->F_r_HZ[IR(k, i + 1, j)] = Fo[2];
                s->K_iph[I3(k, i, j)] = kL;
                s->K_imh[I3(k, i + 1, j)] = kR;
            }
        }
        /* outer interfaces N_r-1/2 and N_r+1/2, src/AdvectJandH.jl:837-965 */
        double ucN = v->u_r_star[(nr - 1) + (nr + 1) * j] * inv_c;
        double ucNp1 = v->u_r_star[nr + (nr + 1) * j] * inv_c;
        for (int k = k0; k <= k1; k++) {
            int N = nr - 1;
            double JN = J[I3(k, N, j)], JNm1 = J[I3(k, N - 1, j)];
            double HrN = Hr[I3(k, N, j)], HrNm1 = Hr[I3(k, N - 1, j)];
            double HZN = HZ[I3(k, N, j)], HZNm1 = HZ[I3(k, N - 1, j)];
            double aFN = aF[I3(k, N, j)];
            double JNp1, HrNp1, HZNp1, JNp2, HrNp2, HZNp2;
            if (bc_r_right == ORC_BC_REFLECT) {
                JNp1 = JN; HrNp1 = -HrN; HZNp1 = HZN;
                JNp2 = JNm1; HrNp2 = -HrNm1; HZNp2 = HZNm1;
            } else {
                JNp1 = JN; HrNp1 = dmax(HrN, 0.0); HZNp1 = HZN;
                JNp2 = JNp1; HrNp2 = HrNp1; HZNp2 = HZNp1;
            }
            recon q = reconstruct(JNm1, JN, JNp1, J[I3(k, N - 2, j)], HrNm1, HrN, HrNp1, Hr[I3(k, N - 2, j)],
                                  HZNm1, HZN, HZNp1, HZ[I3(k, N - 2, j)], g->dr_L[N - 1], g->dr_R[N - 1],
                                  g->inv_dr_i_im1[N - 1], g->inv_dr_ip1_i[N - 1], g->inv_dr_ip2_ip1[N - 1],
                                  aF[I3(k, N - 1, j)], aFN);
            double Fo[3], kL, kR;
            face_r(fm, ucN, &q, JNm1, JN, Fo, &kL, &kR);
            s->F_r[IR(k, N, j)] = Fo[0]; s->F_r_Hr[IR(k, N, j)] = Fo[1]; s->F_r_HZ[IR(k, N, j)] = Fo[2];
            s->K_iph[I3(k, N - 1, j)] = kL;
            s->K_imh[I3(k, N, j)] = kR;
            q = reconstruct(JN, JNp1, JNp2, JNm1, HrN, HrNp1, HrNp2, HrNm1, HZN, HZNp1, HZNp2, HZNm1,
                            g->dr_b[5], g->dr_b[6], g->dr_b[7], g->dr_b[8], g->dr_b[9], aFN, aFN);
            face_r(fm, ucNp1, &q, JN, JNp1, Fo, &kL, &kR);
            s->F_r[IR(k, N + 1, j)] = Fo[0]; s->F_r_Hr[IR(k, N + 1, j)] = Fo[1];
            s->F_r_HZ[IR(k, N + 1, j)] = Fo[2];
            s->K_iph[I3(k, N, j)] = kL;
        }
    }

    /* Z-direction, bottom interfaces, src/AdvectJandH.jl:978-1099 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nr; i++) {
        double uc0 = v->u_Z_star[i + nr * 0] * inv_c;
        double uc1 = v->u_Z_star[i + nr * 1] * inv_c;
        for (int k = k0; k <= k1; k++) {
            double J1 = J[I3(k, i, 0)], J2 = J[I3(k, i, 1)];
            double Hr1 = Hr[I3(k, i, 0)], Hr2 = Hr[I3(k, i, 1)];
            double HZ1 = HZ[I3(k, i, 0)], HZ2 = HZ[I3(k, i, 1)];
            double aF1 = aF[I3(k, i, 0)];
            double J0, HZ0, Hr0, Jm1, HZm1, Hrm1;
            if (bc_z_bot == ORC_BC_REFLECT) {
                J0 = J1; HZ0 = -HZ1; Hr0 = Hr1;
                Jm1 = J2; HZm1 = -HZ2; Hrm1 = Hr2;
            } else {
                J0 = J1; HZ0 = dmin(HZ1, 0.0); Hr0 = Hr1;
                Jm1 = J0; HZm1 = HZ0; Hrm1 = Hr0;
            }
            recon q = reconstruct(J0, J1, J2, Jm1, Hr0, Hr1, Hr2, Hrm1, HZ0, HZ1, HZ2, HZm1,
                                  g->dZ_b[0], g->dZ_b[1], g->dZ_b[2], g->dZ_b[3], g->dZ_b[4], aF1, aF1);
            double Fo[3];
            face_z(fm, uc0, &q, J0, J1, Fo);
            s->F_Z[IZ(k, i, 0)] = Fo[0]; s->F_Z_Hr[IZ(k, i, 0)] = Fo[1]; s->F_Z_HZ[IZ(k, i, 0)] = Fo[2];
            q = reconstruct(J1, J2, J[I3(k, i, 2)], J0, Hr1, Hr2, Hr[I3(k, i, 2)], Hr0, HZ1, HZ2,
                            HZ[I3(k, i, 2)], HZ0, g->dZ_L[0], g->dZ_R[0], g->inv_dZ_j_jm1[0],
                            g->inv_dZ_jp1_j[0], g->inv_dZ_jp2_jp1[0], aF1, aF[I3(k, i, 1)]);
            face_z(fm, uc1, &q, J1, J2, Fo);
            s->F_Z[IZ(k, i, 1)] = Fo[0]; s->F_Z_Hr[IZ(k, i, 1)] = Fo[1]; s->F_Z_HZ[IZ(k, i, 1)] = Fo[2];
        }
    }
    /* Z interior interfaces, src/AdvectJandH.jl:1101-1157 (1-based j = 2..N_Z-2) */
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= nz - 3; j++) {
        for (int i = 0; i < nr; i++) {
            double uc = v->u_Z_star[i + nr * (j + 1)] * inv_c;
            for (int k = k0; k <= k1; k++) {
                double Jj = J[I3(k, i, j)], Jjp1 = J[I3(k, i, j + 1)];
                recon q = reconstruct(Jj, Jjp1, J[I3(k, i, j + 2)], J[I3(k, i, j - 1)],
                                      Hr[I3(k, i, j)], Hr[I3(k, i, j + 1)], Hr[I3(k, i, j + 2)], Hr[I3(k, i, j - 1)],
                                      HZ[I3(k, i, j)], HZ[I3(k, i, j + 1)], HZ[I3(k, i, j + 2)], HZ[I3(k, i, j - 1)],
                                      g->dZ_L[j], g->dZ_R[j], g->inv_dZ_j_jm1[j], g->inv_dZ_jp1_j[j],
                                      g->inv_dZ_jp2_jp1[j], aF[I3(k, i, j)], aF[I3(k, i, j + 1)]);
                double Fo[3];
                face_z(fm, uc, &q, Jj, Jjp1, Fo);
                s->F_Z[IZ(k, i, j + 1)] = Fo[0]; s->F_Z_Hr[IZ(k, i, j + 1)] = Fo[1];
                s->F_Z_HZ[IZ(k, i, j + 1)] = Fo[2];
            }
        }
    }
    /* Z top interfaces, src/AdvectJandH.jl:1167-1289 */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nr; i++) {
        int N = nz - 1;
        double ucN = v->u_Z_star[i + nr * N] * inv_c;
        double ucNp1 = v->u_Z_star[i + nr * (N + 1)] * inv_c;
        for (int k = k0; k <= k1; k++) {
            double JN = J[I3(k, i, N)], JNm1 = J[I3(k, i, N - 1)];
            double HrN = Hr[I3(k, i, N)], HrNm1 = Hr[I3(k, i, N - 1)];
            double HZN = HZ[I3(k, i, N)], HZNm1 = HZ[I3(k, i, N - 1)];
            double aFN = aF[I3(k, i, N)];
            double JNp1, HZNp1, HrNp1, JNp2, HZNp2, HrNp2;
            if (bc_z_top == ORC_BC_REFLECT) {
                JNp1 = JN; HZNp1 = -HZN; HrNp1 = HrN;
                JNp2 = JNm1; HZNp2 = -HZNm1; HrNp2 = HrNm1;
            } else {
                JNp1 = JN; HZNp1 = dmax(HZN, 0.0); HrNp1 = HrN;
                JNp2 = JNp1; HZNp2 = HZNp1; HrNp2 = HrNp1;
            }
            recon q = reconstruct(JNm1, JN, JNp1, J[I3(k, i, N - 2)], HrNm1, HrN, HrNp1, Hr[I3(k, i, N - 2)],
                                  HZNm1, HZN, HZNp1, HZ[I3(k, i, N - 2)], g->dZ_L[N - 1], g->dZ_R[N - 1],
                                  g->inv_dZ_j_jm1[N - 1], g->inv_dZ_jp1_j[N - 1], g->inv_dZ_jp2_jp1[N - 1],
                                  aF[I3(k, i, N - 1)], aFN);
            double Fo[3];
            face_z(fm, ucN, &q, JNm1, JN, Fo);
            s->F_Z[IZ(k, i, N)] = Fo[0]; s->F_Z_Hr[IZ(k, i, N)] = Fo[1]; s->F_Z_HZ[IZ(k, i, N)] = Fo[2];
            q = reconstruct(JN, JNp1, JNp2, JNm1, HrN, HrNp1, HrNp2, HrNm1, HZN, HZNp1, HZNp2, HZNm1,
                            g->dZ_b[5], g->dZ_b[6], g->dZ_b[7], g->dZ_b[8], g->dZ_b[9], aFN, aFN);
            face_z(fm, ucNp1, &q, JN, JNp1, Fo);
            s->F_Z[IZ(k, i, N + 1)] = Fo[0]; s->F_Z_Hr[IZ(k, i, N + 1)] = Fo[1];
            s->F_Z_HZ[IZ(k, i, N + 1)] = Fo[2];
        }
    }

    /* cell update, src/AdvectJandH.jl:1302-1382 with UpdateConservativeQuantity (336-354),
     * Delta H aberration (300-312), EnforceCausalReducedFlux (478-493) */
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nz; j++) {
        for (int i = 0; i < nr; i++) {
            double ArL = g->A_r[i + (nr + 1) * j], ArR = g->A_r[(i + 1) + (nr + 1) * j];
            double AZL = g->A_Z[i + nr * j], AZR = g->A_Z[i + nr * (j + 1)];
            double idV = g->inv_dV[i + nr * j];
            size_t c = (size_t)i + (size_t)nr * j;
            double a = v->dur_dr[c], b = v->dur_dZ[c], cc = v->duZ_dr[c], d = v->duZ_dZ[c], e = v->ur_over_r[c];
            double fac = ctdt * idV;
            for (int k = k0; k <= k1; k++) {
                double Js = J[I3(k, i, j)], Hrs = Hr[I3(k, i, j)], HZs = HZ[I3(k, i, j)];
                double D[3];
                orc_D_edd(Hrs, HZs, Js, D);
                double Jn = dmax(Js - fac * ((ArR * s->F_r[IR(k, i + 1, j)] - ArL * s->F_r[IR(k, i, j)]) +
                                             (AZR * s->F_Z[IZ(k, i, j + 1)] - AZL * s->F_Z[IZ(k, i, j)])), JEPS);
                double HZn = HZs - fac * ((ArR * s->F_r_HZ[IR(k, i + 1, j)] - ArL * s->F_r_HZ[IR(k, i, j)]) +
                                          (AZR * s->F_Z_HZ[IZ(k, i, j + 1)] - AZL * s->F_Z_HZ[IZ(k, i, j)]));
                double Hrn = Hrs - fac * ((ArR * s->F_r_Hr[IR(k, i + 1, j)] - ArL * s->F_r_Hr[IR(k, i, j)]) +
                                          (AZR * s->F_Z_Hr[IZ(k, i, j + 1)] - AZL * s->F_Z_Hr[IZ(k, i, j)]));
                double DdU = d_colon_grad_u(D[0], D[2], D[1], a, b, cc, d, e);
                double Kav = 0.5 * (s->K_imh[I3(k, i, j)] + s->K_iph[I3(k, i, j)]);
                Hrn += ctdt * Kav * g->inv_r_cell[i];
                double dHr = -ctdt_c * (Hrs * a + HZs * b);
                double dHZ = -ctdt_c * (Hrs * cc + HZs * d);
                Hrn = Hrn + dHr;
                HZn = HZn + dHZ;
                Jn = dmax(Jn - ctdt_c * DdU * Js, JEPS);
                double Jc = dmax(Jn, JEPS);
                double H2 = Hrn * Hrn + HZn * HZn;
                if (H2 > Jc * Jc) {
                    double f = Jc / sqrt(H2);
                    Hrn *= f; HZn *= f;
                }
                Hr[I3(k, i, j)] = Hrn;
                HZ[I3(k, i, j)] = HZn;
                J[I3(k, i, j)] = Jn;
            }
        }
    }
    if (update_jold)
        memcpy(s->J_old, s->J, sizeof(double) * (size_t)nnu * nr * nz);
#undef IR
#undef IZ
#undef I3
}

/* AdvectLya!: src/UpdateLyaJandH.jl:107-171 */
void orc_advect_lya(orc_lya *s, const orc_geom *g, const orc_vel *v, double ctdt,
                    int bc_r_right, int bc_z_bot, int bc_z_top, int *kmin_out, int *kmax_out) {
    int kmin, kmax;
    orc_find_active_bins(s, g, &kmin, &kmax);
    orc_advect_jh(s, g, v, ctdt, 1, bc_r_right, bc_z_bot, bc_z_top, kmin, kmax);
    size_t n = (size_t)s->nnu * s->nr * s->nz;
    memcpy(s->H_r_old, s->H_r, sizeof(double) * n);
    memcpy(s->H_Z_old, s->H_Z, sizeof(double) * n);
    if (kmin_out) *kmin_out = kmin;
    if (kmax_out) *kmax_out = kmax;
}

/* LyaEmissionAbsorptionUpdate! + AbsorptionUpdateJorH:
 * src/ConstantsAndFunctions.jl:483-573, 451-462 */
void orc_emission_absorption(orc_lya *s, double c_tilde, double dt) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    const double inv_ct = 1.0 / c_tilde;
    const double fpc_ict = (FOUR_PI / C_LIGHT) * inv_ct;
    const int ncell = nr * nz;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncell; c++) {
        size_t base = (size_t)nnu * c;
        double ac = s->alpha_c[c], al = s->alpha[c], pdv = s->pd[c], js = s->js[c];
        double al_pd = al * pdv;
        double js_ct = js * c_tilde;
        for (int k = 0; k < nnu; k++) {
            size_t x = base + k;
            double aabs = ac + al_pd * s->Hvoigt[x];
            double dJdt = js_ct * s->phi_nu[x];
            s->J[x] = (s->J_old[x] + dJdt * dt) / (1.0 + aabs * c_tilde * dt);
            s->H_r_old[x] = s->H_r[x];
            s->H_Z_old[x] = s->H_Z[x];
            double aH = s->alpha_F[x];
            s->H_r[x] = (s->H_r_old[x] + 0.0 * dt) / (1.0 + aH * c_tilde * dt);
            s->H_Z[x] = (s->H_Z_old[x] + 0.0 * dt) / (1.0 + aH * c_tilde * dt);
        }
        double sr = 0.0, sz = 0.0;
        for (int k = 0; k < nnu; k++) {
            size_t x = base + k;
            sr += s->dnu[k] * (s->H_r_old[x] - s->H_r[x]);
            sz += s->dnu[k] * (s->H_Z_old[x] - s->H_Z[x]);
        }
        s->dru_r[c] += fpc_ict * sr;
        s->dru_Z[c] += fpc_ict * sz;
        for (int k = 0; k < nnu; k++) {
            size_t x = base + k;
            s->J_old[x] = s->J[x];
            s->H_r_old[x] = s->H_r[x];
            s->H_Z_old[x] = s->H_Z[x];
        }
    }
}

/* OneMinusphi_L_and_chi_L / OneMinusphi_R_and_chi_R: src/FreqFactors.jl:54-133 */
static void omphi_L(double P, double *omp, double *chi) {
    if (P >= PMAX) { *omp = exp(-PMAX); *chi = (1.0 - exp(-PMAX)) / PMAX; return; }
    if (P <= -PMAX) { *omp = exp(PMAX); *chi = (1.0 - exp(PMAX)) / (-PMAX); return; }
    if (fabs(P) < PMIN) { *omp = 1.0 - P + 0.5 * (P * P); *chi = 1.0 - 0.5 * P; return; }
    double e = exp(-P);
    *omp = e; *chi = (1.0 - e) / P;
}
static void omphi_R(double P, double *omp, double *chi) {
    if (P >= PMAX) { *omp = exp(PMAX); *chi = (1.0 - exp(PMAX)) / PMAX; return; }
    if (P <= -PMAX) { *omp = exp(-PMAX); *chi = (1.0 - exp(-PMAX)) / (-PMAX); return; }
    if (fabs(P) < PMIN) { *omp = 1.0 + P + 0.5 * (P * P); *chi = -1.0 - 0.5 * P; return; }
    double e = exp(P);
    *omp = e; *chi = (1.0 - e) / P;
}

double orc_compute_b(double T) { return sqrt(2.0 * K_BOLTZ / M_H) * sqrt(T); }
double orc_compute_dnuD(double T) { return orc_compute_b(T) * (NU_LYA / C_LIGHT); }
double orc_compute_a(double T) {
    return (A_LYA / (FOUR_PI * NU_LYA * 1.0 / C_LIGHT)) / orc_compute_b(T);
}
double orc_compute_sigma0(double T) {
    return (sqrt(M_PI) * (E_CHARGE * E_CHARGE) * F_LU_LYA / (M_ELEC * NU_LYA)) / orc_compute_b(T);
}

/* UpdateFreqFactors!: src/FreqFactors.jl:142-278 */
void orc_update_freq_factors(orc_lya *s, const orc_vel *v) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    const int ncell = nr * nz;
    const double h_kB = H_PLANCK / K_BOLTZ;
    const double inv_c = 1.0 / C_LIGHT;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncell; c++) {
        size_t base = (size_t)nnu * c;
        double dnuD = orc_compute_dnuD(s->T[c]);
        double pref = 0.5 * dmax(s->alpha[c], s->alpha_floor) * (dnuD * dnuD);
        double rec0 = h_kB / s->T[c];
        double a = v->dur_dr[c], b = v->dur_dZ[c], cc = v->duZ_dr[c], d = v->duZ_dZ[c], e = v->ur_over_r[c];
        for (int k = 1; k <= nnu - 2; k++) {
            double nC_k = s->nuC[k], nC_kp = s->nuC[k + 1], nC_km = s->nuC[k - 1];
            double dn_kp = nC_kp - s->nu[k + 1];
            double dn_k = s->nu[k + 1] - nC_k;
            double dn_km = s->nu[k] - nC_km;
            double iDnu = s->inv_dnu[k];
            double iC_k = s->inv_nuC[k], iC_kp = s->inv_nuC[k + 1], iC_km = s->inv_nuC[k - 1];
            double D[3];
            orc_D_edd(s->H_r[base + k], s->H_Z[base + k], s->J[base + k], D);
            double vel = d_colon_grad_u(D[0], D[2], D[1], a, b, cc, d, e) * inv_c;
            double Kkp = pref * s->Hvoigt[base + k + 1];
            double Kk = pref * s->Hvoigt[base + k];
            double Kkm = pref * s->Hvoigt[base + k - 1];
            double Ckp = vel * nC_kp, Ck = vel * nC_k, Ckm = vel * nC_km;
            if (s->recoil) {
                Ckp += Kkp * (rec0 - 2.0 * iC_kp);
                Ck += Kk * (rec0 - 2.0 * iC_k);
                Ckm += Kkm * (rec0 - 2.0 * iC_km);
            }
            double r_kp = dn_kp * (1.0 / Kkp);
            double r_k = dn_k * (1.0 / Kk);
            double r_km = dn_km * (1.0 / Kkm);
            double Pkp = dclamp(Ckp * r_kp, -PMAX, PMAX);
            double Pk = dclamp(Ck * r_k, -PMAX, PMAX);
            double Pkm = dclamp(Ckm * r_km, -PMAX, PMAX);
            double oR_kp, xR_kp, oL_k, xL_k, oR_k, xR_k, oL_km, xL_km;
            omphi_R(Pkp, &oR_kp, &xR_kp);
            omphi_L(Pk, &oL_k, &xL_k);
            omphi_R(Pk, &oR_k, &xR_k);
            omphi_L(Pkm, &oL_km, &xL_km);
            double den_kp = iDnu * (1.0 / (xL_k * r_k - xR_kp * r_kp));
            s->Fkp[base + k] = oR_kp * den_kp;
            double den_km = iDnu * (1.0 / (xL_km * r_km - xR_k * r_k));
            s->Fkm[base + k] = oL_km * den_km;
            s->Fk[base + k] = oL_k * den_kp + oR_k * den_km;
        }
    }
}

/* LAPACK dgtsv, one right-hand side: Gaussian elimination with partial pivoting of a
 * tridiagonal matrix, followed by back substitution (the published LAPACK algorithm,
 * called by src/TridiagonalSolver.jl:54). Returns INFO; *npiv counts interchanges. */
static int dgtsv_count(int n, double *dl, double *d, double *du, double *b, long *npiv) {
    if (n <= 0) return 0;
    for (int i = 0; i < n - 2; i++) {
        if (fabs(d[i]) >= fabs(dl[i])) {
            if (d[i] != 0.0) {
                double fact = dl[i] / d[i];
                d[i + 1] = d[i + 1] - fact * du[i];
                b[i + 1] = b[i + 1] - fact * b[i];
            } else {
                return i + 1;
            }
            dl[i] = 0.0;
        } else {
            double fact = d[i] / dl[i];
            d[i] = dl[i];
            double temp = d[i + 1];
            d[i + 1] = du[i] - fact * temp;
            dl[i] = du[i + 1];
            du[i + 1] = -fact * dl[i];
            du[i] = temp;
            temp = b[i];
            b[i] = b[i + 1];
            b[i + 1] = temp - fact * b[i + 1];
            if (npiv) (*npiv)++;
        }
    }
    if (n > 1) {
        int i = n - 2;
        if (fabs(d[i]) >= fabs(dl[i])) {
            if (d[i] != 0.0) {
                double fact = dl[i] / d[i];
                d[i + 1] = d[i + 1] - fact * du[i];
                b[i + 1] = b[i + 1] - fact * b[i];
            } else {
                return i + 1;
            }
        } else {
            double fact = d[i] / dl[i];
            d[i] = dl[i];
            double temp = d[i + 1];
            d[i + 1] = du[i] - fact * temp;
            du[i] = temp;
            temp = b[i];
            b[i] = b[i + 1];
            b[i + 1] = temp - fact * b[i + 1];
            if (npiv) (*npiv)++;
        }
    }
    if (d[n - 1] == 0.0) return n;
    b[n - 1] = b[n - 1] / d[n - 1];
    if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
    for (int i = n - 3; i >= 0; i--)
        b[i] = (b[i] - du[i] * b[i + 1] - dl[i] * b[i + 2]) / d[i];
    return 0;
}
int orc_dgtsv(int n, double *dl, double *d, double *du, double *b) {
    return dgtsv_count(n, dl, d, du, b, NULL);
}

/* FrequencyUpdateJLya_AllCells!: src/UpdateLyaJandH.jl:231-391, with
 * FrequencyUpdateJLya! (178-227) and TridiagonalSolve (src/TridiagonalSolver.jl:33-58) */
int orc_frequency_update_all_cells(orc_lya *s, const orc_vel *v, double ctdt, int update_ff,
                                   long *n_pivots) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    const int ncell = nr * nz;
    const double dw = 1.0 / ctdt;
    if (update_ff) orc_update_freq_factors(s, v);
    const int n = nnu - 2;
    int nfail = 0;
    long npiv = 0;
#pragma omp parallel reduction(+ : nfail, npiv)
    {
        double *A = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * 5);
        double *B = A + n, *C = B + n, *dl = C + n, *x = dl + n;
#pragma omp for schedule(static)
        for (int c = 0; c < ncell; c++) {
            size_t base = (size_t)nnu * c;
            for (int row = 0; row < n; row++) {
                int k = row + 1;
                A[row] = s->Fkm[base + k];
                B[row] = -(s->Fk[base + k] + dw);
                C[row] = s->Fkp[base + k];
                x[row] = -dw * s->J_old[base + k];
            }
            /* dl <- A[2:end], du <- C[1:end-1] (TridiagonalSolver.jl:45-46) */
            for (int r = 0; r < n - 1; r++) dl[r] = A[r + 1];
            long p = 0;
            int info = dgtsv_count(n, dl, B, C, x, &p);
            npiv += p;
            if (info != 0) { nfail++; continue; }
            for (int row = 0; row < n; row++) s->J[base + row + 1] = x[row];
        }
        free(A);
    }
    /* flux correction, src/UpdateLyaJandH.jl:335-379 */
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncell; c++) {
        size_t base = (size_t)nnu * c;
        for (int k = 0; k < nnu; k++) {
            size_t x = base + k;
            double Jk = dmax(s->J[x], JEPS);
            s->J[x] = Jk;
            double hr = s->H_r[x], hz = s->H_Z[x];
            double ratio = Jk * (1.0 / dmax(s->J_old[x], JEPS));
            hr = hr * ratio;
            hz = hz * ratio;
            double H2 = hr * hr + hz * hz;
            if (H2 > Jk * Jk) {
                double f = Jk / sqrt(H2);
                hr = hr * f; hz = hz * f;
            }
            s->H_r[x] = hr; s->H_Z[x] = hz;
            s->J_old[x] = Jk;
            s->H_r_old[x] = hr; s->H_Z_old[x] = hz;
        }
    }
    if (n_pivots) *n_pivots = npiv;
    return nfail;
}

/* Update_f_Lya_MF_L_Lya!: src/ConstantsAndFunctions.jl:588-674 */
void orc_update_f_mf(orc_lya *s, const orc_geom *g, double dt, double z_center, int bc_z_bot,
                     double out[4]) {
    const int nr = s->nr, nz = s->nz;
    double inv_dt = 1.0 / dt;
    for (int c = 0; c < nr * nz; c++) {
        s->f_r[c] = s->dru_r[c] * inv_dt;
        s->f_Z[c] = s->dru_Z[c] * inv_dt;
    }
    double MF = 0.0, L = 0.0;
    for (int j = 0; j < nz; j++)
        for (int i = 0; i < nr; i++) {
            int c = i + nr * j;
            MF += g->dV[c] * sqrt(s->f_r[c] * s->f_r[c] + s->f_Z[c] * s->f_Z[c]);
            L += FOUR_PI * g->dV[c] * s->js[c];
        }
    double net = 0.0, outw = 0.0;
    for (int j = 0; j < nz; j++)
        for (int i = 0; i < nr; i++) {
            int c = i + nr * j;
            double dr = g->rCoM[i], dz = g->ZCoM[j] - z_center;
            double dist = sqrt(dr * dr + dz * dz);
            double frad;
            if (dist > 0.0) {
                double id = 1.0 / dist;
                frad = s->f_r[c] * (dr * id) + s->f_Z[c] * (dz * id);
            } else {
                frad = 0.0;
            }
            net += g->dV[c] * frad;
            outw += g->dV[c] * dmax(frad, 0.0);
        }
    if (L > 0.0) {
        double k = 1.0 / (L / C_LIGHT);
        MF *= k; net *= k; outw *= k;
    } else {
        MF = 0.0; net = 0.0; outw = 0.0;
    }
    out[0] = MF; out[1] = net; out[2] = outw;
    out[3] = (bc_z_bot == ORC_BC_REFLECT) ? 2.0 * L : L;
}

/* Update_f_Lya_MF_L_Lya! with gravity, src/ConstantsAndFunctions.jl:691-804: the same f and
 * M_F family plus M_F_antigravity = sum dV (-f . g_hat) / (L/c) (zero where g = 0).
 * out = {M_F, M_F_antigravity, M_F_radial_net, M_F_radial_out, L_tot}. */
void orc_update_f_mf_gravity(orc_lya *s, const orc_geom *g, double dt, const double *fg_r, const double *fg_Z,
                             double z_center, int bc_z_bot, double out[5]) {
    double base[4];
    orc_update_f_mf(s, g, dt, z_center, bc_z_bot, base);
    const int nr = s->nr, nz = s->nz;
    double L = 0.0, anti = 0.0;
    for (int j = 0; j < nz; j++)
        for (int i = 0; i < nr; i++) {
            int c = i + nr * j;
            L += FOUR_PI * g->dV[c] * s->js[c];
            double gm = sqrt(fg_r[c] * fg_r[c] + fg_Z[c] * fg_Z[c]);
            double fa = gm > 0.0 ? -(s->f_r[c] * fg_r[c] + s->f_Z[c] * fg_Z[c]) / gm : 0.0;
            anti += g->dV[c] * fa;
        }
    anti = L > 0.0 ? anti * (1.0 / (L / C_LIGHT)) : 0.0;
    out[0] = base[0]; out[1] = anti; out[2] = base[1]; out[3] = base[2]; out[4] = base[3];
}

/* Compute_f_esc_Lya_Cylindrical + Compute_f_esc_Cylindrical:
 * src/ConstantsAndFunctions.jl:969-993, 914-961 */
double orc_f_esc_lya(const orc_lya *s, const orc_geom *g, double L_all, int bc_z_bot) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    if (L_all <= 0.0) return 0.0;
    double Lsim = (bc_z_bot == ORC_BC_REFLECT) ? 0.5 * L_all : L_all;
    double fesc = 0.0;
    for (int k = 0; k < nnu; k++) {
        double Lesc = 0.0;
        for (int j = 0; j < nz; j++)
            Lesc += g->A_r[nr + (nr + 1) * j] * FOUR_PI * dmax(s->H_r[ix3(nnu, nr, k, nr - 1, j)], 0.0);
        for (int i = 0; i < nr; i++)
            Lesc += g->A_Z[i + nr * nz] * FOUR_PI * dmax(s->H_Z[ix3(nnu, nr, k, i, nz - 1)], 0.0);
        if (bc_z_bot == ORC_BC_OUTFLOW)
            for (int i = 0; i < nr; i++)
                Lesc += g->A_Z[i] * FOUR_PI * dmax(-s->H_Z[ix3(nnu, nr, k, i, 0)], 0.0);
        double f = (Lsim > 0.0) ? Lesc / Lsim : 0.0;
        fesc += s->dnu[k] * f;
    }
    return fesc;
}

/* Reset_Delta_rho_u!: src/ConstantsAndFunctions.jl:809-816 */
void orc_reset_dru(orc_lya *s) {
    memset(s->dru_r, 0, sizeof(double) * (size_t)s->nr * s->nz);
    memset(s->dru_Z, 0, sizeof(double) * (size_t)s->nr * s->nz);
}

/* GetRHDCFLTimeStep: src/AdvectJandH.jl:29-68 */
double orc_cfl_dt(const orc_geom *g, double c_tilde, const double *u_r, const double *u_Z, double cfl) {
    double m = INFINITY;
    for (int j = 0; j < g->nz; j++) {
        double dZ = g->Z[j + 1] - g->Z[j];
        for (int i = 0; i < g->nr; i++) {
            double dr = g->r[i + 1] - g->r[i];
            double u = hypot(u_r[i + g->nr * j], u_Z[i + g->nr * j]);
            double dt = 0.5 * dmin(dr, dZ) / (c_tilde + u);
            if (dt < m) m = dt;
        }
    }
    return cfl * m;
}

/* pd_Lya: src/LymanAlphaDestruction.jl:43-97 */
double orc_pd_lya(double nHII, double ne, double nHI, double nHeI, double nH2, double T, double z) {
    T = dclamp(T, 1.0, 1e5);
    double T100 = T / 100.0;
    double lT = log10(T);
    double lT2 = lT * lT, lT3 = lT2 * lT, lT4 = lT3 * lT;
    double G_p2s = 3.1e-6 * (1.0 + z);
    double G_s2p = 3.0 * G_p2s;
    double r25 = 2.5 / T;
    double C_e = 5e-5 * exp(-(r25 * r25)) * ne / (1.0 + pow(T100, 0.45));
    double C_HII = (6.98e-3 * (1.0 + 0.933 * lT) * exp(-pow(601.0 / T, 0.406)) / pow(T, 0.5) +
                    pow(10.0, -7.69 + 1.21 * lT + 0.455 * lT2 - 0.199 * lT3 + 0.0182 * lT4)) * nHII;
    double C_HeI = 2.6e-9 * pow(T100, 0.315) * nHeI;
    double C_H2 = 1.7e-9 * pow(T100, 0.3) * nH2;
    double den = 8.9 * pow(T, -0.55) + 0.078 * pow(T, 0.35);
    double C_HI = (4.1e-11 * exp(-pow(1.6 / T, 0.75) - 0.15 * T) +
                   (1.6e-10 + 1.57e-12 * pow(T, 1.1)) / (den * den)) * nHI;
    double C_s2p = C_e + C_HII + C_HeI + C_H2 + C_HI;
    double C_p2s = ONE_THIRD * C_s2p;
    double R_p2s = TWO_THIRDS * A_2P2S + C_p2s + G_p2s;
    double R_s2p = A_2S2P + C_s2p + G_s2p;
    double pd_HI = R_p2s / ((A_LYA / A_2GAM) * (A_2GAM + R_s2p) + R_p2s);
    double pd_H2;
    if (nHI > 1e-20) {
        double num = 33.0 * exp(-14540.0 / T) + 13.0 * exp(-15564.0 / T);
        double dd = 46.0 + 1e3 * exp(-pow(1e3 / T, 1.5));
        pd_H2 = dmin(num / dd, 1.3e-3) * (nH2 / nHI);
    } else {
        pd_H2 = 0.0;
    }
    return dmin(pd_HI + pd_H2, 1.0);
}

/* EvaluateLUT: src/FastInterpolations.jl:83-112 */
static double lut_eval(const orc_voigt_lut *L, const double *y, double x) {
    double xt = (x - L->xmin) * L->inv_dx;
    long i = (long)floor(xt);
    if (i + 2 > L->nx) i = L->nx - 2;
    double dx = (double)(i + 1) - xt;
    return dx * y[i] + (1.0 - dx) * y[i + 1];
}
/* DawsonFast/ErfFast/GaussianFast/xGaussianFast/OneMinusx2GaussianFast:
 * src/FastInterpolations.jl:202-275 */
static double dawson_fast(const orc_voigt_lut *L, double x) {
    if (fabs(x) >= L->xmax) { double ix = 1.0 / x; double ix3 = ix * ix * ix; return 0.5 * ix + 0.25 * ix3; }
    return lut_eval(L, L->dawson_y, x);
}
static double erf_fast(const orc_voigt_lut *L, double x) {
    if (fabs(x) >= L->xmax) return copysign(1.0, x);
    return lut_eval(L, L->erf_y, x);
}
static double gauss_fast(const orc_voigt_lut *L, double x) {
    return fabs(x) >= L->xmax ? 0.0 : lut_eval(L, L->gauss_y, x);
}
static double xgauss_fast(const orc_voigt_lut *L, double x) {
    return fabs(x) >= L->xmax ? 0.0 : lut_eval(L, L->xgauss_y, x);
}
static double omx2gauss_fast(const orc_voigt_lut *L, double x) {
    return fabs(x) >= L->xmax ? 0.0 : lut_eval(L, L->omx2gauss_y, x);
}

/* H(x,a): src/ConstantsAndFunctions.jl:227-239 */
double orc_voigt_H(const orc_voigt_lut *L, double x, double a) {
    const double inv_sqrtpi_2 = 1.0 / (sqrt(M_PI) / 2.0);
    return gauss_fast(L, x) + inv_sqrtpi_2 * a * (2.0 * x * dawson_fast(L, x) - 1.0) +
           (a * a) * omx2gauss_fast(L, x);
}
/* int_0^x H dx: src/ConstantsAndFunctions.jl:246-256 */
double orc_voigt_intH(const orc_voigt_lut *L, double x, double a) {
    const double sqrtpi_2 = sqrt(M_PI) / 2.0;
    const double inv_sqrtpi_2 = 1.0 / sqrtpi_2;
    return sqrtpi_2 * erf_fast(L, x) - inv_sqrtpi_2 * a * dawson_fast(L, x) + (a * a) * xgauss_fast(L, x);
}
/* Htophat: src/ConstantsAndFunctions.jl:265-279 */
double orc_voigt_tophat(const orc_voigt_lut *L, double x, double xmax, double xmin, double a) {
    double dx = xmax - xmin;
    if (dx > 1e-5) return (orc_voigt_intH(L, xmax, a) - orc_voigt_intH(L, xmin, a)) / dx;
    return orc_voigt_H(L, x, a);
}
/* UpdateVoigtAndEmissionProfile! (a, inv dnuD) + Update_Hvoigt!:
 * src/FreqFactors.jl:24-51, src/ConstantsAndFunctions.jl:319-357 */
void orc_update_hvoigt(const orc_voigt_lut *L, orc_lya *s) {
    const int nnu = s->nnu, ncell = s->nr * s->nz;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncell; c++) {
        double a = orc_compute_a(s->T[c]);
        double inv_dnuD = 1.0 / orc_compute_dnuD(s->T[c]);
        for (int k = 0; k < nnu; k++) {
            double x = (s->nuC[k] - NU_LYA) * inv_dnuD;
            double xmax = (s->nu[k + 1] - NU_LYA) * inv_dnuD;
            double xmin = (s->nu[k] - NU_LYA) * inv_dnuD;
            s->Hvoigt[(size_t)nnu * c + k] = orc_voigt_tophat(L, x, xmax, xmin, a);
        }
    }
}
/* Update_phi_nu!: src/ConstantsAndFunctions.jl:362-393 */
void orc_update_phi_nu(orc_lya *s, int kmin, int kmax) {
    const int nnu = s->nnu, ncell = s->nr * s->nz;
    for (int c = 0; c < ncell; c++) {
        size_t base = (size_t)nnu * c;
        double sum = 0.0;
        for (int k = kmin; k <= kmax; k++) sum += s->dnu[k] * s->Hvoigt[base + k];
        double inv = 1.0 / sum;
        for (int k = kmin; k <= kmax; k++) s->phi_nu[base + k] = s->Hvoigt[base + k] * inv;
    }
}

/* edge ring: src/SaveHDF5Data_StaticCloudTests.jl:152-199 (indices), 392-420 (spectra) */
int orc_edge_count(int nr, int nz) { return (nz - 2) + 2 * (nr - 3); }
void orc_edge_spectra(const orc_lya *s, double *out_raw, double *out_norm, int *ridx, int *zidx) {
    const int nnu = s->nnu, nr = s->nr, nz = s->nz;
    int e = 0;
    for (int j = 1; j <= nz - 2; j++) { ridx[e] = nr - 2; zidx[e] = j; e++; }
    for (int i = 1; i <= nr - 3; i++) { ridx[e] = i; zidx[e] = nz - 2; e++; }
    for (int i = 1; i <= nr - 3; i++) { ridx[e] = i; zidx[e] = 1; e++; }
    for (int q = 0; q < e; q++) {
        const double *Jc = s->J + ix3(nnu, nr, 0, ridx[q], zidx[q]);
        double integ = 0.0;
        for (int k = 0; k < nnu; k++) integ += Jc[k] * s->dnu[k];
        for (int k = 0; k < nnu; k++) {
            out_raw[(size_t)q * nnu + k] = Jc[k];
            out_norm[(size_t)q * nnu + k] = integ > 0.0 ? Jc[k] / integ : Jc[k];
        }
    }
}

/* One step of the static-cloud driver loop: src/StaticCloudTest.jl:357-392 */
void orc_static_step(orc_lya *s, const orc_geom *g, const orc_vel *v, double c_tilde, double dt,
                     double z_center, int bc_r_right, int bc_z_bot, int bc_z_top, double diag[7]) {
    double ctdt = c_tilde * dt;
    int kmin, kmax;
    orc_advect_lya(s, g, v, ctdt, bc_r_right, bc_z_bot, bc_z_top, &kmin, &kmax);
    orc_emission_absorption(s, c_tilde, dt);
    orc_frequency_update_all_cells(s, v, ctdt, 1, NULL);
    double mf[4];
    orc_update_f_mf(s, g, dt, z_center, bc_z_bot, mf);
    double fesc = orc_f_esc_lya(s, g, mf[3], bc_z_bot);
    orc_reset_dru(s);
    diag[0] = mf[0]; diag[1] = mf[1]; diag[2] = mf[2]; diag[3] = mf[3];
    diag[4] = fesc; diag[5] = (double)kmin; diag[6] = (double)kmax;
}

void orc_static_run(orc_lya *s, const orc_geom *g, const orc_vel *v, double c_tilde, double dt,
                    double z_center, int bc_r_right, int bc_z_bot, int bc_z_top, int n_steps,
                    double *diag_hist) {
    double scratch[7];
    for (int n = 0; n < n_steps; n++)
        orc_static_step(s, g, v, c_tilde, dt, z_center, bc_r_right, bc_z_bot, bc_z_top,
                        diag_hist ? diag_hist + 7 * (size_t)n : scratch);
}
