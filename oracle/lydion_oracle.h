/*
 * lydion_oracle.h -- CPU FP64 restatement of LYDION's multi-frequency Lyman-alpha
 * M1 transport step, used ONLY as test infrastructure (the checker of the CUDA
 * path, and the CPU baseline timed beside it). Nothing in the product library links
 * or calls this code.
 *
 * PARITY STATUS: partially pinned.
 *   - The reference is Julia; no Julia toolchain exists on the build or GPU hosts, so
 *     the reference itself cannot be run and no J/H golden vectors exist anywhere in
 *     the reference tree. The step as a whole is therefore "parity unpinned": this
 *     file restates the reference algorithm function by function (citations below are
 *     paths inside the LYDION source tree), and the CUDA kernels are checked against it.
 *   - Two third-party pieces on the path ARE pinned by committed fixtures:
 *       * LAPACK dgtsv (called by src/TridiagonalSolver.jl:54) -- orc_dgtsv is checked
 *         against scipy.linalg.lapack.dgtsv outputs (tests/golden/dgtsv_cases.npz);
 *       * SpecialFunctions erf/dawson feeding the Voigt look-up tables
 *         (src/FastInterpolations.jl:178-197) -- the tables are built from
 *         scipy.special.erf / scipy.special.dawsn (tests/golden/voigt_*.npz).
 *
 * Layout: every (frequency, r, Z) array is Julia column-major [k,i,j], i.e. in C
 * index k + n_nu*(i + n_r*j) with k fastest. Per-cell arrays are [i,j] -> i + n_r*j.
 * Face arrays in r are (n_nu, n_r+1, n_z); in Z (n_nu, n_r, n_z+1).
 * All indices in this API are 0-based (the reference is 1-based).
 */
#ifndef LYDION_ORACLE_H
#define LYDION_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_BC_REFLECT = 0, ORC_BC_OUTFLOW = 1 };
enum { ORC_FLUX_GLF = 0, ORC_FLUX_HLL = 1 };

/* Cylindrical geometry, mirrors the fields of GeometryCylindrical used by the
 * Lyman-alpha path (src/Structs.jl, filled by src/SpatialGrid.jl:606-913). */
typedef struct orc_geom {
    int nr, nz;
    const double *r, *Z;              /* interfaces, nr+1 / nz+1               */
    const double *rCoM, *ZCoM;        /* cell centroids, nr / nz               */
    const double *dV, *inv_dV;        /* nr*nz                                 */
    const double *A_r;                /* (nr+1)*nz                             */
    const double *A_Z;                /* nr*(nz+1)                             */
    const double *inv_r_cell;         /* nr, <1/r>                             */
    /* PLM intervals along r (src/SpatialGrid.jl:516-586), arrays of length nr   */
    const double *dr_L, *dr_R, *inv_dr_i_im1, *inv_dr_ip1_i, *inv_dr_ip2_ip1;
    /* boundary intervals: [0..4] inner (L, R, i_im1, ip1_i, ip2_ip1), [5..9] outer */
    double dr_b[10];
    const double *dZ_L, *dZ_R, *inv_dZ_j_jm1, *inv_dZ_jp1_j, *inv_dZ_jp2_jp1;
    double dZ_b[10];
    /* boundary at the first r interface: ORC_BC_REFLECT (the axis of a cylindrical grid) or,
     * on a Cartesian grid (inv_r_cell = 0, u_r/r = 0; src/AdvectJandH.jl:1396-2222),
     * ORC_BC_OUTFLOW */
    int bc_r_left;
} orc_geom;

/* The Lyman-alpha state, mirrors LyaArrays{FluxMethod} (src/Structs.jl:23-124). */
typedef struct orc_lya {
    int nnu, nr, nz;
    double *J, *J_old, *H_r, *H_Z, *H_r_old, *H_Z_old;    /* nnu*nr*nz          */
    double *alpha_F, *Hvoigt, *phi_nu;                    /* nnu*nr*nz          */
    double *alpha, *alpha_c, *pd, *js;                    /* nr*nz              */
    double *T;                                            /* nr*nz (gas temp)   */
    double *dru_r, *dru_Z, *f_r, *f_Z;                    /* nr*nz              */
    const double *nu;                                     /* nnu+1 interfaces   */
    const double *nuC, *dnu, *inv_dnu, *inv_nuC;          /* nnu                */
    int kcore_min, kcore_max;                             /* 0-based, inclusive */
    int recoil;
    int flux_method;
    double alpha_floor;
    /* scratch the reference keeps in LyaArrays: face fluxes, K_phiphi, F+/F/F- */
    double *F_r, *F_Z, *F_r_Hr, *F_Z_Hr, *F_r_HZ, *F_Z_HZ;
    double *K_iph, *K_imh;
    double *Fkp, *Fk, *Fkm;
} orc_lya;

/* Gas velocity field (cylindrical). */
typedef struct orc_vel {
    const double *u_r_star;   /* (nr+1)*nz */
    const double *u_Z_star;   /* nr*(nz+1) */
    const double *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;  /* nr*nz */
} orc_vel;

/* --- elementary functions (exposed for unit tests) ---------------------------- */
double orc_minmod(double a, double b);
double orc_chi_L84(double f);
void   orc_D_edd(double Hr, double HZ, double J, double out[3]);
void   orc_D_edd_from_f_n(double f, double nr, double nZ, double out[3]);
void   orc_hll_eigenvalues(double f, double mu, double out[2]);
/* LAPACK dgtsv for one right-hand side. dl, du have length n-1; d, b length n.
 * Returns LAPACK's INFO (0 on success, i>0 if U(i,i) is exactly zero). */
int    orc_dgtsv(int n, double *dl, double *d, double *du, double *b);
double orc_pd_lya(double nHII, double ne, double nHI, double nHeI, double nH2, double T, double z);
double orc_compute_b(double T);
double orc_compute_dnuD(double T);
double orc_compute_a(double T);
double orc_compute_sigma0(double T);

/* Voigt look-up tables (src/FastInterpolations.jl:54-112, 178-275). The five tables
 * (erf, dawson, exp(-x^2), x exp(-x^2), (1-2x^2) exp(-x^2)) are tabulated by the caller
 * on the grid x_i = xmin + i*dx, i = 0..nx-1. */
typedef struct orc_voigt_lut {
    double xmax, xmin, inv_dx;
    int nx;
    const double *erf_y, *dawson_y, *gauss_y, *xgauss_y, *omx2gauss_y;
} orc_voigt_lut;
double orc_voigt_H(const orc_voigt_lut *L, double x, double a);
double orc_voigt_intH(const orc_voigt_lut *L, double x, double a);
double orc_voigt_tophat(const orc_voigt_lut *L, double x, double xmax, double xmin, double a);
void   orc_update_hvoigt(const orc_voigt_lut *L, orc_lya *s);
void   orc_update_phi_nu(orc_lya *s, int kmin, int kmax);

/* --- the step ------------------------------------------------------------------ */
void   orc_find_active_bins(const orc_lya *s, const orc_geom *g, int *kmin, int *kmax);
void   orc_advect_jh(orc_lya *s, const orc_geom *g, const orc_vel *v,
                     double ctdt, int update_jold, int bc_r_right, int bc_z_bot, int bc_z_top,
                     int kmin, int kmax);
void   orc_advect_lya(orc_lya *s, const orc_geom *g, const orc_vel *v, double ctdt,
                      int bc_r_right, int bc_z_bot, int bc_z_top, int *kmin_out, int *kmax_out);
void   orc_emission_absorption(orc_lya *s, double c_tilde, double dt);
void   orc_update_freq_factors(orc_lya *s, const orc_vel *v);
/* returns the number of cells whose tridiagonal solve reported INFO != 0 and, in
 * *n_pivots, the number of row interchanges dgtsv performed over all cells */
int    orc_frequency_update_all_cells(orc_lya *s, const orc_vel *v, double ctdt,
                                      int update_freq_factors, long *n_pivots);
/* Update_f_Lya_MF_L_Lya!: out = {M_F, M_F_radial_net, M_F_radial_out, L_tot} */
void   orc_update_f_mf(orc_lya *s, const orc_geom *g, double dt, double z_center,
                       int bc_z_bot, double out[4]);
void   orc_update_f_mf_gravity(orc_lya *s, const orc_geom *g, double dt, const double *fg_r, const double *fg_Z,
                               double z_center, int bc_z_bot, double out[5]);
double orc_f_esc_lya(const orc_lya *s, const orc_geom *g, double L_allspace, int bc_z_bot);
void   orc_reset_dru(orc_lya *s);
double orc_cfl_dt(const orc_geom *g, double c_tilde, const double *u_r, const double *u_Z,
                  double cfl);
/* edge ring of the static-cloud output (src/SaveHDF5Data_StaticCloudTests.jl:152-199,
 * 392-420). n_edge = (nz-2) + 2*(nr-3). out_raw/out_norm are (n_edge, nnu) row-major. */
int    orc_edge_count(int nr, int nz);
void   orc_edge_spectra(const orc_lya *s, double *out_raw, double *out_norm, int *ridx, int *zidx);

/* One full static-cloud step in the driver's order (src/StaticCloudTest.jl:357-392).
 * diag = {M_F, M_F_radial_net, M_F_radial_out, L_tot, f_esc, kmin, kmax}. */
void   orc_static_step(orc_lya *s, const orc_geom *g, const orc_vel *v, double c_tilde,
                       double dt, double z_center, int bc_r_right, int bc_z_bot, int bc_z_top,
                       double diag[7]);
void   orc_static_run(orc_lya *s, const orc_geom *g, const orc_vel *v, double c_tilde,
                      double dt, double z_center, int bc_r_right, int bc_z_bot, int bc_z_top,
                      int n_steps, double *diag_hist /* n_steps*7 */);

/* RHD-side Lyman-alpha block (lydion_oracle_rhd.c) */
typedef struct orc_dust_lya {
    double kappa_abs[3], kappa_F[3];   /* Sil, C, PAH (cm^2 g^-1) */
    double rho_ignore;                 /* dust densities at or below this are ignored */
} orc_dust_lya;
double orc_prob_lya_sh95(double T, double ne, int caseB);
double orc_krec_hii(double T, int ots);
double orc_js_rec_lya(double T, double nHII, double ne, int ots);
double orc_js_coll_lya(double T, double nHI, double ne);
void   orc_rhd_lya_prepare_cell(const double sp[11], const orc_dust_lya *d, double z, int ots, int destruction,
                                double out[8]);
int    orc_rhd_lya_absorb_cell(int nnu, const double *dnu, const double *Hv, const double *phi, const double *J_old,
                               const double *Hr_old, const double *HZ_old, double *J, double *Hr, double *HZ,
                               const double cell[8], double dt, double c_tilde, double e_old, double jeps,
                               double out[13]);

double orc_find_rsl_lya(int nr, int nz, const double *r, const double *Z, const double *u_r, const double *u_Z,
                        const double *P, const double *rho, const double *gamma_ad, const double *T,
                        const double *xHII, const double *xH2, const double *rho_d, const double *pd,
                        const double kappa_abs[3], double eps_rsl, double X_over_mH, double ct_old,
                        double ct_min);

int    orc_num_threads(void);
void   orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
