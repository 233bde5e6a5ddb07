/*
 * lydion_m1.h -- C ABI of the B200 Lyman-alpha M1 transport step.
 *
 * One context holds one (frequency x r x Z) Lyman-alpha state on one GPU, in the memory
 * order of the Julia LyaArrays: a field F[k, i, j] (column-major, k fastest) is the flat
 * array F[k + n_nu*(i + n_r*j)]; per-cell arrays are [i + n_r*j]; r-face arrays are
 * [f + (n_r+1)*j], Z-face arrays [i + n_r*f]. All host pointers are borrowed for the
 * duration of the call; device memory is owned by the context. Indices are 0-based.
 *
 * Every entry point returns LYD_OK (0) or a negative status; lyd_last_error() returns a
 * description of the last failure on that context. A context is not re-entrant: calls on
 * one context must come from one host thread at a time. Work is issued on the context's
 * own CUDA stream; lyd_download* and the diagnostic calls return after the stream drains.
 *
 * Each step entry point names the Julia function of LYDION it replaces (path:line within
 * the LYDION source tree), whose argument meaning it keeps.
 */
#ifndef LYDION_M1_H
#define LYDION_M1_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LYD_ABI_VERSION 6

/* status codes */
#define LYD_OK              0
#define LYD_ERR_ARG        -1   /* bad argument (size, pointer, enum)                  */
#define LYD_ERR_CUDA       -2   /* CUDA runtime error                                   */
#define LYD_ERR_NONFINITE  -3   /* a NaN/Inf appeared in J or H                          */
#define LYD_ERR_SOLVE      -4   /* a frequency tridiagonal system had a zero pivot      */
#define LYD_ERR_STATE      -5   /* call needs an input that was never provided           */
#define LYD_ERR_NOMEM      -6   /* device allocation failed                              */
#define LYD_ERR_TIMEOUT    -7   /* a bounded wait inside a kernel ran out (a bulk copy
                                   never completed, or a grid barrier of the persistent
                                   step); the kernel skipped its remaining work             */

/* boundary conditions (Symbol :Reflect / :Outflow in the reference) */
#define LYD_BC_REFLECT 0
#define LYD_BC_OUTFLOW 1
/* flux methods (LyaArrays{FluxMethod}, Val(:GLF) / Val(:HLL)) */
#define LYD_FLUX_GLF 0
#define LYD_FLUX_HLL 1
/* precision of the step */
#define LYD_PREC_FP64   0   /* everything in FP64 (the reference's arithmetic)             */
#define LYD_PREC_MIXED  1   /* FP64 state storage; the advection's reconstruction, closure,
                               fluxes and limiters in FP32 with the cell update accumulated
                               in FP64; the frequency step (factors, tridiagonal solve) and
                               all reductions in FP64, bar the cell-centre closure that sets
                               the Doppler velocity of the factors (FP32)                    */
#define LYD_PREC_FP32   2   /* FP32 storage and bulk arithmetic; FP64 tridiagonal solve and
                               reductions (fastest, least accurate: weak bins lose digits)  */

typedef struct lyd_ctx lyd_ctx;

typedef struct lyd_dims {
    int32_t n_nu;   /* frequency bins (N_nu), 4 <= n_nu <= 256 */
    int32_t n_r;    /* radial cells, >= 3                      */
    int32_t n_z;    /* vertical cells, >= 3                    */
    int32_t reserved;
} lyd_dims;

typedef struct lyd_config {
    int32_t flux_method;        /* LYD_FLUX_GLF or LYD_FLUX_HLL                           */
    int32_t recoil;             /* LyaArrays.Recoil                                        */
    int32_t precision;          /* LYD_PREC_*                                              */
    int32_t kcore_min;          /* LyaArrays.kcore_min - 1 (0-based, inclusive)            */
    int32_t kcore_max;          /* LyaArrays.kcore_max - 1                                 */
    int32_t keep_freq_factors;  /* keep F+/F/F- on the device so that a later frequency
                                   update may pass update_freq_factors = 0                 */
    double alpha_floor;         /* LyaArrays.alpha_Lya_floor                               */
    double j_scale;             /* LYD_PREC_MIXED / _FP32: J and H are held as value / j_scale
                                   (inside the FP32 range); 0 selects 1e-12                */
    int32_t device;             /* CUDA device ordinal                                     */
    int32_t geometry;           /* LYD_GEOM_CYLINDRICAL (0) or LYD_GEOM_CARTESIAN (1)         */
    int32_t bc_r_left;          /* boundary at the first r (X) interface of the static-driver
                                   steps: always LYD_BC_REFLECT (the axis) for a cylindrical
                                   grid; LYD_BC_REFLECT or LYD_BC_OUTFLOW for a Cartesian one  */
    int32_t reserved[5];
} lyd_config;

/* Geometries (LyaArrays on GeometryCylindrical or GeometryCartesian). A Cartesian context runs
 * AdvectJandH_Cartesian! (src/AdvectJandH.jl:1396-2222): r and Z stand for X and Y, the areas
 * and volumes of lyd_set_geometry are the Cartesian ones (A_X = dY, A_Y = dX, dV = dX dY, per
 * unit depth; src/SpatialGrid.jl:1061-1135), there is no K_phiphi source and no u_r / r term
 * (the context ignores inv_r_cell and rejects u_r / r), and the first X interface may be an
 * outflow boundary (ghost H_X = min(H_X, 0)). */
#define LYD_GEOM_CYLINDRICAL 0
#define LYD_GEOM_CARTESIAN   1

/* Cylindrical geometry: the fields of GeometryCylindrical read by AdvectJandH!
 * (src/AdvectJandH.jl:2272-2319). Arrays as described at the top of this file. */
typedef struct lyd_geometry {
    const double *r, *Z;                 /* interfaces, n_r+1 and n_z+1   */
    const double *rCoM, *ZCoM;           /* centroids, n_r and n_z         */
    const double *dV, *inv_dV;           /* n_r*n_z                        */
    const double *A_r;                   /* (n_r+1)*n_z                    */
    const double *A_Z;                   /* n_r*(n_z+1)                    */
    const double *inv_r_cell;            /* n_r                            */
    const double *dr_L, *dr_R, *inv_dr_i_im1, *inv_dr_ip1_i, *inv_dr_ip2_ip1;   /* n_r each */
    double dr_bnd[10];  /* inner: dr_L, dr_R, inv_i_im1, inv_ip1_i, inv_ip2_ip1; then outer */
    const double *dZ_L, *dZ_R, *inv_dZ_j_jm1, *inv_dZ_jp1_j, *inv_dZ_jp2_jp1;   /* n_z each */
    double dZ_bnd[10];
} lyd_geometry;

/* Frequency grid of LyaArrays: interfaces nu (n_nu+1), centres nuC, widths dnu, and the
 * stored inverses inv_dnu, inv_nuC (n_nu each). */
typedef struct lyd_freq_grid {
    const double *nu, *nuC, *dnu, *inv_dnu, *inv_nuC;
} lyd_freq_grid;

/* Fields that can be uploaded / downloaded (FP64 host arrays in the layouts above). */
enum lyd_field {
    /* (n_nu, n_r, n_z) */
    LYD_F_J = 0, LYD_F_J_OLD = 1, LYD_F_H_R = 2, LYD_F_H_Z = 3, LYD_F_H_R_OLD = 4, LYD_F_H_Z_OLD = 5,
    LYD_F_HVOIGT = 6,
    LYD_F_PHI_NU = 7,    /* uploading phi_nu makes the step read it; otherwise phi_nu is
                            derived from H_voigt by lyd_update_phi_nu                        */
    LYD_F_ALPHA_F = 8,   /* uploading alpha_F makes the step read it; otherwise
                            alpha_F = alpha*H_voigt (+ alpha_cF if uploaded)                 */
    /* (n_r, n_z) */
    LYD_F_ALPHA = 16, LYD_F_ALPHA_C = 17, LYD_F_ALPHA_CF = 18, LYD_F_PD = 19, LYD_F_JS = 20,
    LYD_F_T = 21, LYD_F_DUR_DR = 22, LYD_F_DUR_DZ = 23, LYD_F_DUZ_DR = 24, LYD_F_DUZ_DZ = 25,
    LYD_F_UR_OVER_R = 26, LYD_F_DRU_R = 27, LYD_F_DRU_Z = 28, LYD_F_F_R = 29, LYD_F_F_Z = 30,
    LYD_F_E_LYA = 31,     /* e_Lya, the Lya energy density of the RHD sub-cycle (erg cm^-3) */
    /* faces */
    LYD_F_U_R_STAR = 40,  /* (n_r+1, n_z) */
    LYD_F_U_Z_STAR = 41   /* (n_r, n_z+1) */
};

/* Diagnostics of one static-driver step. */
typedef struct lyd_diag {
    double M_F, M_F_radial_net, M_F_radial_out, L_tot, f_esc;
    int32_t kmin, kmax;   /* active window used by this step's advection (0-based) */
} lyd_diag;

/* Parameters of lyd_static_steps: one static-cloud driver iteration is
 * AdvectLya! -> LyaEmissionAbsorptionUpdate! -> FrequencyUpdateJLya_AllCells!(true)
 * -> Update_f_Lya_MF_L_Lya! -> Compute_f_esc_Lya_Cylindrical -> Reset_Delta_rho_u!
 * (src/StaticCloudTest.jl:357-392). */
typedef struct lyd_step_params {
    double c_tilde;        /* reduced speed of light                  */
    double dt;             /* time step                               */
    double z_center;       /* cloud centre for the radial M_F         */
    int32_t bc_r_right, bc_z_bot, bc_z_top;   /* the first r interface: lyd_config.bc_r_left */
    int32_t n_steps;
} lyd_step_params;

/* ---- context -------------------------------------------------------------------------- */
int  lyd_create(lyd_ctx **out, const lyd_dims *dims, const lyd_config *cfg);
int  lyd_destroy(lyd_ctx *ctx);
const char *lyd_last_error(const lyd_ctx *ctx);
int  lyd_abi_version(void);
/* The device's FP64 arithmetic helpers on n host values (device 0 or the current device), for
 * checks of their accuracy: fn 0: 1/sqrt(x) (approximation refined by Newton steps; x normal,
 * positive), 1: 1/x (likewise; x normal, nonzero), 2: sqrt(x) as x * (1/sqrt(x)), 3: the
 * closure chi(f) = (5 - 2 sqrt(4 - 3 f^2)) / 3 for f in [0, 1], 4: exp(x) for |x| <= 40 (the
 * table-driven form of the frequency factors). */
int  lyd_math_check(int32_t fn, const double *x, double *y, size_t n);
/* Page-locked host memory (cudaHostAlloc, portable to every context): copies between it and a
 * context run at the link's rate instead of through a pageable staging buffer, and the
 * host-state step's copies overlap. lyd_host_free releases it. */
int  lyd_host_alloc(size_t bytes, void **out);
int  lyd_host_free(void *p);
int  lyd_set_geometry(lyd_ctx *ctx, const lyd_geometry *g);
int  lyd_set_freq_grid(lyd_ctx *ctx, const lyd_freq_grid *f);
int  lyd_upload(lyd_ctx *ctx, int32_t field, const double *host, size_t count);
int  lyd_download(lyd_ctx *ctx, int32_t field, double *host, size_t count);
int  lyd_synchronize(lyd_ctx *ctx);
/* The CUDA stream (cudaStream_t) all work of this context is issued on. */
int  lyd_get_stream(lyd_ctx *ctx, void **stream);

/* ---- the Lyman-alpha step (drop-in replacements) -------------------------------------- */
/* FindActiveBins, src/UpdateLyaJandH.jl:47-97 */
int  lyd_find_active_bins(lyd_ctx *ctx, int32_t *kmin, int32_t *kmax);
/* AdvectLya!, src/UpdateLyaJandH.jl:107-171 (FindActiveBins + AdvectJandH! with
 * UpdateJold = true + H_old = H); bc_r_left must be LYD_BC_REFLECT (cylindrical axis). */
int  lyd_advect(lyd_ctx *ctx, double ctdt, int32_t bc_r_left, int32_t bc_r_right,
                int32_t bc_z_bot, int32_t bc_z_top);
/* AdvectJandH!, src/AdvectJandH.jl:2227-2464, with the caller's bin range [kmin, kmax]
 * (0-based) and J_old rule: update_jold != 0 sets J_old = J after the step, otherwise J_old
 * keeps its value; H_old is left alone. This is the form the stellar/IR bands use
 * (PhotoThermoChemistry.jl:3854-3868: all bands, UpdateJold = false, explicit alpha_F). */
int  lyd_advect_jh(lyd_ctx *ctx, double ctdt, int32_t kmin, int32_t kmax, int32_t update_jold,
                   int32_t bc_r_left, int32_t bc_r_right, int32_t bc_z_bot, int32_t bc_z_top);
/* LyaEmissionAbsorptionUpdate!, src/ConstantsAndFunctions.jl:483-573 (reads the uploaded
 * alpha, alpha_c, pd, js, H_voigt, phi_nu, alpha_F; accumulates into Delta rho u). */
int  lyd_emission_absorption(lyd_ctx *ctx, double c_tilde, double dt);
/* FrequencyUpdateJLya_AllCells!, src/UpdateLyaJandH.jl:231-391 with UpdateFreqFactors!
 * (src/FreqFactors.jl:142-278) and the per-cell tridiagonal solve
 * (src/TridiagonalSolver.jl:33-58). */
int  lyd_frequency_update(lyd_ctx *ctx, double ctdt, int32_t update_freq_factors);
/* UpdateLyaJandH!, src/UpdateLyaJandH.jl:409-486 (advection then frequency update). */
int  lyd_update_J_and_H(lyd_ctx *ctx, double dt, double c_tilde, int32_t update_freq_factors,
                        int32_t bc_r_left, int32_t bc_r_right, int32_t bc_z_bot, int32_t bc_z_top);
/* Update_f_Lya_MF_L_Lya!, src/ConstantsAndFunctions.jl:588-674: fills f_r, f_Z on the
 * device and returns {M_F, M_F_radial_net, M_F_radial_out, L_tot} in out[4]. */
int  lyd_force_multiplier(lyd_ctx *ctx, double dt, double z_center, int32_t bc_z_bot, double out[4]);
/* The gravity method of Update_f_Lya_MF_L_Lya!, src/ConstantsAndFunctions.jl:691-804:
 * f_grav_r, f_grav_Z are host arrays (n_r*n_z) of the gravitational force; out[5] =
 * {M_F, M_F_antigravity, M_F_radial_net, M_F_radial_out, L_tot}. */
int  lyd_force_multiplier_gravity(lyd_ctx *ctx, double dt, const double *f_grav_r, const double *f_grav_Z,
                                  double z_center, int32_t bc_z_bot, double out[5]);
/* Compute_f_esc_Lya_Cylindrical, src/ConstantsAndFunctions.jl:969-993 */
int  lyd_f_esc(lyd_ctx *ctx, double L_allspace, int32_t bc_z_bot, double *f_esc);
/* Reset_Delta_rho_u!, src/ConstantsAndFunctions.jl:809-816 */
int  lyd_reset_dru(lyd_ctx *ctx);
/* n_steps iterations of the static-cloud driver loop, src/StaticCloudTest.jl:357-392, as
 * fused kernels replayed from a CUDA graph. diag_hist (may be NULL) receives one lyd_diag
 * per step; with diag_hist == NULL the call returns once the steps are enqueued and any
 * error is reported by the next synchronising call. */
int  lyd_static_steps(lyd_ctx *ctx, const lyd_step_params *p, lyd_diag *diag_hist);
/* One static-driver iteration on host state: J, H_r, H_Z (n_nu x n_r x n_z doubles each, the
 * layout of lyd_upload) go up, the step runs, the new J, H_r, H_Z come back into the *_out
 * arrays (which may be the inputs themselves) and diag receives its record (may be NULL).
 * p->n_steps is ignored. The copies and the step are pipelined over `chunks` row chunks
 * (1..16; 8 is a good choice): a chunk's rows advect once the next chunk has landed, its cells
 * take the frequency step and go back down while later chunks still go up. For that the step
 * uses the active window the previous step decided, and checks it against FindActiveBins of the
 * uploaded J; when they differ (the caller changed J in between, or on the first call) the call
 * steps again from the uploaded state, unpipelined. One cloud, the FP64 form (LYD_PREC_FP64,
 * whose state is held in the caller's units), no Z slab; other contexts get LYD_ERR_STATE. The
 * host arrays should be page-locked for the copies to overlap. The call returns when the
 * outputs are written. */
int  lyd_static_step_host(lyd_ctx *ctx, const lyd_step_params *p, const double *J, const double *H_r,
                          const double *H_Z, double *J_out, double *H_r_out, double *H_Z_out, int32_t chunks,
                          lyd_diag *diag);
/* Per-kernel device time of the last lyd_static_steps call that had timing enabled:
 * ms[0] = advection kernel, ms[1] = frequency kernel, ms[2] = reductions (totals). */
int  lyd_set_timing(lyd_ctx *ctx, int32_t enable);
int  lyd_get_timing(lyd_ctx *ctx, double ms[3]);

/* ---- batches of independent clouds ------------------------------------------------------ */
/* A context may hold many independent clouds of different (n_r, n_z) sharing one frequency
 * grid and one configuration: the batched form of the static-cloud run (512 clouds of
 * uneven size advancing together). Every step kernel covers all clouds in one launch (a work
 * list of per-cloud tiles), each cloud with its own time step and boundary conditions, and
 * the step is replayed from one CUDA graph. lyd_create is a batch of one cloud.
 *
 * On a context of several clouds: lyd_upload / lyd_download move every cloud's values,
 * concatenated cloud after cloud; lyd_find_active_bins writes n_clouds entries to each of
 * kmin and kmax; lyd_static_steps runs every cloud with the same parameters and writes
 * n_steps * n_clouds records; the step phases (lyd_advect ... lyd_update_J_and_H) apply one
 * c_tilde, dt and boundary set to all clouds; lyd_set_geometry, lyd_force_multiplier,
 * lyd_f_esc, lyd_cfl_dt and lyd_edge_spectra return LYD_ERR_STATE (use the per-cloud forms
 * and the lyd_batch_steps records). An explicitly uploaded phi_nu or alpha_F must be
 * uploaded for every cloud. */
int  lyd_batch_create(lyd_ctx **out, int32_t n_clouds, const int32_t *n_r, const int32_t *n_z, int32_t n_nu,
                      const lyd_config *cfg);
int  lyd_batch_info(lyd_ctx *ctx, int32_t *n_clouds, int64_t *cell_bins);
int  lyd_set_geometry_cloud(lyd_ctx *ctx, int32_t cloud, const lyd_geometry *g);
int  lyd_upload_cloud(lyd_ctx *ctx, int32_t cloud, int32_t field, const double *host, size_t count);
int  lyd_download_cloud(lyd_ctx *ctx, int32_t cloud, int32_t field, double *host, size_t count);
int  lyd_edge_spectra_cloud(lyd_ctx *ctx, int32_t cloud, double *raw, double *norm, int32_t *r_index,
                            int32_t *z_index);

typedef struct lyd_cloud_params {
    double c_tilde, dt, z_center;
    int32_t bc_r_right, bc_z_bot, bc_z_top, reserved;
} lyd_cloud_params;
/* n_steps static-driver iterations of every cloud, cloud q with params[q]; hist (may be NULL)
 * receives n_steps * n_clouds records, step-major. */
int  lyd_batch_steps(lyd_ctx *ctx, const lyd_cloud_params *params, int32_t n_steps, lyd_diag *hist);
/* lyd_batch_steps with each step as ONE cooperative launch of a persistent kernel (a grid of
 * resident CTAs runs the advection tiles, the frequency-kernel cells and the reduction, with
 * a grid barrier between the phases) instead of three launches; the results are bit-for-bit
 * those of lyd_batch_steps. A CTA that waits at a barrier for more than barrier_polls polls
 * (~0.1 us each) gives up and the call reports LYD_ERR_TIMEOUT (at the next synchronising
 * call when hist is NULL); the state is then undefined and the context stays usable.
 * barrier_polls must be positive; 1 << 24 is ample. The rows are staged by per-lane loads. */
int  lyd_batch_steps_persistent(lyd_ctx *ctx, const lyd_cloud_params *params, int32_t n_steps,
                                int64_t barrier_polls, lyd_diag *hist);
/* Whether the persistent step is replayed from a CUDA graph: 1 yes, -1 launched directly (the
 * runtime refused to capture it), 0 not run yet. */
int  lyd_persistent_info(lyd_ctx *ctx, int32_t *graph);

/* Launch-shape knobs chosen by the autotuner (lydion_b200/autotune.py): rows of the
 * advection tile (4..64), cells per frequency-kernel block (8..1024, or 0 for automatic), the
 * frequency solver (0: parallel cyclic reduction across the warp; 1: lane-serial
 * elimination), the advection kernel's resident CTAs per SM (2..4 with FP32 arithmetic,
 * 2..3 with FP64, or 0 for the default: 4 and 3), and how the advection stages its rows
 * (LYD_STAGING_*). lyd_get_tuning reports an automatic cell count as its negative and the
 * staging actually used. */
#define LYD_STAGING_AUTO   0   /* the library's choice: bulk copies with FP32 storage, per-lane
                                  loads otherwise                                               */
#define LYD_STAGING_LANES  1   /* per-lane loads of every staged cell                         */
#define LYD_STAGING_TMA    2   /* bulk tensor copies (TMA) of each row's 32-bin x 12-column box,
                                  a row ahead, when a row of n_nu bins is a multiple of 16 bytes */
typedef struct lyd_tuning {
    int32_t rows_per_tile, cells_per_block, solver, adv_ctas_per_sm, adv_staging;
} lyd_tuning;
int  lyd_set_tuning(lyd_ctx *ctx, const lyd_tuning *t);
int  lyd_get_tuning(lyd_ctx *ctx, lyd_tuning *t);

/* ---- adjoint ------------------------------------------------------------------------------ */
/* Gradients of  objective = w_MF * M_F(last step) + sum_k w_spec[k] * S_k(final J)  over
 * n_steps static-driver steps from the current state, S being the edge-ring mean spectrum of
 * lyd_edge_spectra. With checkpoint_every = 1, or 0 when they fit in free device memory
 * (7 doubles per cell-bin per step), the forward sweep keeps every step's state and advection
 * tape, plus its frequency factors when 10 doubles per cell-bin per step fit, and nothing is
 * recomputed; with checkpoint_every = K > 1 (0 otherwise: 100)
 * it stores the state every K steps and the reverse sweep recomputes each segment once (with
 * timing off, and when the room is there, into a second buffer of K states and tapes on a
 * second stream while the segment after it is reversed); with
 * checkpoint_every < 0 it keeps `snapshots` + 1 states in Griewank's binomial (Revolve)
 * schedule, advancing no step more than r times, r the least with C(snapshots + 1 + r, r) >=
 * n_steps, and records each step's tape right before its reverse (with timing off, the advances
 * and records run on a second stream ahead of the reversals, two steps' records in flight). The
 * reverse sweep runs hand-written adjoint kernels of the step (advection, emission/absorption,
 * frequency factors, transposed tridiagonal solve, flux correction). The active window of every step is the forward's.
 * Non-smooth points (MinMod, floors, clamps, limiters) take the derivative of the branch the
 * forward took. Needs a single-cloud FP64 context (GLF or HLL flux) and alpha_F derived from
 * alpha and H_voigt. The context ends in the final state of the forward sweep.
 * grad_T includes the H_voigt(T) chain when H_voigt was computed by lyd_update_hvoigt (not
 * uploaded), and the T of the frequency factors (Doppler width, recoil); gradients with
 * respect to n_H and a dust opacity follow from grad_alpha and grad_alpha_c by the caller's
 * parametrisation (alpha = x_HI n_H sigma0(T)). No counterpart exists in the reference. */
typedef struct lyd_adjoint_cfg {
    lyd_step_params step;        /* c_tilde, dt, z_center, boundaries, n_steps */
    int32_t checkpoint_every;    /* 1: keep every step; K > 1: a checkpoint every K steps; 0:
                                    every step when it fits, else K = 100; < 0: the binomial
                                    schedule with `snapshots` state snapshots */
    int32_t snapshots;           /* binomial schedule: snapshots besides the initial state (0:
                                    the fewest with which no step is advanced more than twice) */
    double w_MF;
    const double *w_spec;        /* n_nu weights, or NULL */
} lyd_adjoint_cfg;

typedef struct lyd_adjoint_out { /* host arrays; any may be NULL */
    double *objective, *M_F;     /* 1 each */
    double *spectrum;            /* n_nu */
    double *grad_alpha, *grad_alpha_c, *grad_T;                /* n_r*n_z each */
    double *grad_Hv;             /* n_nu*n_r*n_z: H_voigt as an independent input */
    double *grad_u_r_star;       /* (n_r+1)*n_z */
    double *grad_u_Z_star;       /* n_r*(n_z+1) */
    double *grad_du[5];          /* dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r: n_r*n_z each */
    double *grad_J0, *grad_H_r0, *grad_H_Z0;                   /* initial state, n_nu*n_r*n_z each */
} lyd_adjoint_out;

int  lyd_adjoint_run(lyd_ctx *ctx, const lyd_adjoint_cfg *cfg, lyd_adjoint_out *out);
/* Device time of the phases of the last lyd_adjoint_run made with timing enabled (ms):
 * forward sweep, segment recomputation (which also records the advection's tapes), 0
 * (reserved), frequency-step adjoint, advection adjoint. */
int  lyd_get_adjoint_timing(lyd_ctx *ctx, double ms[5]);

/* ---- set-up and output helpers --------------------------------------------------------- */
/* Update_Hvoigt! from the uploaded temperature, src/ConstantsAndFunctions.jl:319-357, using
 * the Voigt look-up tables of src/FastInterpolations.jl:175-275 built on the device. */
int  lyd_update_hvoigt(lyd_ctx *ctx);
/* Update_phi_nu!, src/ConstantsAndFunctions.jl:362-393 (normalised over bins kmin..kmax) */
int  lyd_update_phi_nu(lyd_ctx *ctx, int32_t kmin, int32_t kmax);
/* pd_Lya, src/LymanAlphaDestruction.jl:43-97, evaluated on the device for n cells; inputs
 * and output are host arrays of length n. */
int  lyd_pd_lya(lyd_ctx *ctx, size_t n, const double *nHII, const double *ne, const double *nHI,
                const double *nHeI, const double *nH2, const double *T, double z, double *pd_out);
/* GetRHDCFLTimeStep, src/AdvectJandH.jl:29-68, with cell-centred u_r, u_Z (host arrays). */
int  lyd_cfl_dt(lyd_ctx *ctx, double c_tilde, const double *u_r, const double *u_Z, double cfl,
                double *dt_out);
/* Edge-ring spectra of src/SaveHDF5Data_StaticCloudTests.jl:152-199, 392-420:
 * n_edge = (n_z-2) + 2*(n_r-3) cells; raw and normalised are (n_edge, n_nu) row-major. */
int  lyd_edge_count(int32_t n_r, int32_t n_z);
int  lyd_edge_spectra(lyd_ctx *ctx, double *raw, double *norm, int32_t *r_index, int32_t *z_index);
/* ---- Z-slab domain decomposition of one field --------------------------------------------------
 * One large field split into slabs of rows over ranks (one GPU each). A rank's context holds its
 * rows plus two halo rows on each side that has a neighbour; its geometry, frequency grid and
 * per-cell inputs are the global ones sliced to those rows. Per step, with the communication done
 * by the caller (all-reduce of the column sums, exchange of the halo rows; e.g. NCCL through
 * torch.distributed) on buffers in device memory:
 *   lyd_dd_step_partials -> all-reduce(colsum) -> lyd_dd_finish -> lyd_dd_halo(pack) ->
 *   exchange -> lyd_dd_halo(unpack)
 * and once before the first step lyd_dd_find_active_partials -> all-reduce -> lyd_dd_finish(step
 * = 0). The advection updates only the owned rows; its stencil reads the halo rows; the
 * frequency step, FindActiveBins and the diagnostics run on the owned cells, and the window and
 * diagnostics come from the all-reduced sums, so every rank takes the same window. There is no
 * counterpart in the reference, which runs one field on one node. */
int  lyd_dd_set_halo(lyd_ctx *ctx, int32_t h_bot, int32_t h_top);   /* 0 or 2 rows each */
int  lyd_dd_columns(lyd_ctx *ctx);   /* length of the column-sum vector (n_nu + 6 doubles) */
int  lyd_dd_find_active_partials(lyd_ctx *ctx, double *colsum_dev);
int  lyd_dd_step_partials(lyd_ctx *ctx, const lyd_step_params *p, double *colsum_dev);
/* the window of the next step from the all-reduced sums, and with step != 0 the step's record */
int  lyd_dd_finish(lyd_ctx *ctx, const double *colsum_dev, int32_t step, lyd_diag *rec);
/* side 0: lower neighbour, 1: upper; pack copies the two owned rows next to that neighbour, unpack
 * fills the two halo rows; buf_dev holds J, H_r, H_Z of two rows (6 n_r n_nu values in the
 * storage type: 8 bytes in FP64 and mixed, 4 in FP32). */
int  lyd_dd_halo(lyd_ctx *ctx, int32_t side, int32_t pack, void *buf_dev);

/* ---- RHD-side Lyman-alpha block ---------------------------------------------------------------
 * The Lya part of the per-cell photo-thermochemistry sub-cycle of the RHD drivers, on the device
 * for every cell of the context at once, so that an RHD code whose chemistry runs on the GPU
 * never copies J and H to the host between transport steps. */
typedef struct lyd_dust_lya {
    double kappa_abs[3];   /* Lya absorption opacity per dust mass, Sil / C / PAH (cm^2 g^-1)  */
    double kappa_F[3];     /* Lya flux (absorption + scattering) opacity per dust mass         */
    double rho_ignore;     /* dust densities at or below this are ignored (rho_d_IGNORE)       */
} lyd_dust_lya;
/* PrepareLyaSubCycling!, src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:2087-2155, for
 * every cell: T and the species number densities (cm^-3) and the three dust mass densities
 * rho_d[3][n_r*n_z] (g cm^-3) are host arrays. Sets T; H_voigt (lyd_update_hvoigt) and phi_nu
 * normalised over all bins (Update_Hvoigt_And_phinu_cell!, :2039-2080); alpha = nHI sigma0(T);
 * alpha_c (dust and gas continuum absorption); alpha_cF (dust and gas continuum flux opacity,
 * so that alpha_F = alpha H_voigt + alpha_cF); pd (pd_Lya when destruction != 0, else 0); and
 * js = recombination (Case B if ots, else Case A) + collisional emissivity
 * (src/LymanAlphaEmission.jl:106-175). */
int  lyd_rhd_lya_prepare(lyd_ctx *ctx, const double *T, const double *nHI, const double *nH2, const double *nHII,
                         const double *nHeI, const double *ne, const double *nOHx, const double *nCHx,
                         const double *rho_d, const lyd_dust_lya *dust, double z, int32_t ots,
                         int32_t destruction);
/* Per-cell results of lyd_rhd_lya_absorb, host arrays of n_r*n_z (split: 8 per cell,
 * split[q*n_r*n_z + cell] for q = gas r, gas Z, Sil r, Sil Z, C r, C Z, PAH r, PAH Z); any may be
 * NULL. */
typedef struct lyd_rhd_lya_out {
    int32_t *reject;       /* 1 where the sub-step is rejected                                    */
    double *de;            /* |e_new - e_Lya| / (e_Lya + e_floor)                                 */
    double *e_new;         /* 4 pi / c sum_k dnu_k J_k after the sub-step (erg cm^-3)             */
    double *dru_r, *dru_Z; /* radiation momentum of the sub-step (g cm^-2 s^-1)                   */
    double *split;         /* its split between gas and the three dust kinds (SplitRadPressure)   */
    double *dt_lya;        /* the absorption time 1 / (c~ (alpha_c + pd alpha)) (s)               */
} lyd_rhd_lya_out;
/* The Lya block of AbsorptionStep, src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:
 * 1580-1680, for every cell over its own sub-step dt[cell] (host array, s): J = max((J_old +
 * dt c~ js phi)/(1 + (alpha_c + pd alpha H_voigt) c~ dt), Jeps), H = H_old/(1 + alpha_F c~ dt),
 * the momentum and its split, e_new and the rejection test (relative change of e_Lya above 0.1
 * while dt exceeds 0.1 of the absorption time, or not finite). J and H are written for every
 * cell. With commit != 0, accepted cells then take J_old = J, H_old = H and e_Lya = e_new
 * (:3197-3206) and rejected cells get J = J_old, H = H_old back (RestoreLyaRejection, :980-991). */
int  lyd_rhd_lya_absorb(lyd_ctx *ctx, const double *dt, double c_tilde, int32_t commit, lyd_rhd_lya_out *out);

/* FindRSL_LyaRT, src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:614-711: the reduced speed
 * of light the Lya transport needs from the hydro and chemistry state, a maximum over the cells
 * (single-cloud contexts). Host arrays of n_r*n_z: cell velocities u_r, u_Z (cm/s), pressure,
 * density, adiabatic index, T, x_HII, x_H2, and rho_d[3][n_r*n_z]; the context supplies the cell
 * widths (lyd_set_geometry) and pd (lyd_rhd_lya_prepare or an upload). eps_rsl is the reference's
 * eps_RSL (4), X_over_mH the hydrogen mass fraction over m_H. The result is clamped to
 * [c_tilde_min, c], and to [0.75, 4] times c_tilde_old. */
int  lyd_find_rsl_lya(lyd_ctx *ctx, double c_tilde_old, double c_tilde_min, const double *u_r, const double *u_Z,
                      const double *P, const double *rho, const double *gamma_ad, const double *T,
                      const double *xHII, const double *xH2, const double *rho_d, const lyd_dust_lya *dust,
                      double eps_rsl, double X_over_mH, double *c_tilde_new);

/* The five Voigt look-up tables the device evaluates (CreateVoigtLUTs,
 * src/FastInterpolations.jl:178-197): erf, Dawson's integral, exp(-x^2), x exp(-x^2) and
 * (1-2x^2) exp(-x^2) at x_i = -xmax + 2 xmax i/(n-1), written to out[5*n] table after table.
 * Host-only; needs no GPU. */
int  lyd_voigt_tables(double *out, int32_t n, double xmax);

/* ---- FindActiveBins without any device allocation ----------------------------------------
 * No counterpart in the reference. For callers that may not allocate device memory (a host
 * framework that owns every allocation through its own pool, a plugin inside a fixed memory
 * budget, a time loop that must not allocate): computes the active-bin window of
 * FindActiveBins from caller-owned device arrays J (n_nu*n_r*n_z, FP64 in physical units,
 * [k,i,j]: the Jeps floor of 1e-60 applies to J as given, so a state a context holds as
 * value / j_scale must be scaled back first), dnu (n_nu) and dV (n_r*n_z), on `stream` (a cudaStream_t; NULL is the legacy default stream), and
 * returns kmin/kmax (0-based) to the host after synchronising that stream. It creates no
 * context and calls no cudaMalloc/cudaFree: its scratch is a file-scope 1 MiB device array
 * (131072 FP64 partial sums) that every GPU loading the library holds until exit. The first
 * call on each device looks up that array's address, so make the first call before any
 * stream capture. All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. Returns LYD_ERR_ARG for n_nu > 256 (or n_nu < 4, n_r < 3,
 * n_z < 3, a bad core range, a null pointer). */
int  lyd_find_active_bins_noalloc(const double *J, const double *dnu, const double *dV, int32_t n_nu,
                                  int32_t n_r, int32_t n_z, int32_t kcore_min, int32_t kcore_max,
                                  void *stream, int32_t *kmin, int32_t *kmax);

#ifdef __cplusplus
}
#endif
#endif /* LYDION_M1_H */
