// lyd_internal.h -- device-side argument blocks and launch wrappers of the Lyman-alpha
// step kernels (shared by lyd_kernels.cu, lyd_aux.cu and lyd_api.cu).
//
// A context holds one or more independent clouds ("a batch"). Every field of every cloud
// lives in one concatenated device array per field; a CloudDesc gives each cloud's offsets,
// grid size, boundary conditions and time step. The step kernels walk work lists:
// advection tiles (cloud, i0, j0, k0) and frequency-kernel items (cloud, first cell, end
// cell). A single cloud is a batch of one.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace lyd {

struct CloudDesc {
    long long o3;        // offset of the (k, i, j) fields, in cell-bins
    long long oc;        // offset of the per-cell fields
    long long orf;       // offset of the r-face fields ((n_r+1) n_z: A_r, u*_r)
    long long ozf;       // offset of the Z-face fields (n_r (n_z+1): A_Z, u*_Z)
    int ocol, orow;      // per-column (n_r: <1/r>, rCoM) and per-row (n_z: ZCoM) fields
    int orint, ozint;    // PLM intervals per face ((n_r+1)*5, (n_z+1)*5)
    int orif, ozif;      // interface coordinates (n_r+1, n_z+1)
    int nr, nz;
    int bc_r_left, bc_r_right, bc_z_bot, bc_z_top;
    int j_own0, j_own1;  // rows this context updates; outside them, halo rows of a Z-slab
                         // decomposition (domain neighbours' rows, read by the stencil only)
    int pb0, npb;        // this cloud's blocks in the frequency-kernel work list / partials
    double ctdt, dt, c_tilde, z_center;
};

// Columns of the per-block reduction partials written by the step kernels:
// [0, nnu)        E_bin(k)  = sum dnu_k max(J - 10 Jeps, 0) dV          (FindActiveBins)
// nnu + 0         E_tot     = sum dnu_k max(J - Jeps, 0) dV
// nnu + 1..3      sum dV |f|, sum dV f.r_out, sum dV max(f.r_out, 0)     (M_F family)
// nnu + 4         sum 4 pi dV js                                         (L_Lya)
// nnu + 5         sum dnu_k A 4 pi max(+-H, 0) over escaping faces        (f_esc numerator)
constexpr int kExtraCols = 6;

enum { PART_ACTIVE = 1, PART_DIAG = 2 };

// Kernel precision variants (the values of LYD_PREC_*): storage type S / arithmetic type R.
enum { PREC_K_FP64 = 0,     // S = double, R = double
       PREC_K_MIXED = 1,    // S = double, R = float in the advection fluxes
       PREC_K_FP32 = 2 };   // S = float,  R = float

// Advection: AdvectJandH_Cylindrical! (src/AdvectJandH.jl:526-1390), reads set `in`,
// writes set `out`. Bins outside each cloud's active window are copied through.
template <typename S>
struct AdvArgs {
    const S *J, *Hr, *HZ;
    S *Jo, *Hro, *HZo;
    const S *aF;                 // explicit alpha_F, or nullptr to derive alpha*H_voigt (+alpha_cF)
    const S *Hv;
    const double *alpha, *alpha_cF;
    const double *A_r, *A_Z, *inv_dV, *inv_r_cell;
    const double *rint, *zint;   // PLM intervals per face, [(n+1)][5] per cloud
    const double *u_r_star, *u_Z_star;
    const double *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;
    const int *kwin;             // device {kmin, kmax} per cloud
    const CloudDesc *cl;
    const int4 *tiles;           // (cloud, i0, j0, k0)
    int rows;                    // rows per tile
    int nnu;
    double jeps, heps2;          // closure floors in storage units
    double *tape;                // adjoint recomputation: the cell update's values before its
                                 // floors and limiter, 4 fields of tape_stride (or nullptr)
    long long tape_stride;
    const unsigned char *tmaps;  // tensor maps of the input J, H_r, H_Z, [cloud][3] of
                                 // kTensorMapBytes each in device memory, or nullptr: per-lane loads
    int *err;                    // device error bits (ERRB_TIMEOUT)
};

// Emission/absorption + frequency step + flux correction (+ partial reductions).
template <typename S>
struct FreqArgs {
    const S *Jin, *Hrin, *HZin;  // current J, H
    const S *Jold;               // J_old (== Jin when the old set aliases the current one);
                                 // H_old is never read: every phase overwrites it first
    S *Jout, *Hrout, *HZout;
    const S *Hv;
    const S *phi;                // explicit phi_nu, or nullptr to derive H_voigt * phi_inv
    const double *phi_inv;       // per-cell 1 / sum_core dnu H_voigt
    int phi_kmin, phi_kmax;
    const S *aF;                 // explicit alpha_F or nullptr
    const double *alpha, *alpha_c, *alpha_cF, *pd, *js, *T;
    const double *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;
    double *dru_r, *dru_Z;       // accumulated momentum (nullptr: not stored)
    double *f_r, *f_Z;           // fused step: this step's force Delta rho u / dt (or nullptr)
    double *Fkp, *Fk, *Fkm;      // stored frequency factors (nullptr: not kept)
    const double *nu, *nuC, *dnu, *inv_dnu, *inv_nuC;
    const double *dV, *A_r, *A_Z, *rCoM, *ZCoM;
    const CloudDesc *cl;
    const int4 *items;           // (cloud, first cell, end cell) per block
    double alpha_floor;
    double jeps, heps2, j_scale;
    int do_emission, do_freq, update_ff, recoil;
    int parts;                   // PART_* bits
    double *partials;            // [ncols][nblocks]
    int *err;                    // device error bits
    int nnu;
    int solver;                  // SOLVER_*
    int vec16;                   // set by the launcher: rows move as whole 16-byte words
    int item0, nitems_all;       // a launch over items item0 .. of a list of nitems_all (0: the grid's)
};

enum { SOLVER_PCR = 0, SOLVER_THOMAS = 1 };

// Reduction of the partials into each cloud's kmin/kmax and step diagnostics (one CTA per
// cloud).
struct RedArgs {
    const double *partials;
    int nblocks;                 // total frequency-kernel blocks (partial stride)
    int nnu, nclouds;
    int parts;
    int kcore_min, kcore_max;
    double j_scale;
    const CloudDesc *cl;
    int *kwin;                   // out {kmin, kmax} per cloud
    double *diag;                // out: [step][cloud][7], or nullptr
    int *step_counter;           // record index (incremented once per launch)
    int *done;                   // completion counter of the CTAs of one launch
    int hist_capacity;           // steps
    double *last;                // out: latest record per cloud [cloud][7]
    // Column sums over several CTAs per cloud (8 columns each), the last CTA of a cloud to
    // finish taking the decision: the sums [cloud][N_nu + kExtraCols] and the per-cloud CTA
    // counters (zero between launches). Both null: one CTA per cloud sums every column.
    double *colsum;
    int *cnt;
    int *kwin_copy;              // optional second destination of the decided window [cloud][2]
};

// error bits
enum { ERRB_NONFINITE = 1, ERRB_SOLVE = 2, ERRB_TIMEOUT = 4 };
// size of one CUtensorMap (an opaque 64-byte-aligned record)
constexpr int kTensorMapBytes = 128;

int bins_per_lane(int nnu);
// `prec` of the step launches is a PREC_K_* variant; `sprec` of the others is the storage
// type of the state arrays (0: double, 1: float).
void launch_find_active(int sprec, const void *J, int nnu, const double *dnu, const double *dV, const CloudDesc *cl,
                        const int4 *items, int nitems, double jeps, double *partials, cudaStream_t st);
void launch_advect(int prec, int flux, const void *args, int ntiles, int ctas_per_sm, cudaStream_t st);
int adv_ctas_per_sm(int prec, int want);   // the occupancy variant launch_advect uses
void launch_freq(int prec, const void *args, int nnu, int nitems, cudaStream_t st);
// fn 0: rsqrt_nr, 1: rcp<double>, 2: x * rsqrt_nr(x), 3: chi_L84<double>, 4: exp_tab
void launch_math(int fn, const double *x, double *y, size_t n, cudaStream_t st);
// one fused step in one cooperative launch (advection, frequency step, reduction, with bounded
// grid barriers between them); bar: two unsigned of device memory
cudaError_t launch_persistent(int prec, int flux, const void *adv, const void *freq, const RedArgs &red, int nnu,
                              int ntiles, int nitems, unsigned *bar, long long polls, int *err, cudaStream_t st);
void launch_reduce(const RedArgs &a, cudaStream_t st);
int freq_blocks(int ncell, int dev);

// auxiliary kernels (lyd_aux.cu)
void launch_convert_in(int prec, const double *src, void *dst, size_t n, double scale, cudaStream_t st);
void launch_convert_out(int prec, const void *src, double *dst, size_t n, double scale, cudaStream_t st);
void launch_hvoigt(int prec, void *Hv, const double *T, const double *nu, const double *nuC, int nnu, size_t ncell,
                   const double *lut, int lut_n, double lut_xmax, cudaStream_t st);
void launch_phi_inv(int prec, const void *Hv, const double *dnu, int nnu, size_t ncell, int kmin, int kmax,
                    double *phi_inv, cudaStream_t st);
void launch_pd(size_t n, const double *nHII, const double *ne, const double *nHI, const double *nHeI,
               const double *nH2, const double *T, double z, double *out, cudaStream_t st);
void launch_mf(const double *dru_r, const double *dru_Z, double *f_r, double *f_Z, const double *js,
               const double *dV, const double *rCoM, const double *ZCoM, int nr, int nz, double dt,
               double z_center, const double *g_r, const double *g_Z, double *partials, int nblocks,
               cudaStream_t st);   // g_r/g_Z: gravity field for M_F_antigravity, or nullptr
void launch_fesc(int prec, const void *Hr, const void *HZ, const double *A_r, const double *A_Z,
                 const double *dnu, int nnu, int nr, int nz, int bc_z_bot, double j_scale,
                 double *out, cudaStream_t st);
void launch_column_sums(const double *partials, int ncols, int nblocks, double *out, cudaStream_t st);
void launch_cfl(const double *r, const double *Z, const double *u_r, const double *u_Z, int nr, int nz,
                double c_tilde, double *out, cudaStream_t st);
void launch_edge(int prec, const void *J, const double *dnu, int nnu, int nr, int nz, double j_scale,
                 double *raw, double *norm, cudaStream_t st);
void build_voigt_lut(double *host, int n, double xmax);   // host: 5 tables of n entries

// RHD-side Lyman-alpha block (lyd_rhd.cu)
struct RhdPrepArgs {
    const double *T, *nHI, *nH2, *nHII, *nHeI, *ne, *nOHx, *nCHx, *rho_d;   // rho_d: [3][ncell]
    double kabs[3], kF[3], rho_ignore, z;
    int ots, destruction;
    size_t ncell;
    double *alpha, *alpha_c, *alpha_cF, *pd, *js, *T_out, *dust_F;         // dust_F: [3][ncell]
};
template <typename S>
struct RhdAbsorbArgs {
    const double *dt;                          // per cell
    const double *alpha, *alpha_c, *alpha_cF, *pd, *js, *phi_inv, *dust_F, *dnu;
    const S *Hv;
    S *J, *Hr, *HZ;                            // written
    S *Jold, *Hrold, *HZold;                   // read; written by an accepting commit
    double *e_lya;                             // per cell: read, and written by a commit
    double *out;                               // [14][ncell]
    double c_tilde, jeps, j_scale;
    int nnu, commit;
    size_t ncell;
};
struct RslArgs {
    const double *r_if, *Z_if;                 // interface coordinates
    const double *u_r, *u_Z, *P, *rho, *gamma, *T, *xHII, *xH2, *rho_d, *pd;   // rho_d: [3][ncell]
    double kabs[3], eps_rsl, X_over_mH;
    int nr;
    size_t ncell;
    unsigned long long *out;                   // bits of the maximum (non-negative double)
};
void launch_rhd_prep(const RhdPrepArgs &a, cudaStream_t st);
void launch_rsl(const RslArgs &a, cudaStream_t st);
void launch_rhd_absorb(int sprec, const void *args, cudaStream_t st);

}  // namespace lyd
