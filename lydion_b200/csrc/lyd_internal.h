// lyd_internal.h -- device-side argument blocks and launch wrappers of the Lyman-alpha
// step kernels (shared by lyd_kernels.cu and lyd_api.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace lyd {

// Columns of the per-block reduction partials written by the step kernels:
// [0, nnu)        E_bin(k)  = sum dnu_k max(J - 10 Jeps, 0) dV          (FindActiveBins)
// nnu + 0         E_tot     = sum dnu_k max(J - Jeps, 0) dV
// nnu + 1..3      sum dV |f|, sum dV f.r_out, sum dV max(f.r_out, 0)     (M_F family)
// nnu + 4         sum 4 pi dV js                                         (L_Lya)
// nnu + 5         sum dnu_k A 4 pi max(+-H, 0) over escaping faces        (f_esc numerator)
constexpr int kExtraCols = 6;

enum { PART_ACTIVE = 1, PART_DIAG = 2 };

// Advection: AdvectJandH_Cylindrical! (src/AdvectJandH.jl:526-1390), reads set `in`,
// writes set `out`. Bins outside the active window are copied through.
template <typename S>
struct AdvArgs {
    const S *J, *Hr, *HZ;
    S *Jo, *Hro, *HZo;
    const S *aF;                 // explicit alpha_F, or nullptr to derive alpha*H_voigt (+alpha_cF)
    const S *Hv;
    const double *alpha, *alpha_cF;
    const double *A_r, *A_Z, *inv_dV, *inv_r_cell;
    const double *rint, *zint;   // PLM intervals per face, [(n+1)][5]
    const double *u_r_star, *u_Z_star;
    const double *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;
    const int *kwin;             // device {kmin, kmax}
    int nnu, nr, nz;
    double ctdt;
    double jeps, heps2;          // closure floors in storage units
    int bc_r_right, bc_z_bot, bc_z_top;
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
    double c_tilde, dt, ctdt, z_center;
    double alpha_floor;
    double jeps, heps2, j_scale;
    int do_emission, do_freq, update_ff, recoil;
    int bc_z_bot;
    int parts;                   // PART_* bits
    double *partials;            // [ncols][nblocks]
    int *err;                    // device error bits
    int nnu, nr, nz;
};

// Reduction of the partials into kmin/kmax and the step diagnostics.
struct RedArgs {
    const double *partials;
    int nblocks, nnu;
    int parts;
    int kcore_min, kcore_max;
    double dt, c_tilde, j_scale;
    int bc_z_bot;
    int *kwin;                   // out {kmin, kmax}
    double *diag;                // out: per-step record base (7 doubles per step), or nullptr
    int *step_counter;           // index of the record to write (incremented)
    int hist_capacity;
    double *last;                // out: the latest record (7 doubles)
    int *err;
};

// error bits
enum { ERRB_NONFINITE = 1, ERRB_SOLVE = 2 };

void launch_find_active(int prec, const void *J, int nnu, int nr, int nz, const double *dnu, const double *dV,
                        double jeps, double *partials, int nblocks, cudaStream_t st);
void launch_advect(int prec, int flux, const void *args, int nnu, int nr, int nz, cudaStream_t st);
void launch_freq(int prec, const void *args, int nnu, int ncell, int nblocks, cudaStream_t st);
void launch_reduce(const RedArgs &a, cudaStream_t st);
int freq_blocks(int ncell, int dev);

// auxiliary kernels (lyd_aux.cu)
void launch_convert_in(int prec, const double *src, void *dst, size_t n, double scale, cudaStream_t st);
void launch_convert_out(int prec, const void *src, double *dst, size_t n, double scale, cudaStream_t st);
void launch_hvoigt(int prec, void *Hv, const double *T, const double *nu, const double *nuC, int nnu, int ncell,
                   const double *lut, int lut_n, double lut_xmax, cudaStream_t st);
void launch_phi_inv(int prec, const void *Hv, const double *dnu, int nnu, int ncell, int kmin, int kmax,
                    double *phi_inv, cudaStream_t st);
void launch_pd(size_t n, const double *nHII, const double *ne, const double *nHI, const double *nHeI,
               const double *nH2, const double *T, double z, double *out, cudaStream_t st);
void launch_mf(const double *dru_r, const double *dru_Z, double *f_r, double *f_Z, const double *js,
               const double *dV, const double *rCoM, const double *ZCoM, int nr, int nz, double dt,
               double z_center, double *partials, int nblocks, cudaStream_t st);
void launch_fesc(int prec, const void *Hr, const void *HZ, const double *A_r, const double *A_Z,
                 const double *dnu, int nnu, int nr, int nz, int bc_z_bot, double j_scale,
                 double *out, cudaStream_t st);
void launch_column_sums(const double *partials, int ncols, int nblocks, double *out, cudaStream_t st);
void launch_cfl(const double *r, const double *Z, const double *u_r, const double *u_Z, int nr, int nz,
                double c_tilde, double *out, cudaStream_t st);
void launch_edge(int prec, const void *J, const double *dnu, int nnu, int nr, int nz, double j_scale,
                 double *raw, double *norm, cudaStream_t st);
void build_voigt_lut(double *host, int n, double xmax);   // host: 5 tables of n entries

}  // namespace lyd
