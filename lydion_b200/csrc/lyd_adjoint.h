// lyd_adjoint.h -- argument blocks and launch wrappers of the reverse-mode kernels
// (lyd_adjoint.cu), used by the adjoint driver in lyd_api.cu. FP64, one cloud.
#pragma once
#include <cuda_runtime.h>

#include "lyd_internal.h"

namespace lyd {

// Frequency step adjoint: forward inputs (the step's input state s_n, the advection tape and
// the step's active window, from which the advected state x_A is rebuilt, and the per-cell
// fields), the adjoint of the step's output, and the outputs (adjoint of x_A, accumulated
// gradients).
struct FreqAdjArgs {
    const double *J, *Hr, *HZ;          // s_n (x_A outside the step's window)
    const double *tape;                 // [4][tape_stride] of the step's advection
    long long tape_stride;
    int kmin, kmax;                     // the step's active window
    const double *Fkp, *Fk, *Fkm;       // the step's frequency factors, or nullptr: recomputed
    const double *Hv, *phi, *phi_inv;   // phi: explicit profile or nullptr (derived from Hv)
    int phi_kmin, phi_kmax;
    const double *alpha, *alpha_c, *alpha_cF, *pd, *js, *T;
    const double *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;
    const double *nu, *nuC, *dnu, *inv_dnu, *inv_nuC, *dV;
    const CloudDesc *cl;
    const int4 *items;
    double alpha_floor, jeps, heps2, j_scale;
    int recoil, nnu;
    long long ncell;
    const double *gJ, *gHr, *gHZ;       // adjoint of the step output
    double *oJ, *oHr, *oHZ;             // adjoint of x_A (written)
    double *g_alpha, *g_alpha_c, *g_T;  // per cell (+=)
    double *g_u;                        // [5][ncell]: dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r (+=)
    double *g_Hv;                       // per cell-bin (+=)
    int mf_seed;                        // 1: add the adjoint of w * M_F of this step
    double mf_w;                        // w_MF * c / L
};

// Advection adjoint (cell and face kernels).
struct AdjAdvArgs {
    const double *J, *Hr, *HZ;          // the step's input state s_n
    const double *tape;                 // [4][n3] from the forward recomputation
    long long n3;
    const double *gJ, *gHr, *gHZ;       // adjoint of the advected state
    double *lJ, *lHr, *lHZ;             // adjoint of s_n (written by the cell kernel, += by faces)
    double *pJ, *pHr, *pHZ;             // adjoint of the flux-divergence sums, per cell-bin
    const double *Hv, *alpha, *alpha_cF;
    const double *A_r, *A_Z, *inv_dV, *inv_r_cell, *rint, *zint, *u_r_star, *u_Z_star;
    const double *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;
    double *g_aF;                       // per cell-bin (+=)
    double *g_u;                        // [5][ncell] (+=)
    double *g_ur, *g_uZ;                // face velocities (+=)
    int nnu, nr, nz, kmin, kmax;
    int bc_r_left, bc_r_right, bc_z_bot, bc_z_top;
    int flux;                           // 0 = GLF, 1 = HLL
    double ctdt, jeps, heps2;
};

void launch_freq_adj(const FreqAdjArgs &a, int nitems, cudaStream_t st);
void launch_adv_adj(const AdjAdvArgs &a, cudaStream_t st);
void launch_seed_spectrum(double *gJ, const double *w, int nnu, int nr, int nz, cudaStream_t st);
void launch_af_params(const double *g_aF, const double *alpha, const double *Hv, int nnu, long long ncell,
                      double *g_alpha, double *g_Hv, cudaStream_t st);
void launch_hvoigt_adj(const double *g_Hv, const double *T, const double *nu, const double *nuC, int nnu,
                       long long ncell, const double *lut, int lut_n, double lut_xmax, double *g_T, cudaStream_t st);

}  // namespace lyd
