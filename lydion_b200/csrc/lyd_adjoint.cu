// lyd_adjoint.cu -- reverse-mode kernels of the Lyman-alpha step (FP64, GLF or HLL flux, one cloud).
//
// One static-driver step maps the state s_n = (J, H_r, H_Z) to s_{n+1} through
//   A  AdvectLya!               s_n -> x_A        (active window of the step)
//   E  LyaEmissionAbsorption    x_A -> x_E
//   F  frequency factors, tridiagonal solve and flux correction   x_E -> s_{n+1}
// and the adjoint step maps lambda_{n+1} back to lambda_n while accumulating the gradients of
// the per-cell inputs. The kernels recompute the forward quantities they need from s_n and
// x_A (x_A is recomputed by the forward advection kernel, which also records its values
// before the floors and the causality limiter):
//   k_freq_adj      one warp per cell: E and F forward, then F^T (flux correction, transposed
//                   tridiagonal solve by the same warp PCR, frequency factors) and E^T
//   k_adv_adj_cell  one thread per cell-bin: the cell update's local terms and the adjoints
//                   of its face-flux sums
//   k_adv_adj_face  one thread per (face, active bin), the step's active bins packed densely
//                   across the threads: the adjoint of one face's reconstruction, closure and
//                   GLF/HLL + upwind flux, scattered onto its four stencil cells
// Scatters use FP64 atomics, so gradients agree run to run to rounding (~1e-15), not bitwise.
#include <cuda_runtime.h>

#include "lyd_adjoint.cuh"
#include "lyd_adjoint.h"
#include "lyd_internal.h"
#include "lyd_physics.cuh"

namespace lyd {

constexpr int ADJ_THREADS = 256;

__device__ __forceinline__ double wsum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Segmented warp sum: the lanes form runs of equal `key` (keys are contiguous runs across the
// warp). Returns, in the first lane of each run (head), the run's sum; other lanes get partial
// sums. Every lane of the warp must call it.
__device__ __forceinline__ double seg_sum(double v, long long key, int lane, bool &head) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double w = __shfl_down_sync(0xffffffffu, v, o);
        const long long kk = __shfl_down_sync(0xffffffffu, key, o);
        if (lane + o < 32 && kk == key) v += w;
    }
    const long long kp = __shfl_up_sync(0xffffffffu, key, 1);
    head = lane == 0 || kp != key;
    return v;
}

// ---- frequency step ------------------------------------------------------------------------

// Row r = lane*M + m of a warp-held tridiagonal system (sub a, diag b, super c, rhs d).
template <int M>
struct RowA {
    double a[M], b[M], c[M], d[M];
};

// v of row r-1 (dir = -1) or r+1 (dir = +1) for every owned row; outside the warp: idv.
template <int M>
__device__ __forceinline__ void nbr1(const double (&v)[M], double (&out)[M], int dir, int lane, double idv) {
#pragma unroll
    for (int m = 0; m < M; m++) {
        int mm = m + dir;
        if (mm >= 0 && mm < M) {
            out[m] = v[mm];
        } else {
            int src = mm < 0 ? M - 1 : 0;
            double got = dir < 0 ? __shfl_up_sync(0xffffffffu, v[src], 1) : __shfl_down_sync(0xffffffffu, v[src], 1);
            bool oob = dir < 0 ? (lane == 0) : (lane == 31);
            out[m] = oob ? idv : got;
        }
    }
}

template <int M>
__device__ __forceinline__ void nbrs(const double (&v)[M], double (&out)[M], int s, int dir, int lane, double idv) {
    if (s < M) {
#pragma unroll
        for (int m = 0; m < M; m++) {
            int mm = m + dir * s;
            if (mm >= 0 && mm < M) {
                out[m] = v[mm];
            } else {
                int src = mm < 0 ? mm + M : mm - M;
                double got = dir < 0 ? __shfl_up_sync(0xffffffffu, v[src], 1) : __shfl_down_sync(0xffffffffu, v[src], 1);
                bool oob = dir < 0 ? (lane == 0) : (lane == 31);
                out[m] = oob ? idv : got;
            }
        }
    } else {
        int t = s / M;
#pragma unroll
        for (int m = 0; m < M; m++) {
            double got = dir < 0 ? __shfl_up_sync(0xffffffffu, v[m], t) : __shfl_down_sync(0xffffffffu, v[m], t);
            bool oob = dir < 0 ? (lane < t) : (lane + t > 31);
            out[m] = oob ? idv : got;
        }
    }
}

// Parallel cyclic reduction of the warp's 32*M-row system; x returned in d.
template <int M>
__device__ __forceinline__ void pcr(RowA<M> &R_, int lane) {
#pragma unroll
    for (int s = 1; s < 32 * M; s <<= 1) {
        double ib[M];
#pragma unroll
        for (int m = 0; m < M; m++) ib[m] = rcp<double>(R_.b[m]);
        double am[M], cm[M], dm[M], ibm[M], ap[M], cp[M], dp[M], ibp[M];
        nbrs<M>(R_.a, am, s, -1, lane, 0.0);
        nbrs<M>(R_.c, cm, s, -1, lane, 0.0);
        nbrs<M>(R_.d, dm, s, -1, lane, 0.0);
        nbrs<M>(ib, ibm, s, -1, lane, 1.0);
        nbrs<M>(R_.a, ap, s, +1, lane, 0.0);
        nbrs<M>(R_.c, cp, s, +1, lane, 0.0);
        nbrs<M>(R_.d, dp, s, +1, lane, 0.0);
        nbrs<M>(ib, ibp, s, +1, lane, 1.0);
#pragma unroll
        for (int m = 0; m < M; m++) {
            double al = -R_.a[m] * ibm[m];
            double ga = -R_.c[m] * ibp[m];
            double nb = R_.b[m] + al * cm[m] + ga * ap[m];
            double nd = R_.d[m] + al * dm[m] + ga * dp[m];
            R_.a[m] = al * am[m];
            R_.c[m] = ga * cp[m];
            R_.b[m] = nb;
            R_.d[m] = nd;
        }
    }
#pragma unroll
    for (int m = 0; m < M; m++) R_.d[m] = R_.d[m] * rcp<double>(R_.b[m]);
}

// Two rows per lane: one cyclic-reduction step over the odd rows, PCR across the warp on the
// even rows, back-substitution of the odd rows (the same scheme as the forward frequency
// kernel's two-bins-per-lane solve).
__device__ __forceinline__ void cr_pcr2(RowA<2> &R_, int lane) {
    const double ibo = rcp<double>(R_.b[1]);
    double a_om = __shfl_up_sync(0xffffffffu, R_.a[1], 1);
    double c_om = __shfl_up_sync(0xffffffffu, R_.c[1], 1);
    double d_om = __shfl_up_sync(0xffffffffu, R_.d[1], 1);
    double ib_om = __shfl_up_sync(0xffffffffu, ibo, 1);
    if (lane == 0) { a_om = 0.0; c_om = 0.0; d_om = 0.0; ib_om = 1.0; }
    double al = -R_.a[0] * ib_om, ga = -R_.c[0] * ibo;
    double ea = al * a_om;
    double eb = R_.b[0] + al * c_om + ga * R_.a[1];
    double ec = ga * R_.c[1];
    double ed = R_.d[0] + al * d_om + ga * R_.d[1];
    // PCR over the even rows, each scaled to a unit diagonal (three values per neighbour)
    double ib = rcp<double>(eb);
    double na = ea * ib, nc = ec * ib, nd = ed * ib;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        double am = __shfl_up_sync(0xffffffffu, na, s), cm = __shfl_up_sync(0xffffffffu, nc, s);
        double dm = __shfl_up_sync(0xffffffffu, nd, s);
        double ap = __shfl_down_sync(0xffffffffu, na, s), cp = __shfl_down_sync(0xffffffffu, nc, s);
        double dp = __shfl_down_sync(0xffffffffu, nd, s);
        if (lane < s) { am = 0.0; cm = 0.0; dm = 0.0; }
        if (lane + s > 31) { ap = 0.0; cp = 0.0; dp = 0.0; }
        eb = fma(-na, cm, fma(-nc, ap, 1.0));
        const double a2 = -na * am, c2 = -nc * cp;
        const double d2 = fma(-na, dm, fma(-nc, dp, nd));
        ib = rcp<double>(eb);
        na = a2 * ib;
        nc = c2 * ib;
        nd = d2 * ib;
    }
    const double xe = nd;
    double xe2 = __shfl_down_sync(0xffffffffu, xe, 1);
    if (lane == 31) xe2 = 0.0;
    R_.d[0] = xe;
    R_.d[1] = (R_.d[1] - R_.a[1] * xe - R_.c[1] * xe2) * ibo;
}

template <int M>
__device__ __forceinline__ void solve(RowA<M> &R_, int lane) {
    if constexpr (M == 2) cr_pcr2(reinterpret_cast<RowA<2> &>(R_), lane);
    else pcr<M>(R_, lane);
}

// Frequency factors F+, F, F- of one row k (src/FreqFactors.jl:181-275) and, with g != 0,
// their adjoint: returns the adjoints of vel, K_{k-1}, K_k, K_{k+1} and rec0.
struct FfIn {
    double vel, Kkm, Kk, Kkp, nCkm, nCk, nCkp, ICkm, ICk, ICkp, DNKM, DNK, DNKP, idn, rec0;
    int recoil;
};

// phi / chi of one P and their P-derivatives with one exponential and one reciprocal
// (OneMinusphi_L/R_and_chi_L/R, src/FreqFactors.jl:54-133). L: omp = e^-P, chi = (1 - omp)/P;
// R: omp = e^P, chi = (1 - omp)/P; the clamp and Taylor branches as the forward takes them.
// The exponentials are exp_tab's, as in the forward, with its table at `tab`.
struct Omphi { double o, x, d_o, d_x; };
template <bool LEFT>
__device__ __forceinline__ Omphi omphi_d(double P, const double *tab) {
    Omphi r;
    const double sg = LEFT ? -1.0 : 1.0;
    if (P >= kPmax || P <= -kPmax) {
        const double Pc = P >= kPmax ? kPmax : -kPmax;
        r.o = exp_tab(sg * Pc, tab);
        r.x = (1.0 - r.o) / Pc;
        r.d_o = 0.0; r.d_x = 0.0;
        return r;
    }
    if (fabs(P) < kPmin) {
        r.o = 1.0 + sg * P + 0.5 * (P * P);
        r.x = -sg - 0.5 * P;
        r.d_o = sg + P;
        r.d_x = -0.5;
        return r;
    }
    r.o = exp_tab(sg * P, tab);
    const double iP = rcp<double>(P);
    r.x = (1.0 - r.o) * iP;
    r.d_o = sg * r.o;
    r.d_x = (-r.d_o - r.x) * iP;
    return r;
}
// Both sides of the same P: e^P = 1 / e^-P and one reciprocal of P serve the two.
__device__ __forceinline__ void omphi_d_LR(double P, Omphi &L, Omphi &R_, const double *tab) {
    if (P >= kPmax || P <= -kPmax || fabs(P) < kPmin) {
        L = omphi_d<true>(P, tab);
        R_ = omphi_d<false>(P, tab);
        return;
    }
    const double e = exp_tab(-P, tab), ie = rcp<double>(e), iP = rcp<double>(P);
    L.o = e; L.x = (1.0 - e) * iP; L.d_o = -e; L.d_x = (e - L.x) * iP;
    R_.o = ie; R_.x = (1.0 - ie) * iP; R_.d_o = ie; R_.d_x = (-ie - R_.x) * iP;
}

// `tab`: exp_tab's table (the forward frequency kernel's exponentials).
__device__ __forceinline__ void ff_fwd(const FfIn &q, double &Fp, double &F0, double &Fm, const double *tab) {
    double iKkm = rcp<double>(q.Kkm), iKk = rcp<double>(q.Kk), iKkp = rcp<double>(q.Kkp);
    double Ckp = q.vel * q.nCkp, Ck = q.vel * q.nCk, Ckm = q.vel * q.nCkm;
    if (q.recoil) {
        Ckp += q.Kkp * (q.rec0 - 2.0 * q.ICkp);
        Ck += q.Kk * (q.rec0 - 2.0 * q.ICk);
        Ckm += q.Kkm * (q.rec0 - 2.0 * q.ICkm);
    }
    double rkp = q.DNKP * iKkp, rk = q.DNK * iKk, rkm = q.DNKM * iKkm;
    double Pkp = fmin(fmax(Ckp * rkp, -kPmax), kPmax);
    double Pk = fmin(fmax(Ck * rk, -kPmax), kPmax);
    double Pkm = fmin(fmax(Ckm * rkm, -kPmax), kPmax);
    double oRkp, xRkp, oLk, xLk, oRk, xRk, oLkm, xLkm;
    omphi_R(Pkp, oRkp, xRkp, tab);
    omphi_LR(Pk, oLk, xLk, oRk, xRk, tab);
    omphi_L(Pkm, oLkm, xLkm, tab);
    double dkp = q.idn * rcp<double>(xLk * rk - xRkp * rkp);
    double dkm = q.idn * rcp<double>(xLkm * rkm - xRk * rk);
    Fp = oRkp * dkp;
    Fm = oLkm * dkm;
    F0 = oLk * dkp + oRk * dkm;
}

__device__ __forceinline__ void ff_adj(const FfIn &q, double gFp, double gF0, double gFm, double &gvel, double &gKkm,
                                       double &gKk, double &gKkp, double &grec0, const double *tab) {
    double iKkm = rcp<double>(q.Kkm), iKk = rcp<double>(q.Kk), iKkp = rcp<double>(q.Kkp);
    double Ckp = q.vel * q.nCkp, Ck = q.vel * q.nCk, Ckm = q.vel * q.nCkm;
    const double ekp = q.rec0 - 2.0 * q.ICkp, ek = q.rec0 - 2.0 * q.ICk, ekm = q.rec0 - 2.0 * q.ICkm;
    if (q.recoil) {
        Ckp += q.Kkp * ekp;
        Ck += q.Kk * ek;
        Ckm += q.Kkm * ekm;
    }
    double rkp = q.DNKP * iKkp, rk = q.DNK * iKk, rkm = q.DNKM * iKkm;
    double Pkp0 = Ckp * rkp, Pk0 = Ck * rk, Pkm0 = Ckm * rkm;
    double Pkp = fmin(fmax(Pkp0, -kPmax), kPmax);
    double Pk = fmin(fmax(Pk0, -kPmax), kPmax);
    double Pkm = fmin(fmax(Pkm0, -kPmax), kPmax);
    const Omphi Rkp = omphi_d<false>(Pkp, tab), Lkm = omphi_d<true>(Pkm, tab);
    Omphi Lk, Rk;
    omphi_d_LR(Pk, Lk, Rk, tab);
    double Dp = Lk.x * rk - Rkp.x * rkp, Dm = Lkm.x * rkm - Rk.x * rk;
    const double iDp = rcp<double>(Dp), iDm = rcp<double>(Dm);
    double dkp = q.idn * iDp, dkm = q.idn * iDm;
    // F+ = oR(Pkp) dkp ; F- = oL(Pkm) dkm ; F = oL(Pk) dkp + oR(Pk) dkm
    double gdkp = gFp * Rkp.o + gF0 * Lk.o;
    double gdkm = gFm * Lkm.o + gF0 * Rk.o;
    double goRkp = gFp * dkp, goLkm = gFm * dkm, goLk = gF0 * dkp, goRk = gF0 * dkm;
    double gDp = -gdkp * dkp * iDp, gDm = -gdkm * dkm * iDm;
    double gxLk = gDp * rk, gxRkp = -gDp * rkp, gxLkm = gDm * rkm, gxRk = -gDm * rk;
    double grk = gDp * Lk.x - gDm * Rk.x, grkp = -gDp * Rkp.x, grkm = gDm * Lkm.x;
    double gPkp = goRkp * Rkp.d_o + gxRkp * Rkp.d_x;
    double gPk = goLk * Lk.d_o + gxLk * Lk.d_x + goRk * Rk.d_o + gxRk * Rk.d_x;
    double gPkm = goLkm * Lkm.d_o + gxLkm * Lkm.d_x;
    // clamps pass nothing when active
    if (!(Pkp0 > -kPmax && Pkp0 < kPmax)) gPkp = 0.0;
    if (!(Pk0 > -kPmax && Pk0 < kPmax)) gPk = 0.0;
    if (!(Pkm0 > -kPmax && Pkm0 < kPmax)) gPkm = 0.0;
    double gCkp = gPkp * rkp, gCk = gPk * rk, gCkm = gPkm * rkm;
    grkp += gPkp * Ckp; grk += gPk * Ck; grkm += gPkm * Ckm;
    double giKkp = grkp * q.DNKP, giKk = grk * q.DNK, giKkm = grkm * q.DNKM;
    gKkp += -giKkp * iKkp * iKkp;
    gKk += -giKk * iKk * iKk;
    gKkm += -giKkm * iKkm * iKkm;
    gvel += gCkp * q.nCkp + gCk * q.nCk + gCkm * q.nCkm;
    if (q.recoil) {
        gKkp += gCkp * ekp;
        gKk += gCk * ek;
        gKkm += gCkm * ekm;
        grec0 += gCkp * q.Kkp + gCk * q.Kk + gCkm * q.Kkm;
    }
}

// 2 CTAs per SM (128 registers, a few hundred bytes of spills) measured 1.7x faster than the
// unconstrained 202-register form at 1 CTA per SM.
template <int M>
__global__ void __launch_bounds__(ADJ_THREADS, 2) k_freq_adj(FreqAdjArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nnu = a.nnu;
    const int4 it = a.items[blockIdx.x];
    const CloudDesc &cd = a.cl[it.x];
    const double c_tilde = cd.c_tilde, dt = cd.dt, ctdt = cd.ctdt;
    const double jeps = a.jeps, dw = 1.0 / ctdt;
    __shared__ double etab[32];
    if (threadIdx.x < 32) etab[threadIdx.x] = kExp2Tab[threadIdx.x];
    __syncthreads();
    for (int cl = it.y + warp; cl < it.z; cl += nw) {
        const long long c = cd.oc + cl;
        const long long base = cd.o3 + (long long)cl * nnu;
        double JA[M], HrA[M], HZA[M], Hv[M], dn[M];
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            bool v = k < nnu;
            Hv[m] = v ? a.Hv[base + k] : 1.0;
            dn[m] = v ? a.dnu[k] : 0.0;
            if (v && k >= a.kmin && k <= a.kmax) {
                // x_A from the advection's tape: the second J floor and the causality limiter
                // of the cell update, as k_advect applies them
                const double t1 = a.tape[base + k + a.tape_stride];
                double hr = a.tape[base + k + 2 * a.tape_stride], hz = a.tape[base + k + 3 * a.tape_stride];
                const double Jn = t1 > jeps ? t1 : jeps;
                const double H2 = hr * hr + hz * hz;
                if (H2 > Jn * Jn) {
                    const double fsc = Jn * rsqrt_nr(H2);
                    hr *= fsc;
                    hz *= fsc;
                }
                JA[m] = Jn; HrA[m] = hr; HZA[m] = hz;
            } else {
                JA[m] = v ? a.J[base + k] : 0.0;
                HrA[m] = v ? a.Hr[base + k] : 0.0;
                HZA[m] = v ? a.HZ[base + k] : 0.0;
            }
        }
        // ---- emission / absorption forward, src/ConstantsAndFunctions.jl:526-567 ----
        const double al = a.alpha[c], acv = a.alpha_c[c], pdv = a.pd[c];
        const double al_pd = al * pdv;
        const double js_ct = a.js[c] * c_tilde / a.j_scale;
        const double pinv = a.phi ? 0.0 : a.phi_inv[c];
        const double acF = a.alpha_cF ? a.alpha_cF[c] : 0.0;
        double J1[M], Hr1[M], HZ1[M], eden[M], idn[M], phi[M];
        double dr_sum = 0.0, dz_sum = 0.0;
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            phi[m] = (k >= nnu) ? 0.0
                     : (a.phi ? a.phi[base + k] : ((k >= a.phi_kmin && k <= a.phi_kmax) ? Hv[m] * pinv : 0.0));
            double aabs = acv + al_pd * Hv[m];
            double dJdt = js_ct * phi[m];
            eden[m] = rcp<double>(1.0 + aabs * c_tilde * dt);     // held as its reciprocal
            J1[m] = (JA[m] + dJdt * dt) * eden[m];
            double aH = a.alpha_cF ? al * Hv[m] + acF : al * Hv[m];
            idn[m] = rcp<double>(1.0 + aH * c_tilde * dt);
            Hr1[m] = HrA[m] * idn[m];
            HZ1[m] = HZA[m] * idn[m];
            if (k < nnu) {
                dr_sum += dn[m] * (HrA[m] - Hr1[m]);
                dz_sum += dn[m] * (HZA[m] - HZ1[m]);
            } else {
                J1[m] = 0.0; Hr1[m] = 0.0; HZ1[m] = 0.0;
            }
        }
        // ---- frequency factors forward ----
        const double T = a.T[c];
        const double dnuD = compute_dnuD(T);
        const double alv = al;
        const double pref = 0.5 * (alv > a.alpha_floor ? alv : a.alpha_floor) * (dnuD * dnuD);
        const double rec0 = kHOverKB / T;
        const double gu0 = a.dur_dr[c], gu1 = a.dur_dZ[c], gu2 = a.duZ_dr[c], gu3 = a.duZ_dZ[c], gu4 = a.ur_over_r[c];
        double Kb[M];
#pragma unroll
        for (int m = 0; m < M; m++) Kb[m] = pref * Hv[m];
        double Km[M], Kp[M];
        nbr1<M>(Kb, Km, -1, lane, 1.0);
        nbr1<M>(Kb, Kp, +1, lane, 1.0);
        RowA<M> sys;
        double Fp[M], F0[M], Fm[M], vel[M];
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            Fp[m] = F0[m] = Fm[m] = 0.0;
            vel[m] = 0.0;
            if (k >= 1 && k <= nnu - 2) {
                double Drr, DZZ, DrZ;
                D_edd<double>(Hr1[m], HZ1[m], J1[m], jeps, a.heps2, Drr, DZZ, DrZ);
                vel[m] = d_colon_grad_u<double>(Drr, DrZ, DZZ, gu0, gu1, gu2, gu3, gu4) * kInvC;
                if (a.Fkp) {
                    // the factors the forward sweep stored
                    Fp[m] = a.Fkp[base + k]; F0[m] = a.Fk[base + k]; Fm[m] = a.Fkm[base + k];
                } else {
                    FfIn q;
                    q.vel = vel[m]; q.Kkm = Km[m]; q.Kk = Kb[m]; q.Kkp = Kp[m];
                    q.nCkm = a.nuC[k - 1]; q.nCk = a.nuC[k]; q.nCkp = a.nuC[k + 1];
                    q.ICkm = a.inv_nuC[k - 1]; q.ICk = a.inv_nuC[k]; q.ICkp = a.inv_nuC[k + 1];
                    q.DNKM = a.nu[k] - a.nuC[k - 1]; q.DNK = a.nu[k + 1] - a.nuC[k];
                    q.DNKP = a.nuC[k + 1] - a.nu[k + 1];
                    q.idn = a.inv_dnu[k]; q.rec0 = rec0; q.recoil = a.recoil;
                    ff_fwd(q, Fp[m], F0[m], Fm[m], etab);
                }
            }
            bool in = (k >= 1 && k <= nnu - 2);
            sys.a[m] = (in && k >= 2) ? Fm[m] : 0.0;
            sys.b[m] = in ? -(F0[m] + dw) : 1.0;
            sys.c[m] = (in && k <= nnu - 3) ? Fp[m] : 0.0;
            sys.d[m] = in ? -dw * J1[m] : 0.0;
        }
        double sa[M], sb[M], sc[M];
#pragma unroll
        for (int m = 0; m < M; m++) { sa[m] = sys.a[m]; sb[m] = sys.b[m]; sc[m] = sys.c[m]; }
        solve<M>(sys, lane);
        double x[M];
#pragma unroll
        for (int m = 0; m < M; m++) x[m] = sys.d[m];

        // ---- reverse: flux correction, src/UpdateLyaJandH.jl:341-377 ----
        double gx[M], gJ1[M], gHr1[M], gHZ1[M];
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            gx[m] = gJ1[m] = gHr1[m] = gHZ1[m] = 0.0;
            if (k >= nnu) continue;
            bool in = (k >= 1 && k <= nnu - 2);
            double Jn = in ? x[m] : J1[m];
            double Jf = Jn > jeps ? Jn : jeps;
            double Jod = J1[m] > jeps ? J1[m] : jeps;
            const double iJod = rcp<double>(Jod);
            double ratio = Jf * iJod;
            double hr = Hr1[m] * ratio, hz = HZ1[m] * ratio;
            double H2 = hr * hr + hz * hz;
            double gJo = a.gJ[base + k], gHo = a.gHr[base + k], gZo = a.gHZ[base + k];
            double ghr, ghz, gJf = gJo;
            if (H2 > Jf * Jf) {
                double h = sqrt(H2);
                double nr = hr / h, nz = hz / h, s = Jf / h;
                double dot = nr * gHo + nz * gZo;
                ghr = s * (gHo - nr * dot);
                ghz = s * (gZo - nz * dot);
                gJf += dot;
            } else {
                ghr = gHo;
                ghz = gZo;
            }
            gHr1[m] = ghr * ratio;
            gHZ1[m] = ghz * ratio;
            double gratio = ghr * Hr1[m] + ghz * HZ1[m];
            gJf += gratio * iJod;
            if (J1[m] > jeps) gJ1[m] += -gratio * ratio * iJod;
            double gJn = Jn > jeps ? gJf : 0.0;
            if (in) gx[m] = gJn;
            else gJ1[m] += gJn;
        }
        // ---- reverse: tridiagonal solve A x = d (rows k = 1..nnu-2), A^T mu = g_x ----
        {
            double cm1[M], ap1[M];
            nbr1<M>(sc, cm1, -1, lane, 0.0);
            nbr1<M>(sa, ap1, +1, lane, 0.0);
            RowA<M> tr;
#pragma unroll
            for (int m = 0; m < M; m++) {
                tr.a[m] = cm1[m];
                tr.b[m] = sb[m];
                tr.c[m] = ap1[m];
                tr.d[m] = gx[m];
            }
            solve<M>(tr, lane);
            double xm[M], xp[M];
            nbr1<M>(x, xm, -1, lane, 0.0);
            nbr1<M>(x, xp, +1, lane, 0.0);
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                bool in = (k >= 1 && k <= nnu - 2);
                double mu = tr.d[m];
                if (!in) { Fp[m] = F0[m] = Fm[m] = 0.0; continue; }
                gJ1[m] += -dw * mu;
                // reuse Fp/F0/Fm as their adjoints
                Fm[m] = (k >= 2) ? -mu * xm[m] : 0.0;
                F0[m] = mu * x[m];                    // b = -(F0 + dw): gF0 = -gb = mu x
                Fp[m] = (k <= nnu - 3) ? -mu * xp[m] : 0.0;
            }
        }
        // ---- reverse: frequency factors ----
        double gKown[M], gKtoP[M], gKtoM[M];
        double grec0 = 0.0, gu[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            gKown[m] = gKtoP[m] = gKtoM[m] = 0.0;
            if (!(k >= 1 && k <= nnu - 2)) continue;
            FfIn q;
            q.vel = vel[m]; q.Kkm = Km[m]; q.Kk = Kb[m]; q.Kkp = Kp[m];
            q.nCkm = a.nuC[k - 1]; q.nCk = a.nuC[k]; q.nCkp = a.nuC[k + 1];
            q.ICkm = a.inv_nuC[k - 1]; q.ICk = a.inv_nuC[k]; q.ICkp = a.inv_nuC[k + 1];
            q.DNKM = a.nu[k] - a.nuC[k - 1]; q.DNK = a.nu[k + 1] - a.nuC[k]; q.DNKP = a.nuC[k + 1] - a.nu[k + 1];
            q.idn = a.inv_dnu[k]; q.rec0 = rec0; q.recoil = a.recoil;
            double gvel = 0.0;
            ff_adj(q, Fp[m], F0[m], Fm[m], gvel, gKtoM[m], gKown[m], gKtoP[m], grec0, etab);
            // vel = D:grad u / c with D from (H_r, H_Z, J) after emission
            double Drr, DZZ, DrZ;
            D_edd<double>(Hr1[m], HZ1[m], J1[m], jeps, a.heps2, Drr, DZZ, DrZ);
            double gDrr = 0.0, gDrZ = 0.0, gDZZ = 0.0;
            adj_d_colon_grad_u(Drr, DrZ, DZZ, gu0, gu1, gu2, gu3, gu4, gvel * kInvC, gDrr, gDrZ, gDZZ, gu);
            adj_D_edd(Hr1[m], HZ1[m], J1[m], jeps, a.heps2, gDrr, gDZZ, gDrZ, gHr1[m], gHZ1[m], gJ1[m]);
        }
        // K_k collects its own row's adjoint and those of rows k-1 (as K_{k+1}) and k+1 (as K_{k-1})
        double fromM[M], fromP[M];
        nbr1<M>(gKtoP, fromM, -1, lane, 0.0);
        nbr1<M>(gKtoM, fromP, +1, lane, 0.0);
        double gHv[M], gpref = 0.0;
#pragma unroll
        for (int m = 0; m < M; m++) {
            double gK = gKown[m] + fromM[m] + fromP[m];
            gHv[m] = gK * pref;
            gpref += gK * Hv[m];
        }
        // ---- reverse: emission / absorption (and the M_F seed of the last step) ----
        double galpha = 0.0, galpha_c = 0.0, gpinv = 0.0;
        if (a.mf_seed) {
            double drs = wsum_d(dr_sum), dzs = wsum_d(dz_sum);
            const double k4 = kFourPiOverC * (1.0 / c_tilde) * a.j_scale;
            double fr = k4 * drs / dt, fz = k4 * dzs / dt;
            double fm = sqrt(fr * fr + fz * fz);
            if (fm > 0.0) {
                double w = a.mf_w * a.dV[c] / fm;
                double gdr = w * fr * k4 / dt, gdz = w * fz * k4 / dt;
#pragma unroll
                for (int m = 0; m < M; m++) {
                    gHr1[m] -= gdr * dn[m];
                    gHZ1[m] -= gdz * dn[m];
                    HrA[m] = gdr * dn[m];        // reused: direct adjoint of H_A through dru
                    HZA[m] = gdz * dn[m];
                }
            } else {
#pragma unroll
                for (int m = 0; m < M; m++) { HrA[m] = 0.0; HZA[m] = 0.0; }
            }
        } else {
#pragma unroll
            for (int m = 0; m < M; m++) { HrA[m] = 0.0; HZA[m] = 0.0; }
        }
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            if (k >= nnu) continue;
            // recover H_A (the arrays were reused for the M_F adjoint)
            const double hden = 1.0 + (a.alpha_cF ? al * Hv[m] + acF : al * Hv[m]) * c_tilde * dt;
            double hrA = Hr1[m] * hden, hzA = HZ1[m] * hden;
            double gHrA = gHr1[m] * idn[m] + HrA[m];
            double gHZA = gHZ1[m] * idn[m] + HZA[m];
            double gidn = gHr1[m] * hrA + gHZ1[m] * hzA;
            double gaH = -gidn * idn[m] * idn[m] * c_tilde * dt;
            galpha += gaH * Hv[m];
            gHv[m] += gaH * al;
            double gJA = gJ1[m] * eden[m];
            double gdJdt = gJ1[m] * eden[m] * dt;
            double gaabs = -gJ1[m] * J1[m] * eden[m] * c_tilde * dt;
            galpha_c += gaabs;
            galpha += gaabs * pdv * Hv[m];
            gHv[m] += gaabs * al_pd;
            double gphi = gdJdt * js_ct;
            if (!a.phi && k >= a.phi_kmin && k <= a.phi_kmax) {
                gHv[m] += gphi * pinv;
                gpinv += gphi * Hv[m];
            }
            a.oJ[base + k] = gJA;
            a.oHr[base + k] = gHrA;
            a.oHZ[base + k] = gHZA;
        }
        gpinv = wsum_d(gpinv);
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            if (k >= nnu) continue;
            if (!a.phi && k >= a.phi_kmin && k <= a.phi_kmax) gHv[m] += -gpinv * pinv * pinv * dn[m];
            a.g_Hv[base + k] += gHv[m];
        }
        galpha = wsum_d(galpha);
        galpha_c = wsum_d(galpha_c);
        gpref = wsum_d(gpref);
        grec0 = wsum_d(grec0);
#pragma unroll
        for (int q = 0; q < 5; q++) gu[q] = wsum_d(gu[q]);
        if (lane == 0) {
            if (alv > a.alpha_floor) galpha += gpref * 0.5 * dnuD * dnuD;
            a.g_alpha[c] += galpha;
            a.g_alpha_c[c] += galpha_c;
            // pref ~ dnuD^2 ~ T ; rec0 = h / (k_B T)
            a.g_T[c] += gpref * pref / T - grec0 * rec0 / T;
#pragma unroll
            for (int q = 0; q < 5; q++) a.g_u[(size_t)q * a.ncell + c] += gu[q];
        }
    }
}

// ---- advection -----------------------------------------------------------------------------

// A stencil cell read from the step's input state with the ghost-cell rules of
// src/AdvectJandH.jl:662-673, 853-871 (r) and 1000-1018, 1185-1203 (Z): the value, the
// in-grid cell it comes from, and the factors its H components were multiplied by.
struct GCell {
    double J, Hr, HZ;
    int i, j;
    double sHr, sHZ;
};

__device__ __forceinline__ GCell gcell(const AdjAdvArgs &a, int i, int j, int k) {
    GCell g;
    g.sHr = 1.0; g.sHZ = 1.0;
    const int nr = a.nr, nz = a.nz;
    if (i < 0) { if (a.bc_r_left == 0) { g.i = -1 - i; g.sHr = -1.0; } else { g.i = 0; g.sHr = -2.0; } }
    else if (i >= nr) { if (a.bc_r_right == 0) { g.i = 2 * nr - 1 - i; g.sHr = -1.0; } else { g.i = nr - 1; g.sHr = 2.0; } }
    else g.i = i;
    if (j < 0) { if (a.bc_z_bot == 0) { g.j = -1 - j; g.sHZ = -1.0; } else { g.j = 0; g.sHZ = -2.0; } }
    else if (j >= nz) { if (a.bc_z_top == 0) { g.j = 2 * nz - 1 - j; g.sHZ = -1.0; } else { g.j = nz - 1; g.sHZ = 2.0; } }
    else g.j = j;
    long long x = (long long)k + (long long)a.nnu * ((long long)g.i + (long long)nr * g.j);
    g.J = a.J[x];
    double hr = a.Hr[x], hz = a.HZ[x];
    // outflow ghosts keep only the outgoing sign: 2.0 marks max(H, 0), -2.0 min(H, 0)
    if (g.sHr == 2.0) { g.sHr = hr > 0.0 ? 1.0 : 0.0; }
    else if (g.sHr == -2.0) { g.sHr = hr < 0.0 ? 1.0 : 0.0; }
    if (g.sHZ == 2.0) { g.sHZ = hz > 0.0 ? 1.0 : 0.0; }
    else if (g.sHZ == -2.0) { g.sHZ = hz < 0.0 ? 1.0 : 0.0; }
    g.Hr = g.sHr * hr;
    g.HZ = g.sHZ * hz;
    return g;
}

__device__ __forceinline__ double alpha_F_at(const AdjAdvArgs &a, int i, int j, int k) {
    long long c = (long long)i + (long long)a.nr * j;
    double v = a.alpha[c] * a.Hv[(long long)k + (long long)a.nnu * c];
    if (a.alpha_cF) v += a.alpha_cF[c];
    return v;
}

// Cell update adjoint (src/AdvectJandH.jl:1302-1382 reversed): warp = one cell x 32 bins.
// One thread per cell-bin, cell-major (a warp may span two or three cells).
__global__ void __launch_bounds__(ADJ_THREADS) k_adv_adj_cell(AdjAdvArgs a) {
    const int lane = threadIdx.x & 31;
    const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ncell = (long long)a.nr * a.nz;
    const bool valid = item < ncell * a.nnu;
    const long long c = valid ? item / a.nnu : -1;
    const int k = valid ? (int)(item % a.nnu) : 0;
    const int i = valid ? (int)(c % a.nr) : 0;
    const bool act = valid && k >= a.kmin && k <= a.kmax;
    const long long x = (long long)k + (long long)a.nnu * c;
    double gu[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (valid && !act) {
        a.lJ[x] = a.gJ[x]; a.lHr[x] = a.gHr[x]; a.lHZ[x] = a.gHZ[x];
        a.pJ[x] = 0.0; a.pHr[x] = 0.0; a.pHZ[x] = 0.0;
    } else if (act) {
        const double jeps = a.jeps, ctdt = a.ctdt, cc = ctdt * kInvC;
        const double sJ = a.J[x], sHr = a.Hr[x], sHZ = a.HZ[x];
        const double Jn0 = a.tape[x], Jn1b = a.tape[x + a.n3], Hrp = a.tape[x + 2 * a.n3], HZp = a.tape[x + 3 * a.n3];
        const double ga = a.dur_dr[c], gb = a.dur_dZ[c], gc = a.duZ_dr[c], gd = a.duZ_dZ[c], ge = a.ur_over_r[c];
        double gJo = a.gJ[x], gHo = a.gHr[x], gZo = a.gHZ[x];
        // causality limiter
        double J2 = Jn1b > jeps ? Jn1b : jeps;
        double H2 = Hrp * Hrp + HZp * HZp;
        double gHrp, gHZp, gJ2 = gJo;
        if (H2 > J2 * J2) {
            double h = sqrt(H2);
            double nr = Hrp / h, nz = HZp / h, s = J2 / h;
            double dot = nr * gHo + nz * gZo;
            gHrp = s * (gHo - nr * dot);
            gHZp = s * (gZo - nz * dot);
            gJ2 += dot;
        } else {
            gHrp = gHo;
            gHZp = gZo;
        }
        double gJn1 = Jn1b > jeps ? gJ2 : 0.0;
        // J after the first floor minus c~dt/c D:grad u J
        double Drr, DZZ, DrZ;
        D_edd<double>(sHr, sHZ, sJ, jeps, a.heps2, Drr, DZZ, DrZ);
        double DdU = d_colon_grad_u<double>(Drr, DrZ, DZZ, ga, gb, gc, gd, ge);
        double gsJ = -gJn1 * cc * DdU, gsHr = 0.0, gsHZ = 0.0;
        double gDdU = -gJn1 * cc * sJ;
        double gJn0 = Jn0 > jeps ? gJn1 : 0.0;
        // aberration terms dH = -c~dt/c (H . grad u)
        gsHr += -cc * (gHrp * ga + gHZp * gc);
        gsHZ += -cc * (gHrp * gb + gHZp * gd);
        gu[0] += -cc * gHrp * sHr;
        gu[1] += -cc * gHrp * sHZ;
        gu[2] += -cc * gHZp * sHr;
        gu[3] += -cc * gHZp * sHZ;
        double gDrr = 0.0, gDrZ = 0.0, gDZZ = 0.0;
        adj_d_colon_grad_u(Drr, DrZ, DZZ, ga, gb, gc, gd, ge, gDdU, gDrr, gDrZ, gDZZ, gu);
        adj_D_edd(sHr, sHZ, sJ, jeps, a.heps2, gDrr, gDZZ, gDrZ, gsHr, gsHZ, gsJ);
        // identity parts of Q - c~dt/dV sum(A F)
        gsJ += gJn0;
        gsHr += gHrp;
        gsHZ += gHZp;
        a.lJ[x] = gsJ; a.lHr[x] = gsHr; a.lHZ[x] = gsHZ;
        a.pJ[x] = gJn0; a.pHr[x] = gHrp; a.pHZ[x] = gHZp;
    }
    (void)i;
    bool head = false;
#pragma unroll
    for (int q = 0; q < 5; q++) gu[q] = seg_sum(gu[q], c, lane, head);
    if (valid && head)
#pragma unroll
        for (int q = 0; q < 5; q++)
            if (gu[q] != 0.0) atomicAdd(a.g_u + (size_t)q * ncell + c, gu[q]);
}

// One face's adjoint: thread = one face x one active bin. ZDIR false: r faces f = 0..nr of
// row j; true: Z faces f = 0..nz of column i.
// 2 CTAs per SM: 1.4x faster than the unconstrained 206-register form.
template <bool ZDIR, int FLUX>
__global__ void __launch_bounds__(ADJ_THREADS, 2) k_adv_adj_face(AdjAdvArgs a) {
    const int lane = threadIdx.x & 31;
    const long long item = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nact = a.kmax - a.kmin + 1;          // the step's active bins, packed densely
    const int nr = a.nr, nz = a.nz;
    const long long nfaces = ZDIR ? (long long)nr * (nz + 1) : (long long)(nr + 1) * nz;
    const bool act = nact > 0 && item < nfaces * nact;
    const long long fi = act ? item / nact : -1;
    const int k = act ? a.kmin + (int)(item % nact) : 0;
    // r face: fi = f + (nr+1) j ; Z face: fi = i + nr f
    const int f = !act ? 0 : (ZDIR ? (int)(fi / nr) : (int)(fi % (nr + 1)));
    const int line = !act ? 0 : (ZDIR ? (int)(fi % nr) : (int)(fi / (nr + 1)));
    double guc = 0.0;
    if (act) {
        const double ctdt = a.ctdt;
        // the two cells sharing the face: lower (f-1) and upper (f) along the sweep direction
        const bool lo = f >= 1, hi = ZDIR ? f <= nz - 1 : f <= nr - 1;
        auto cidx = [&](int p) -> long long { return ZDIR ? (long long)line + (long long)nr * p : (long long)p + (long long)nr * line; };
        const double Af = ZDIR ? a.A_Z[fi] : a.A_r[fi];
        double gF[3] = {0.0, 0.0, 0.0}, gkL = 0.0, gkR = 0.0;
        if (lo) {
            long long cl = cidx(f - 1), xl = (long long)k + (long long)a.nnu * cl;
            double w = -ctdt * a.inv_dV[cl] * Af;
            gF[0] += w * a.pJ[xl]; gF[1] += w * a.pHr[xl]; gF[2] += w * a.pHZ[xl];
            if (!ZDIR) gkL = 0.5 * ctdt * a.inv_r_cell[f - 1] * a.pHr[xl];
        }
        if (hi) {
            long long cu = cidx(f), xu = (long long)k + (long long)a.nnu * cu;
            double w = ctdt * a.inv_dV[cu] * Af;
            gF[0] += w * a.pJ[xu]; gF[1] += w * a.pHr[xu]; gF[2] += w * a.pHZ[xu];
            if (!ZDIR) gkR = 0.5 * ctdt * a.inv_r_cell[f] * a.pHr[xu];
        }
        // stencil cells f-2 .. f+1
        GCell g4[4];
        CellF<double> cs[4], gc[4];
#pragma unroll
        for (int s = 0; s < 4; s++) {
            int p = f - 2 + s;
            g4[s] = ZDIR ? gcell(a, line, p, k) : gcell(a, p, line, k);
            cs[s] = cell_f<double>(g4[s].J, g4[s].Hr, g4[s].HZ, a.jeps);
            gc[s].J = gc[s].fr = gc[s].fZ = 0.0;
        }
        double iv[5];
        const double *ivp = (ZDIR ? a.zint : a.rint) + 5 * f;
#pragma unroll
        for (int t = 0; t < 5; t++) iv[t] = ivp[t];
        const int nl = ZDIR ? nz : nr;
        int pi = f - 1 < 0 ? 0 : (f - 1 >= nl ? nl - 1 : f - 1);
        int pp = f < 0 ? 0 : (f >= nl ? nl - 1 : f);
        double aFi = ZDIR ? alpha_F_at(a, line, pi, k) : alpha_F_at(a, pi, line, k);
        double aFp = ZDIR ? alpha_F_at(a, line, pp, k) : alpha_F_at(a, pp, line, k);
        double uc = (ZDIR ? a.u_Z_star[fi] : a.u_r_star[fi]) * kInvC;
        double gaFi = 0.0, gaFp = 0.0;
        adj_face<ZDIR, FLUX>(cs, iv, aFi, aFp, uc, a.jeps, !ZDIR && f == 0, gF, gkL, gkR, gc, gaFi, gaFp, guc);
#pragma unroll
        for (int s = 0; s < 4; s++) {
            double gJ = 0.0, gHr = 0.0, gHZ = 0.0;
            adj_cell_f(g4[s].J, g4[s].Hr, g4[s].HZ, a.jeps, gc[s], gJ, gHr, gHZ);
            long long xs = (long long)k + (long long)a.nnu * ((long long)g4[s].i + (long long)nr * g4[s].j);
            if (gJ != 0.0) atomicAdd(a.lJ + xs, gJ);
            if (gHr != 0.0 && g4[s].sHr != 0.0) atomicAdd(a.lHr + xs, gHr * g4[s].sHr);
            if (gHZ != 0.0 && g4[s].sHZ != 0.0) atomicAdd(a.lHZ + xs, gHZ * g4[s].sHZ);
        }
        long long xi = ZDIR ? (long long)k + (long long)a.nnu * ((long long)line + (long long)nr * pi)
                            : (long long)k + (long long)a.nnu * ((long long)pi + (long long)nr * line);
        long long xp = ZDIR ? (long long)k + (long long)a.nnu * ((long long)line + (long long)nr * pp)
                            : (long long)k + (long long)a.nnu * ((long long)pp + (long long)nr * line);
        if (gaFi != 0.0) atomicAdd(a.g_aF + xi, gaFi);
        if (gaFp != 0.0) atomicAdd(a.g_aF + xp, gaFp);
    }
    bool head = false;
    guc = seg_sum(guc, fi, lane, head);
    if (act && head && guc != 0.0) atomicAdd((ZDIR ? a.g_uZ : a.g_ur) + fi, guc * kInvC);
}

// ---- seeds and parameter chains --------------------------------------------------------------

// lambda_J += w_k / n_edge on the edge-ring cells (src/SaveHDF5Data_StaticCloudTests.jl:152-199)
__global__ void k_seed_spectrum(double *gJ, const double *w, int nnu, int nr, int nz) {
    const int ne = (nz - 2) + 2 * (nr - 3);
    const double inv = 1.0 / ne;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ne * nnu; q += gridDim.x * blockDim.x) {
        int e = q / nnu, k = q % nnu;
        int i, j;
        if (e < nz - 2) { i = nr - 2; j = 1 + e; }
        else if (e < nz - 2 + nr - 3) { i = 1 + (e - (nz - 2)); j = nz - 2; }
        else { i = 1 + (e - (nz - 2) - (nr - 3)); j = 1; }
        atomicAdd(gJ + (size_t)k + (size_t)nnu * ((size_t)i + (size_t)nr * j), w[k] * inv);
    }
}

// alpha_F = alpha H_voigt (+ alpha_cF): lambda of alpha_F into alpha and H_voigt (warp = cell x 32 bins)
__global__ void k_af_params(const double *g_aF, const double *alpha, const double *Hv, int nnu, long long ncell,
                            double *g_alpha, double *g_Hv) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nkb = (nnu + 31) / 32;
    if (gw >= ncell * nkb) return;
    const long long c = gw / nkb;
    const int k = (int)(gw % nkb) * 32 + lane;
    double s = 0.0;
    if (k < nnu) {
        long long x = (long long)k + (long long)nnu * c;
        double g = g_aF[x];
        s = g * Hv[x];
        g_Hv[x] += g * alpha[c];
    }
    s = wsum_d(s);
    if (lane == 0 && s != 0.0) atomicAdd(g_alpha + c, s);
}

// Update_Hvoigt! (src/ConstantsAndFunctions.jl:319-357) differentiated in T through the
// Doppler width and the Voigt parameter, with the slopes of the linearly interpolated tables
// the forward evaluates (so the derivative is that of the discrete map).
struct LutD {
    const double *y;
    int n;
    double xmax, xmin, inv_dx;
    __device__ __forceinline__ void eval(int table, double x, double &v, double &d) const {
        double xt = (x - xmin) * inv_dx;
        long i = (long)floor(xt);
        if (i + 2 > n) i = n - 2;
        double w = (double)(i + 1) - xt;
        const double *t = y + (size_t)table * n;
        v = w * t[i] + (1.0 - w) * t[i + 1];
        d = (t[i + 1] - t[i]) * inv_dx;
    }
    __device__ __forceinline__ void dawson(double x, double &v, double &d) const {
        if (fabs(x) >= xmax) {
            double ix = 1.0 / x, ix2 = ix * ix;
            v = 0.5 * ix + 0.25 * ix2 * ix;
            d = -0.5 * ix2 - 0.75 * ix2 * ix2;
            return;
        }
        eval(1, x, v, d);
    }
    __device__ __forceinline__ void erf_(double x, double &v, double &d) const {
        if (fabs(x) >= xmax) { v = copysign(1.0, x); d = 0.0; return; }
        eval(0, x, v, d);
    }
    __device__ __forceinline__ void tab(int t, double x, double &v, double &d) const {
        if (fabs(x) >= xmax) { v = 0.0; d = 0.0; return; }
        eval(t, x, v, d);
    }
};

__global__ void k_hvoigt_adj(const double *g_Hv, const double *T, const double *nu, const double *nuC, int nnu,
                             long long ncell, LutD L, double *g_T) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nkb = (nnu + 31) / 32;
    if (gw >= ncell * nkb) return;
    const long long c = gw / nkb;
    const int k = (int)(gw % nkb) * 32 + lane;
    double s = 0.0;
    if (k < nnu) {
        const double sp2 = sqrt(kPi) / 2.0, inv_sp2 = 1.0 / sp2;
        double Tc = T[c];
        double av = compute_a(Tc);
        double inv_dnuD = 1.0 / compute_dnuD(Tc);
        double x = (nuC[k] - kNuLya) * inv_dnuD;
        double xmax = (nu[k + 1] - kNuLya) * inv_dnuD;
        double xmin = (nu[k] - kNuLya) * inv_dnuD;
        double dx = xmax - xmin;
        // every x and a scale as T^(-1/2)
        const double q = -0.5 / Tc;
        double dHdT;
        if (dx > 1e-5) {
            double e1, de1, d1, dd1, g1, dg1, e0, de0, d0, dd0, g0, dg0;
            L.erf_(xmax, e1, de1); L.dawson(xmax, d1, dd1); L.tab(3, xmax, g1, dg1);
            L.erf_(xmin, e0, de0); L.dawson(xmin, d0, dd0); L.tab(3, xmin, g0, dg0);
            double I1 = sp2 * e1 - inv_sp2 * av * d1 + av * av * g1;
            double I0 = sp2 * e0 - inv_sp2 * av * d0 + av * av * g0;
            double Ix1 = sp2 * de1 - inv_sp2 * av * dd1 + av * av * dg1;
            double Ix0 = sp2 * de0 - inv_sp2 * av * dd0 + av * av * dg0;
            double Ia1 = -inv_sp2 * d1 + 2.0 * av * g1;
            double Ia0 = -inv_sp2 * d0 + 2.0 * av * g0;
            double Hvv = (I1 - I0) / dx;
            double dN = (Ix1 * xmax + Ia1 * av) * q - (Ix0 * xmin + Ia0 * av) * q;
            dHdT = dN / dx - Hvv * (dx * q) / dx;
        } else {
            double gv, dg, dv, dd, ov, dov;
            L.tab(2, x, gv, dg); L.dawson(x, dv, dd); L.tab(4, x, ov, dov);
            double Hx = dg + inv_sp2 * av * (2.0 * dv + 2.0 * x * dd) + av * av * dov;
            double Ha = inv_sp2 * (2.0 * x * dv - 1.0) + 2.0 * av * ov;
            dHdT = (Hx * x + Ha * av) * q;
        }
        s = g_Hv[(long long)k + (long long)nnu * c] * dHdT;
    }
    s = wsum_d(s);
    if (lane == 0 && s != 0.0) atomicAdd(g_T + c, s);
}

// ---- launch wrappers ---------------------------------------------------------------------------
template <int M>
static void fa_launch(const FreqAdjArgs &a, int nitems, cudaStream_t st) {
    k_freq_adj<M><<<nitems, ADJ_THREADS, 0, st>>>(a);
}

void launch_freq_adj(const FreqAdjArgs &a, int nitems, cudaStream_t st) {
    if (nitems <= 0) return;
    switch (bins_per_lane(a.nnu)) {
    case 1: fa_launch<1>(a, nitems, st); break;
    case 2: fa_launch<2>(a, nitems, st); break;
    case 4: fa_launch<4>(a, nitems, st); break;
    default: fa_launch<8>(a, nitems, st); break;
    }
}

static int warps_grid(long long nwarps) { return (int)((nwarps * 32 + ADJ_THREADS - 1) / ADJ_THREADS); }

static int threads_grid(long long n) { return (int)((n + ADJ_THREADS - 1) / ADJ_THREADS); }

void launch_adv_adj(const AdjAdvArgs &a, cudaStream_t st) {
    const long long ncell = (long long)a.nr * a.nz;
    k_adv_adj_cell<<<threads_grid(ncell * a.nnu), ADJ_THREADS, 0, st>>>(a);
    const long long nact = a.kmax - a.kmin + 1;
    if (nact <= 0) return;
    const int gr = threads_grid((long long)(a.nr + 1) * a.nz * nact), gz = threads_grid((long long)a.nr * (a.nz + 1) * nact);
    if (a.flux == 0) {
        k_adv_adj_face<false, 0><<<gr, ADJ_THREADS, 0, st>>>(a);
        k_adv_adj_face<true, 0><<<gz, ADJ_THREADS, 0, st>>>(a);
    } else {
        k_adv_adj_face<false, 1><<<gr, ADJ_THREADS, 0, st>>>(a);
        k_adv_adj_face<true, 1><<<gz, ADJ_THREADS, 0, st>>>(a);
    }
}

void launch_seed_spectrum(double *gJ, const double *w, int nnu, int nr, int nz, cudaStream_t st) {
    k_seed_spectrum<<<64, 256, 0, st>>>(gJ, w, nnu, nr, nz);
}

void launch_af_params(const double *g_aF, const double *alpha, const double *Hv, int nnu, long long ncell,
                      double *g_alpha, double *g_Hv, cudaStream_t st) {
    k_af_params<<<warps_grid(ncell * ((nnu + 31) / 32)), ADJ_THREADS, 0, st>>>(g_aF, alpha, Hv, nnu, ncell, g_alpha,
                                                                                g_Hv);
}

void launch_hvoigt_adj(const double *g_Hv, const double *T, const double *nu, const double *nuC, int nnu,
                       long long ncell, const double *lut, int lut_n, double lut_xmax, double *g_T, cudaStream_t st) {
    LutD L;
    L.y = lut; L.n = lut_n; L.xmax = lut_xmax; L.xmin = -lut_xmax;
    L.inv_dx = 1.0 / ((lut_xmax - -lut_xmax) / (lut_n - 1));
    k_hvoigt_adj<<<warps_grid(ncell * ((nnu + 31) / 32)), ADJ_THREADS, 0, st>>>(g_Hv, T, nu, nuC, nnu, ncell, L, g_T);
}

}  // namespace lyd
