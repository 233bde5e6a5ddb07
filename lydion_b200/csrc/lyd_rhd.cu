// lyd_rhd.cu -- the Lyman-alpha block of the radiation-hydrodynamics photo-thermochemistry
// sub-cycle, on the device, for every cell at once:
//   k_rhd_prep    PrepareLyaSubCycling! (src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:
//                 2087-2155) without the profile part: line and continuum opacities, the flux
//                 opacity of the continuum, the destruction probability and the emissivity from
//                 the cell's gas and dust state (one thread per cell). H_voigt and phi_nu over all
//                 bins come from the set-up kernels (Update_Hvoigt_And_phinu_cell!, :2039-2080).
//   k_rhd_absorb  the Lyman-alpha block of AbsorptionStep (:1580-1680) over each cell's own
//                 sub-step: backward-Euler emission/absorption of J and absorption of H from the
//                 sub-cycle's old state, the radiation momentum and its gas/dust split
//                 (SplitRadPressure, :1017-1046), the new energy density and the rejection test
//                 (one warp per cell, bins across the lanes); optionally the commit of accepted
//                 cells (:3197-3206) and the restore of rejected ones (RestoreLyaRejection,
//                 :980-991).
#include <cuda_runtime.h>

#include "lyd_internal.h"
#include "lyd_physics.cuh"
#include "lyd_species.cuh"

namespace lyd {

constexpr double kSigT = 6.6524587321e-25, kSigOHLya = 4.07e-18, kSigCHLya = 0.05e-18, kSigRaman = 2.1e-25;
constexpr double kTolAbs = 0.1;
constexpr double kELyaFloor = kFourPiOverC * 1e-15;   // e_Lya_floor = 4 pi / c J_floor

__global__ void k_rhd_prep(RhdPrepArgs a) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < a.ncell; c += (size_t)gridDim.x * blockDim.x) {
        const double T = a.T[c], nHI = a.nHI[c], nH2 = a.nH2[c], nHII = a.nHII[c], nHeI = a.nHeI[c];
        const double ne = a.ne[c], nOHx = a.nOHx[c], nCHx = a.nCHx[c];
        double rho[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const double r = a.rho_d[q * a.ncell + c];
            rho[q] = r > a.rho_ignore ? r : 0.0;           // dust near the floor is ignored
        }
        const double abs_gas = nH2 * kSigRaman + nOHx * kSigOHLya + nCHx * kSigCHLya;
        const double F_gas = abs_gas + ne * kSigT;
        a.alpha[c] = nHI * compute_sigma0(T);
        a.alpha_c[c] = a.kabs[0] * rho[0] + a.kabs[1] * rho[1] + a.kabs[2] * rho[2] + abs_gas;
        a.alpha_cF[c] = a.kF[0] * rho[0] + a.kF[1] * rho[1] + a.kF[2] * rho[2] + F_gas;
        a.pd[c] = a.destruction ? pd_lya_dev(nHII, ne, nHI, nHeI, nH2, T, a.z) : 0.0;
        a.js[c] = js_rec_lya(T, nHII, ne, a.ots != 0) + js_coll_lya(T, nHI, ne);
        a.T_out[c] = T;
#pragma unroll
        for (int q = 0; q < 3; q++) a.dust_F[q * a.ncell + c] = a.kF[q] * rho[q];
    }
}

void launch_rhd_prep(const RhdPrepArgs &a, cudaStream_t st) {
    const size_t g = (a.ncell + 255) / 256;
    k_rhd_prep<<<(int)(g < 65535 ? g : 65535), 256, 0, st>>>(a);
}

__device__ __forceinline__ double wsum_rhd(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename S>
__global__ void __launch_bounds__(256, 3) k_rhd_absorb(RhdAbsorbArgs<S> a) {
    const int lane = threadIdx.x & 31;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    const double ct = a.c_tilde, ic = 1.0 / ct;
    for (size_t c = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < a.ncell; c += nw) {
        const double dt = a.dt[c];
        const double alpha = a.alpha[c], ac = a.alpha_c[c], acF = a.alpha_cF[c], pd = a.pd[c];
        const double pinv = a.phi_inv[c];
        const double dS = a.dust_F[c], dC = a.dust_F[a.ncell + c], dP = a.dust_F[2 * a.ncell + c];
        const double ct_js = ct * a.js[c] / a.j_scale;                   // in storage units of J
        const double pd_a = pd * alpha;
        const size_t base = c * (size_t)a.nnu;
        double intJ = 0.0, dr = 0.0, dz = 0.0, sp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        auto body = [&](int k, double Hv, double Jo, double Hro, double HZo) {
            const size_t x = base + k;
            const double dJdt = ct_js * (Hv * pinv);
            const double a_abs = ac + pd_a * Hv;
            double Jn = (Jo + dJdt * dt) / (1.0 + a_abs * ct * dt);
            Jn = Jn > a.jeps ? Jn : a.jeps;
            const double aF = alpha * Hv + acF;
            const double hr = Hro / (1.0 + aF * ct * dt), hz = HZo / (1.0 + aF * ct * dt);
            a.J[x] = S(Jn);
            a.Hr[x] = S(hr);
            a.HZ[x] = S(hz);
            const double w = a.dnu[k] * kFourPiOverC * a.j_scale;
            const double mr = w * (ic * (Hro - hr)), mz = w * (ic * (HZo - hz));
            dr += mr;
            dz += mz;
            double ag = aF - dS - dC - dP;
            ag = ag > 0.0 ? ag : 0.0;
            const double tot = ag + dS + dC + dP;
            double f0 = 1.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
            if (tot > 0.0) {
                const double it = 1.0 / tot;
                f0 = ag * it; f1 = dS * it; f2 = dC * it; f3 = dP * it;
            }
            sp[0] += f0 * mr; sp[1] += f0 * mz; sp[2] += f1 * mr; sp[3] += f1 * mz;
            sp[4] += f2 * mr; sp[5] += f2 * mz; sp[6] += f3 * mr; sp[7] += f3 * mz;
            intJ += a.dnu[k] * double(S(Jn));
        };
        // two bins per lane per pass, their loads issued together
        for (int kb = 0; kb < a.nnu; kb += 64) {
            const int k0 = kb + lane, k1 = kb + 32 + lane;
            const bool v0 = k0 < a.nnu, v1 = k1 < a.nnu;
            const size_t x0 = base + k0, x1 = base + k1;
            const double Hv0 = v0 ? double(a.Hv[x0]) : 0.0, Hv1 = v1 ? double(a.Hv[x1]) : 0.0;
            const double Jo0 = v0 ? double(a.Jold[x0]) : 0.0, Jo1 = v1 ? double(a.Jold[x1]) : 0.0;
            const double Hr0 = v0 ? double(a.Hrold[x0]) : 0.0, Hr1 = v1 ? double(a.Hrold[x1]) : 0.0;
            const double HZ0 = v0 ? double(a.HZold[x0]) : 0.0, HZ1 = v1 ? double(a.HZold[x1]) : 0.0;
            if (v0) body(k0, Hv0, Jo0, Hr0, HZ0);
            if (v1) body(k1, Hv1, Jo1, Hr1, HZ1);
        }
        intJ = wsum_rhd(intJ);
        dr = wsum_rhd(dr);
        dz = wsum_rhd(dz);
#pragma unroll
        for (int q = 0; q < 8; q++) sp[q] = wsum_rhd(sp[q]);
        const double e_new = kFourPiOverC * intJ * a.j_scale;
        const double e_old = a.e_lya[c];
        const double de = fabs(e_new - e_old) / (e_old + kELyaFloor);
        const double dt_lya = ic / (ac + pd_a);
        const bool reject = (de > kTolAbs && dt > kTolAbs * dt_lya) || !isfinite(de);
        if (lane == 0) {
            double *o = a.out;
            const size_t n = a.ncell;
            o[c] = reject ? 1.0 : 0.0;
            o[n + c] = de;
            o[2 * n + c] = e_new;
            o[3 * n + c] = dr;
            o[4 * n + c] = dz;
#pragma unroll
            for (int q = 0; q < 8; q++) o[(5 + q) * n + c] = sp[q];
            o[13 * n + c] = dt_lya;
            if (a.commit && !reject) a.e_lya[c] = e_new;
        }
        if (a.commit) {
            // each lane revisits the bins it wrote
            for (int k = lane; k < a.nnu; k += 32) {
                const size_t x = base + k;
                if (reject) {
                    a.J[x] = a.Jold[x]; a.Hr[x] = a.Hrold[x]; a.HZ[x] = a.HZold[x];
                } else {
                    a.Jold[x] = a.J[x]; a.Hrold[x] = a.Hr[x]; a.HZold[x] = a.HZ[x];
                }
            }
        }
    }
}

// FindRSL_LyaRT, src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:614-711: per cell the
// speed eps_RSL max(1, (a tau)^(1/3) f_abs) max(|u|, c_s) that keeps the Lya transport accurate,
// with tau = alpha max(dr, dZ) and f_abs = 1 / (1 + (a tau)^(1/3) tau_c + 0.6 pd tau); the
// maximum over the cells goes to *out (non-negative doubles order like their bit patterns).
__global__ void k_rsl(RslArgs a) {
    double m = 0.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < a.ncell; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % a.nr), j = (int)(c / a.nr);
        const double dr = a.r_if[i + 1] - a.r_if[i], dz = a.Z_if[j + 1] - a.Z_if[j];
        const double rho = a.rho[c], T = a.T[c];
        const double cs = sqrt(a.gamma[c] * a.P[c] / rho);
        double xHI = 1.0 - a.xHII[c] - 2.0 * a.xH2[c];
        xHI = xHI > 0.0 ? xHI : 0.0;
        const double nHI = xHI * a.X_over_mH * rho;
        const double alpha = nHI * compute_sigma0(T);
        const double dX = dr > dz ? dr : dz;
        const double tau = alpha * dX;
        const double tauc = (a.kabs[0] * a.rho_d[c] + a.kabs[1] * a.rho_d[a.ncell + c] +
                             a.kabs[2] * a.rho_d[2 * a.ncell + c]) * dX;
        const double at = compute_a(T) * tau;
        const double at13 = pow(at, 1.0 / 3.0);
        const double fabs_ = 1.0 / (1.0 + at13 * tauc + 0.6 * a.pd[c] * tau);
        const double u = hypot(a.u_r[c], a.u_Z[c]);
        const double f = at13 * fabs_;
        const double v = a.eps_rsl * (f > 1.0 ? f : 1.0) * (u > cs ? u : cs);
        m = v > m ? v : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, m, o);
        m = w > m ? w : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(a.out, (unsigned long long)__double_as_longlong(m));
}

void launch_rsl(const RslArgs &a, cudaStream_t st) {
    cudaMemsetAsync(a.out, 0, 8, st);
    const size_t g = (a.ncell + 255) / 256;
    k_rsl<<<(int)(g < 1184 ? (g > 0 ? g : 1) : 1184), 256, 0, st>>>(a);
}

void launch_rhd_absorb(int sprec, const void *args, cudaStream_t st) {
    const int blocks = 148 * 8;
    if (sprec == 0) k_rhd_absorb<double><<<blocks, 256, 0, st>>>(*static_cast<const RhdAbsorbArgs<double> *>(args));
    else k_rhd_absorb<float><<<blocks, 256, 0, st>>>(*static_cast<const RhdAbsorbArgs<float> *>(args));
}

}  // namespace lyd
