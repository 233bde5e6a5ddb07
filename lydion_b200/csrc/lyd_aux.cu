// lyd_aux.cu -- set-up, conversion and diagnostic kernels around the Lyman-alpha step.
#include <cuda_runtime.h>
#include <math.h>

#include "lyd_internal.h"
#include "lyd_physics.cuh"
#include "lyd_species.cuh"

namespace lyd {

// ---- precision conversion of uploaded / downloaded fields ---------------------------------
__global__ void k_to_float(const double *src, float *dst, size_t n, double inv_scale) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        dst[q] = float(src[q] * inv_scale);
}
__global__ void k_from_float(const float *src, double *dst, size_t n, double scale) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        dst[q] = double(src[q]) * scale;
}
__global__ void k_scale(const double *src, double *dst, size_t n, double s) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        dst[q] = src[q] * s;
}

static int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

void launch_convert_in(int prec, const double *src, void *dst, size_t n, double scale, cudaStream_t st) {
    if (prec == 0) {
        if (scale == 1.0) cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        else k_scale<<<grid_for(n), 256, 0, st>>>(src, static_cast<double *>(dst), n, 1.0 / scale);
    } else {
        k_to_float<<<grid_for(n), 256, 0, st>>>(src, static_cast<float *>(dst), n, 1.0 / scale);
    }
}
void launch_convert_out(int prec, const void *src, double *dst, size_t n, double scale, cudaStream_t st) {
    if (prec == 0) {
        if (scale == 1.0) cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        else k_scale<<<grid_for(n), 256, 0, st>>>(static_cast<const double *>(src), dst, n, scale);
    } else {
        k_from_float<<<grid_for(n), 256, 0, st>>>(static_cast<const float *>(src), dst, n, scale);
    }
}

// ---- Voigt look-up tables (src/FastInterpolations.jl:54-112, 178-275) ----------------------
// Dawson's integral F(x) = exp(-x^2) int_0^x exp(t^2) dt, evaluated with its Maclaurin
// series near 0, the asymptotic series far out, and in between with Rybicki's
// sampling-theorem representation (G. B. Rybicki, Computers in Physics 3, 85 (1989)):
//   F(x) = lim_{h->0} pi^(-1/2) sum_{m odd} exp(-(x - m h)^2) / m,
// whose error for a finite step h falls like exp(-(pi / 2h)^2).
static double dawson_host(double x) {
    double ax = fabs(x);
    if (ax < 0.2) {
        double x2 = x * x, term = x, sum = x;
        for (int n = 1; n < 60; n++) {
            term *= -2.0 * x2 / (2.0 * n + 1.0);
            sum += term;
            if (fabs(term) < 1e-19 * fabs(sum)) break;
        }
        return sum;
    }
    if (ax > 50.0) {
        double ix2 = 1.0 / (2.0 * ax * ax), t = 1.0, s = 1.0;
        for (int n = 1; n < 60; n++) {
            t *= (2.0 * n - 1.0) * ix2;
            s += t;
            if (t < 1e-19) break;
        }
        return copysign(s / (2.0 * ax), x);
    }
    const double h = 0.2;
    double n0 = 2.0 * nearbyint(0.5 * ax / h);
    double xp = ax - n0 * h;
    double sum = 0.0;
    for (int n = -45; n <= 45; n += 2) {
        double t = xp - n * h;
        sum += exp(-t * t) / (n0 + n);
    }
    return copysign(sum / sqrt(kPi), x);
}

void build_voigt_lut(double *host, int n, double xmax) {
    double xmin = -xmax;
    double dx = (xmax - xmin) / (n - 1);
    for (int i = 0; i < n; i++) {
        double x = xmin + i * dx;
        double g = exp(-x * x);
        host[0 * (size_t)n + i] = erf(x);
        host[1 * (size_t)n + i] = dawson_host(x);
        host[2 * (size_t)n + i] = g;
        host[3 * (size_t)n + i] = x * exp(-x * x);
        host[4 * (size_t)n + i] = (1.0 - 2.0 * (x * x)) * exp(-x * x);
    }
}

struct Lut {
    const double *y;
    int n;
    double xmax, xmin, inv_dx;
    // EvaluateLUT, src/FastInterpolations.jl:83-112
    __device__ __forceinline__ double eval(int table, double x) const {
        double xt = (x - xmin) * inv_dx;
        long i = (long)floor(xt);
        if (i + 2 > n) i = n - 2;
        double d = (double)(i + 1) - xt;
        const double *t = y + (size_t)table * n;
        return d * t[i] + (1.0 - d) * t[i + 1];
    }
    __device__ __forceinline__ double dawson(double x) const {
        if (fabs(x) >= xmax) { double ix = 1.0 / x; double ix3 = ix * ix * ix; return 0.5 * ix + 0.25 * ix3; }
        return eval(1, x);
    }
    __device__ __forceinline__ double erf_(double x) const { return fabs(x) >= xmax ? copysign(1.0, x) : eval(0, x); }
    __device__ __forceinline__ double gauss(double x) const { return fabs(x) >= xmax ? 0.0 : eval(2, x); }
    __device__ __forceinline__ double xgauss(double x) const { return fabs(x) >= xmax ? 0.0 : eval(3, x); }
    __device__ __forceinline__ double omx2(double x) const { return fabs(x) >= xmax ? 0.0 : eval(4, x); }
};

// H(x,a), int H, Htophat: src/ConstantsAndFunctions.jl:227-279
__device__ __forceinline__ double voigt_H(const Lut &L, double x, double a) {
    const double inv_sp2 = 1.0 / (sqrt(kPi) / 2.0);
    return L.gauss(x) + inv_sp2 * a * (2.0 * x * L.dawson(x) - 1.0) + (a * a) * L.omx2(x);
}
__device__ __forceinline__ double voigt_intH(const Lut &L, double x, double a) {
    const double sp2 = sqrt(kPi) / 2.0;
    const double inv_sp2 = 1.0 / sp2;
    return sp2 * L.erf_(x) - inv_sp2 * a * L.dawson(x) + (a * a) * L.xgauss(x);
}

// Update_Hvoigt!, src/ConstantsAndFunctions.jl:319-357 (one thread per cell and bin)
template <typename S>
__global__ void k_hvoigt(S *Hv, const double *T, const double *nu, const double *nuC, int nnu, size_t ncell, Lut L) {
    size_t n = (size_t)nnu * ncell;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(q % nnu);
        size_t c = q / nnu;
        double Tc = T[c];
        double a = compute_a(Tc);
        double inv_dnuD = 1.0 / compute_dnuD(Tc);
        double x = (nuC[k] - kNuLya) * inv_dnuD;
        double xmax = (nu[k + 1] - kNuLya) * inv_dnuD;
        double xmin = (nu[k] - kNuLya) * inv_dnuD;
        double dx = xmax - xmin;
        double h = (dx > 1e-5) ? (voigt_intH(L, xmax, a) - voigt_intH(L, xmin, a)) / dx : voigt_H(L, x, a);
        Hv[q] = S(h);
    }
}

void launch_hvoigt(int prec, void *Hv, const double *T, const double *nu, const double *nuC, int nnu, size_t ncell,
                   const double *lut, int lut_n, double lut_xmax, cudaStream_t st) {
    Lut L;
    L.y = lut; L.n = lut_n; L.xmax = lut_xmax; L.xmin = -lut_xmax;
    L.inv_dx = 1.0 / ((lut_xmax - -lut_xmax) / (lut_n - 1));
    size_t n = (size_t)nnu * ncell;
    if (prec == 0) k_hvoigt<double><<<grid_for(n), 256, 0, st>>>(static_cast<double *>(Hv), T, nu, nuC, nnu, ncell, L);
    else k_hvoigt<float><<<grid_for(n), 256, 0, st>>>(static_cast<float *>(Hv), T, nu, nuC, nnu, ncell, L);
}

// Update_phi_nu!, src/ConstantsAndFunctions.jl:362-393: per-cell 1 / sum_{kmin..kmax} dnu Hv
template <typename S>
__global__ void k_phi_inv(const S *Hv, const double *dnu, int nnu, size_t ncell, int kmin, int kmax, double *out) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ncell; c += (size_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = kmin; k <= kmax; k++) s += dnu[k] * double(Hv[(size_t)c * nnu + k]);
        out[c] = 1.0 / s;
    }
}
void launch_phi_inv(int prec, const void *Hv, const double *dnu, int nnu, size_t ncell, int kmin, int kmax,
                    double *phi_inv, cudaStream_t st) {
    int g = grid_for(ncell);
    if (prec == 0) k_phi_inv<double><<<g, 256, 0, st>>>(static_cast<const double *>(Hv), dnu, nnu, ncell, kmin, kmax, phi_inv);
    else k_phi_inv<float><<<g, 256, 0, st>>>(static_cast<const float *>(Hv), dnu, nnu, ncell, kmin, kmax, phi_inv);
}

__global__ void k_pd(size_t n, const double *nHII, const double *ne, const double *nHI, const double *nHeI,
                     const double *nH2, const double *T, double z, double *out) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        out[q] = pd_lya_dev(nHII[q], ne[q], nHI[q], nHeI[q], nH2[q], T[q], z);
}
void launch_pd(size_t n, const double *nHII, const double *ne, const double *nHI, const double *nHeI,
               const double *nH2, const double *T, double z, double *out, cudaStream_t st) {
    k_pd<<<grid_for(n), 256, 0, st>>>(n, nHII, ne, nHI, nHeI, nH2, T, z, out);
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Update_f_Lya_MF_L_Lya!, src/ConstantsAndFunctions.jl:606-650: f = dru / dt stored, and the
// per-CTA partial sums of dV|f|, dV f.r_out, dV max(f.r_out,0), 4 pi dV js and, with a gravity
// field (the variant of src/ConstantsAndFunctions.jl:691-804), dV (-f . g_hat) (5 columns).
__global__ void k_mf(const double *dru_r, const double *dru_Z, double *f_r, double *f_Z, const double *js,
                     const double *dV, const double *rCoM, const double *ZCoM, int nr, int nz, double dt,
                     double z_center, const double *g_r, const double *g_Z, double *partials) {
    __shared__ double sh[5][32];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
    const double inv_dt = 1.0 / dt;
    const int ncell = nr * nz;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        int i = c % nr, j = c / nr;
        double fr = dru_r[c] * inv_dt, fz = dru_Z[c] * inv_dt;
        f_r[c] = fr;
        f_Z[c] = fz;
        double v = dV[c];
        a0 += v * sqrt(fr * fr + fz * fz);
        a3 += kFourPi * v * js[c];
        double dr = rCoM[i], dzz = ZCoM[j] - z_center;
        double d = sqrt(dr * dr + dzz * dzz);
        double frad = 0.0;
        if (d > 0.0) {
            double id = 1.0 / d;
            frad = fr * (dr * id) + fz * (dzz * id);
        }
        a1 += v * frad;
        a2 += v * (frad > 0.0 ? frad : 0.0);
        if (g_r) {
            double gr = g_r[c], gz = g_Z[c];
            double gm = sqrt(gr * gr + gz * gz);
            a4 += v * (gm > 0.0 ? -(fr * gr + fz * gz) / gm : 0.0);
        }
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    a0 = wsum(a0); a1 = wsum(a1); a2 = wsum(a2); a3 = wsum(a3); a4 = wsum(a4);
    if (lane == 0) { sh[0][w] = a0; sh[1][w] = a1; sh[2][w] = a2; sh[3][w] = a3; sh[4][w] = a4; }
    __syncthreads();
    if (threadIdx.x < 5) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += sh[threadIdx.x][q];
        partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}
void launch_mf(const double *dru_r, const double *dru_Z, double *f_r, double *f_Z, const double *js,
               const double *dV, const double *rCoM, const double *ZCoM, int nr, int nz, double dt,
               double z_center, const double *g_r, const double *g_Z, double *partials, int nblocks,
               cudaStream_t st) {
    k_mf<<<nblocks, 256, 0, st>>>(dru_r, dru_Z, f_r, f_Z, js, dV, rCoM, ZCoM, nr, nz, dt, z_center, g_r, g_Z,
                                  partials);
}

// Compute_f_esc_Lya_Cylindrical numerator, src/ConstantsAndFunctions.jl:969-993 / 914-961:
// sum over bins and escaping faces of dnu_k A 4 pi max(+-H, 0); single CTA, fixed order.
template <typename S>
__global__ void k_fesc(const S *Hr, const S *HZ, const double *A_r, const double *A_Z, const double *dnu, int nnu,
                       int nr, int nz, int bc_z_bot, double j_scale, double *out) {
    __shared__ double sh[32];
    int nb = nz + nr + (bc_z_bot == 1 ? nr : 0);
    double acc = 0.0;
    for (int q = threadIdx.x; q < nb * nnu; q += blockDim.x) {
        int b = q / nnu, k = q % nnu;
        double v;
        if (b < nz) {
            int j = b;
            double h = double(Hr[(size_t)k + (size_t)nnu * ((size_t)(nr - 1) + (size_t)nr * j)]) * j_scale;
            v = A_r[nr + (size_t)(nr + 1) * j] * kFourPi * (h > 0.0 ? h : 0.0);
        } else if (b < nz + nr) {
            int i = b - nz;
            double h = double(HZ[(size_t)k + (size_t)nnu * ((size_t)i + (size_t)nr * (nz - 1))]) * j_scale;
            v = A_Z[i + (size_t)nr * nz] * kFourPi * (h > 0.0 ? h : 0.0);
        } else {
            int i = b - nz - nr;
            double h = double(HZ[(size_t)k + (size_t)nnu * (size_t)i]) * j_scale;
            v = A_Z[i] * kFourPi * (-h > 0.0 ? -h : 0.0);
        }
        acc += dnu[k] * v;
    }
    acc = wsum(acc);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
        *out = s;
    }
}
void launch_fesc(int prec, const void *Hr, const void *HZ, const double *A_r, const double *A_Z,
                 const double *dnu, int nnu, int nr, int nz, int bc_z_bot, double j_scale,
                 double *out, cudaStream_t st) {
    if (prec == 0)
        k_fesc<double><<<1, 1024, 0, st>>>(static_cast<const double *>(Hr), static_cast<const double *>(HZ), A_r, A_Z,
                                           dnu, nnu, nr, nz, bc_z_bot, j_scale, out);
    else
        k_fesc<float><<<1, 1024, 0, st>>>(static_cast<const float *>(Hr), static_cast<const float *>(HZ), A_r, A_Z,
                                          dnu, nnu, nr, nz, bc_z_bot, j_scale, out);
}

// Column sums of [ncols][nblocks] partials: one warp per column, fixed order.
__global__ void k_colsum(const double *p, int ncols, int nblocks, double *out) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c = w; c < ncols; c += nw) {
        double s = 0.0;
        for (int b = lane; b < nblocks; b += 32) s += p[(size_t)c * nblocks + b];
        s = wsum(s);
        if (lane == 0) out[c] = s;
    }
}
void launch_column_sums(const double *partials, int ncols, int nblocks, double *out, cudaStream_t st) {
    k_colsum<<<1, 1024, 0, st>>>(partials, ncols, nblocks, out);
}

// GetRHDCFLTimeStep, src/AdvectJandH.jl:29-68: min over cells (order-free, so exact).
__global__ void k_cfl(const double *r, const double *Z, const double *u_r, const double *u_Z, int nr, int nz,
                      double c_tilde, double *out) {
    __shared__ double sh[32];
    double m = INFINITY;
    for (int c = threadIdx.x; c < nr * nz; c += blockDim.x) {
        int i = c % nr, j = c / nr;
        double dZ = Z[j + 1] - Z[j], dr = r[i + 1] - r[i];
        double u = hypot(u_r[c], u_Z[c]);
        double dt = 0.5 * fmin(dr, dZ) / (c_tilde + u);
        m = fmin(m, dt);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = INFINITY;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = fmin(s, sh[w]);
        *out = s;
    }
}
void launch_cfl(const double *r, const double *Z, const double *u_r, const double *u_Z, int nr, int nz,
                double c_tilde, double *out, cudaStream_t st) {
    k_cfl<<<1, 1024, 0, st>>>(r, Z, u_r, u_Z, nr, nz, c_tilde, out);
}

// Edge-ring spectra, src/SaveHDF5Data_StaticCloudTests.jl:152-199, 392-420: one warp per
// edge cell; raw J and J / int dnu J.
template <typename S>
__global__ void k_edge(const S *J, const double *dnu, int nnu, int nr, int nz, double j_scale, double *raw,
                       double *norm) {
    int ne = (nz - 2) + 2 * (nr - 3);
    int lane = threadIdx.x & 31;
    for (int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < ne; e += gridDim.x * (blockDim.x >> 5)) {
        int i, j;
        if (e < nz - 2) { i = nr - 2; j = 1 + e; }
        else if (e < (nz - 2) + (nr - 3)) { i = 1 + (e - (nz - 2)); j = nz - 2; }
        else { i = 1 + (e - (nz - 2) - (nr - 3)); j = 1; }
        const S *Jc = J + (size_t)nnu * ((size_t)i + (size_t)nr * j);
        double integ = 0.0;
        for (int k = lane; k < nnu; k += 32) integ += double(Jc[k]) * j_scale * dnu[k];
        integ = wsum(integ);
        for (int k = lane; k < nnu; k += 32) {
            double v = double(Jc[k]) * j_scale;
            raw[(size_t)e * nnu + k] = v;
            norm[(size_t)e * nnu + k] = integ > 0.0 ? v / integ : v;
        }
    }
}
void launch_edge(int prec, const void *J, const double *dnu, int nnu, int nr, int nz, double j_scale,
                 double *raw, double *norm, cudaStream_t st) {
    if (prec == 0) k_edge<double><<<64, 256, 0, st>>>(static_cast<const double *>(J), dnu, nnu, nr, nz, j_scale, raw, norm);
    else k_edge<float><<<64, 256, 0, st>>>(static_cast<const float *>(J), dnu, nnu, nr, nz, j_scale, raw, norm);
}

// ---- the FP64 arithmetic helpers on host-given arguments, for their accuracy checks ---------
__global__ void k_math(int fn, const double *x, double *y, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const double v = x[q];
        double r;
        switch (fn) {
            case 0: r = rsqrt_nr(v); break;
            case 1: r = rcp<double>(v); break;
            case 2: r = v * rsqrt_nr(v); break;
            case 3: r = chi_L84<double>(v); break;
            default: r = exp_tab(v, kExp2Tab); break;
        }
        y[q] = r;
    }
}
void launch_math(int fn, const double *x, double *y, size_t n, cudaStream_t st) {
    k_math<<<grid_for(n), 256, 0, st>>>(fn, x, y, n);
}

}  // namespace lyd
