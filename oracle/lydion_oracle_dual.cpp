// lydion_oracle_dual.cpp -- forward-mode derivatives of the CPU oracle, by dual numbers.
//
// TEST INFRASTRUCTURE ONLY: the independent derivative check of the library's hand-written
// adjoint (lyd_adjoint_run). Nothing in the product library links or calls this code.
//
// The FP64 restatement in lydion_oracle.c is compiled a second time with every `double`
// replaced by Dual, a number carrying a value and one directional derivative (forward-mode
// automatic differentiation: each arithmetic operation and elementary function propagates the
// derivative by the chain rule; comparisons, clamps, floors, min/max and pivot choices act on
// the value, so the derivative is that of the branch the value takes). This stands in for
// running ForwardDiff.jl through the Julia reference, which needs Julia: the restatement
// follows the reference operation by operation, and its dual build differentiates it without
// any hand-written derivative. No code of the oracle is duplicated here.
//
// orcd_objective_tangent: for a static cloud given as the oracle's plain structs, and seed
// directions for alpha, alpha_c, T (directly and through H_voigt(T), phi_nu and alpha_F),
// u*_r, u*_Z and the initial J, it runs n static-driver steps (src/StaticCloudTest.jl:357-392)
// and returns the objective w_MF * M_F(last step) + sum_k w_k S_k(final J), S the edge-ring
// mean spectrum, and its directional derivative along the seeds.
#include <math.h>
#include <omp.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <vector>

struct Dual {
    double v, d;
    Dual() : v(0.0), d(0.0) {}
    Dual(double x) : v(x), d(0.0) {}   // constants carry no derivative
    Dual(double x, double dx) : v(x), d(dx) {}
    explicit operator int() const { return (int)v; }
    explicit operator long() const { return (long)v; }
    Dual &operator+=(const Dual &b) { v += b.v; d += b.d; return *this; }
    Dual &operator-=(const Dual &b) { v -= b.v; d -= b.d; return *this; }
    // a derivative term whose factor is exactly zero contributes nothing, even where the
    // value it multiplies is not finite (a value that reaches no result)
    Dual &operator*=(const Dual &b) {
        d = (d != 0.0 ? d * b.v : 0.0) + (b.d != 0.0 ? v * b.d : 0.0);
        v *= b.v;
        return *this;
    }
    Dual &operator/=(const Dual &b) {
        const double q = v / b.v;
        d = (d != 0.0 ? d / b.v : 0.0) - (b.d != 0.0 ? q * b.d / b.v : 0.0);
        v = q;
        return *this;
    }
};
static inline Dual operator+(Dual a, const Dual &b) { return a += b; }
static inline Dual operator-(Dual a, const Dual &b) { return a -= b; }
static inline Dual operator*(Dual a, const Dual &b) { return a *= b; }
static inline Dual operator/(Dual a, const Dual &b) { return a /= b; }
static inline Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
static inline Dual operator+(const Dual &a) { return a; }
static inline bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
static inline bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
static inline bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
static inline bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
static inline bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
static inline bool operator!=(const Dual &a, const Dual &b) { return a.v != b.v; }
static inline bool operator!(const Dual &a) { return !a.v; }

static inline Dual exp(const Dual &a) { const double e = std::exp(a.v); return Dual(e, a.d != 0.0 ? e * a.d : 0.0); }
static inline Dual log(const Dual &a) { return Dual(std::log(a.v), a.d != 0.0 ? a.d / a.v : 0.0); }
static inline Dual log10(const Dual &a) {
    return Dual(std::log10(a.v), a.d != 0.0 ? a.d / (a.v * std::log(10.0)) : 0.0);
}
static inline Dual sqrt(const Dual &a) {
    const double s = std::sqrt(a.v);
    return Dual(s, (s > 0.0 && a.d != 0.0) ? a.d / (2.0 * s) : 0.0);
}
static inline Dual fabs(const Dual &a) { return a.v < 0.0 ? -a : a; }
static inline Dual fmin(const Dual &a, const Dual &b) { return b.v < a.v ? b : a; }
static inline Dual fmax(const Dual &a, const Dual &b) { return b.v > a.v ? b : a; }
static inline Dual floor(const Dual &a) { return Dual(std::floor(a.v), 0.0); }
static inline Dual pow(const Dual &a, const Dual &b) {
    const double p = std::pow(a.v, b.v);
    double dp = a.d != 0.0 ? b.v * std::pow(a.v, b.v - 1.0) * a.d : 0.0;
    if (b.d != 0.0 && a.v > 0.0) dp += p * std::log(a.v) * b.d;
    return Dual(p, dp);
}
static inline Dual hypot(const Dual &a, const Dual &b) { return sqrt(a * a + b * b); }
static inline bool isfinite(const Dual &a) { return std::isfinite(a.v) && std::isfinite(a.d); }
static inline Dual copysign(double a, const Dual &b) { return Dual(std::copysign(a, b.v), 0.0); }

// The oracle, with Dual for double, in a namespace of its own. Its system headers are already
// included above, so their include guards keep them out of the namespace.
namespace dual {
#define double Dual
#include "lydion_oracle.c"
#undef double
}  // namespace dual

// ---- the plain (double) layouts of the oracle's structs, as the Python front end fills them ----
struct PGeom {
    int nr, nz;
    const double *r, *Z, *rCoM, *ZCoM, *dV, *inv_dV, *A_r, *A_Z, *inv_r_cell;
    const double *dr_L, *dr_R, *inv_dr_i_im1, *inv_dr_ip1_i, *inv_dr_ip2_ip1;
    double dr_b[10];
    const double *dZ_L, *dZ_R, *inv_dZ_j_jm1, *inv_dZ_jp1_j, *inv_dZ_jp2_jp1;
    double dZ_b[10];
    int bc_r_left;
};
struct PLya {
    int nnu, nr, nz;
    double *J, *J_old, *H_r, *H_Z, *H_r_old, *H_Z_old;
    double *alpha_F, *Hvoigt, *phi_nu;
    double *alpha, *alpha_c, *pd, *js;
    double *T;
    double *dru_r, *dru_Z, *f_r, *f_Z;
    const double *nu;
    const double *nuC, *dnu, *inv_dnu, *inv_nuC;
    int kcore_min, kcore_max;
    int recoil;
    int flux_method;
    double alpha_floor;
    double *F_r, *F_Z, *F_r_Hr, *F_Z_Hr, *F_r_HZ, *F_Z_HZ;
    double *K_iph, *K_imh;
    double *Fkp, *Fk, *Fkm;
};
struct PVel {
    const double *u_r_star, *u_Z_star, *dur_dr, *dur_dZ, *duZ_dr, *duZ_dZ, *ur_over_r;
};
struct PLut {
    double xmax, xmin, inv_dx;
    int nx;
    const double *erf_y, *dawson_y, *gauss_y, *xgauss_y, *omx2gauss_y;
};

namespace {
// a Dual copy of n plain values, with the seed (or zero) as derivative
struct Buf {
    std::vector<Dual> a;
    Buf() {}
    Buf(const double *x, size_t n, const double *seed = nullptr) : a(n) {
        for (size_t q = 0; q < n; q++) a[q] = Dual(x ? x[q] : 0.0, seed ? seed[q] : 0.0);
    }
    explicit Buf(size_t n) : a(n) {}
    Dual *p() { return a.data(); }
};
}  // namespace

extern "C" {

// Seeds (each may be NULL): d_alpha, d_alpha_c, d_T (n_r n_z), d_u_r_star ((n_r+1) n_z),
// d_u_Z_star (n_r (n_z+1)), d_J0 (n_nu n_r n_z). The initial state is the plain struct's J,
// H_r, H_Z (their old arrays equal to them). H_voigt follows T through the look-up tables,
// phi_nu follows H_voigt over the core bins, alpha_F = alpha * H_voigt (the static driver's,
// src/StaticCloudTest.jl:283-285). out[0] = objective, out[1] = its directional derivative,
// out[2] = M_F, out[3] = d M_F. Returns 0.
int orcd_objective_tangent(const PLya *ps, const PGeom *pg, const PVel *pv, const PLut *pl, double c_tilde,
                           double dt, double z_center, int bc_r_right, int bc_z_bot, int bc_z_top, int n_steps,
                           double w_MF, const double *w_spec, const double *d_alpha, const double *d_alpha_c,
                           const double *d_T, const double *d_u_r_star, const double *d_u_Z_star, const double *d_J0,
                           double *out) {
    const int nnu = ps->nnu, nr = ps->nr, nz = ps->nz;
    const size_t n3 = (size_t)nnu * nr * nz, nc = (size_t)nr * nz;
    const size_t nrf = (size_t)(nr + 1) * nz, nzf = (size_t)nr * (nz + 1);
    // geometry and frequency grid: constants
    Buf g_r(pg->r, nr + 1), g_Z(pg->Z, nz + 1), g_rC(pg->rCoM, nr), g_ZC(pg->ZCoM, nz), g_dV(pg->dV, nc),
        g_idV(pg->inv_dV, nc), g_Ar(pg->A_r, nrf), g_AZ(pg->A_Z, nzf), g_irc(pg->inv_r_cell, nr),
        g_drL(pg->dr_L, nr), g_drR(pg->dr_R, nr), g_ra(pg->inv_dr_i_im1, nr), g_rb(pg->inv_dr_ip1_i, nr),
        g_rc(pg->inv_dr_ip2_ip1, nr), g_dZL(pg->dZ_L, nz), g_dZR(pg->dZ_R, nz), g_za(pg->inv_dZ_j_jm1, nz),
        g_zb(pg->inv_dZ_jp1_j, nz), g_zc(pg->inv_dZ_jp2_jp1, nz);
    dual::orc_geom g;
    g.nr = nr; g.nz = nz;
    g.r = g_r.p(); g.Z = g_Z.p(); g.rCoM = g_rC.p(); g.ZCoM = g_ZC.p(); g.dV = g_dV.p(); g.inv_dV = g_idV.p();
    g.A_r = g_Ar.p(); g.A_Z = g_AZ.p(); g.inv_r_cell = g_irc.p();
    g.dr_L = g_drL.p(); g.dr_R = g_drR.p(); g.inv_dr_i_im1 = g_ra.p(); g.inv_dr_ip1_i = g_rb.p();
    g.inv_dr_ip2_ip1 = g_rc.p();
    g.dZ_L = g_dZL.p(); g.dZ_R = g_dZR.p(); g.inv_dZ_j_jm1 = g_za.p(); g.inv_dZ_jp1_j = g_zb.p();
    g.inv_dZ_jp2_jp1 = g_zc.p();
    for (int q = 0; q < 10; q++) { g.dr_b[q] = pg->dr_b[q]; g.dZ_b[q] = pg->dZ_b[q]; }
    g.bc_r_left = pg->bc_r_left;
    Buf f_nu(ps->nu, nnu + 1), f_nuC(ps->nuC, nnu), f_dnu(ps->dnu, nnu), f_idnu(ps->inv_dnu, nnu),
        f_inuC(ps->inv_nuC, nnu);
    // state and inputs, seeded
    Buf J(ps->J, n3, d_J0), Jo(ps->J, n3, d_J0), Hr(ps->H_r, n3), HZ(ps->H_Z, n3), Hro(ps->H_r, n3),
        HZo(ps->H_Z, n3), aF(n3), Hv(n3), phi(n3);
    Buf al(ps->alpha, nc, d_alpha), ac(ps->alpha_c, nc, d_alpha_c), pd(ps->pd, nc), js(ps->js, nc), T(ps->T, nc, d_T);
    Buf dr(nc), dz(nc), fr(nc), fz(nc);
    Buf Fr((size_t)nnu * nrf), FZ((size_t)nnu * nzf), FrH((size_t)nnu * nrf), FZH((size_t)nnu * nzf),
        FrZ((size_t)nnu * nrf), FZZ((size_t)nnu * nzf), Kp(n3), Km(n3), Fkp(n3), Fk(n3), Fkm(n3);
    dual::orc_lya s;
    s.nnu = nnu; s.nr = nr; s.nz = nz;
    s.J = J.p(); s.J_old = Jo.p(); s.H_r = Hr.p(); s.H_Z = HZ.p(); s.H_r_old = Hro.p(); s.H_Z_old = HZo.p();
    s.alpha_F = aF.p(); s.Hvoigt = Hv.p(); s.phi_nu = phi.p();
    s.alpha = al.p(); s.alpha_c = ac.p(); s.pd = pd.p(); s.js = js.p(); s.T = T.p();
    s.dru_r = dr.p(); s.dru_Z = dz.p(); s.f_r = fr.p(); s.f_Z = fz.p();
    s.nu = f_nu.p(); s.nuC = f_nuC.p(); s.dnu = f_dnu.p(); s.inv_dnu = f_idnu.p(); s.inv_nuC = f_inuC.p();
    s.kcore_min = ps->kcore_min; s.kcore_max = ps->kcore_max; s.recoil = ps->recoil; s.flux_method = ps->flux_method;
    s.alpha_floor = ps->alpha_floor;
    s.F_r = Fr.p(); s.F_Z = FZ.p(); s.F_r_Hr = FrH.p(); s.F_Z_Hr = FZH.p(); s.F_r_HZ = FrZ.p(); s.F_Z_HZ = FZZ.p();
    s.K_iph = Kp.p(); s.K_imh = Km.p(); s.Fkp = Fkp.p(); s.Fk = Fk.p(); s.Fkm = Fkm.p();
    Buf ur(pv->u_r_star, nrf, d_u_r_star), uz(pv->u_Z_star, nzf, d_u_Z_star), ga(pv->dur_dr, nc), gb(pv->dur_dZ, nc),
        gc(pv->duZ_dr, nc), gd(pv->duZ_dZ, nc), ge(pv->ur_over_r, nc);
    dual::orc_vel v;
    v.u_r_star = ur.p(); v.u_Z_star = uz.p(); v.dur_dr = ga.p(); v.dur_dZ = gb.p(); v.duZ_dr = gc.p();
    v.duZ_dZ = gd.p(); v.ur_over_r = ge.p();
    // the Voigt tables (constants) and the profiles of T
    const size_t nx = (size_t)pl->nx;
    Buf t0(pl->erf_y, nx), t1(pl->dawson_y, nx), t2(pl->gauss_y, nx), t3(pl->xgauss_y, nx), t4(pl->omx2gauss_y, nx);
    dual::orc_voigt_lut L;
    L.xmax = pl->xmax; L.xmin = pl->xmin; L.inv_dx = pl->inv_dx; L.nx = pl->nx;
    L.erf_y = t0.p(); L.dawson_y = t1.p(); L.gauss_y = t2.p(); L.xgauss_y = t3.p(); L.omx2gauss_y = t4.p();
    dual::orc_update_hvoigt(&L, &s);
    dual::orc_update_phi_nu(&s, s.kcore_min, s.kcore_max);
    for (size_t c = 0; c < nc; c++)
        for (int k = 0; k < nnu; k++) s.alpha_F[c * nnu + k] = s.alpha[c] * s.Hvoigt[c * nnu + k];
    dual::orc_update_freq_factors(&s, &v);      // once at set-up, as the static driver does
    // the steps
    Buf hist((size_t)n_steps * 7);
    dual::orc_static_run(&s, &g, &v, Dual(c_tilde), Dual(dt), Dual(z_center), bc_r_right, bc_z_bot, bc_z_top,
                         n_steps, hist.p());
    const Dual MF = hist.a[(size_t)(n_steps - 1) * 7];
    Dual obj = Dual(w_MF) * MF;
    const int ne = dual::orc_edge_count(nr, nz);
    if (w_spec && ne > 0) {
        Buf raw((size_t)ne * nnu), norm((size_t)ne * nnu);
        std::vector<int> ri(ne), zi(ne);
        dual::orc_edge_spectra(&s, raw.p(), norm.p(), ri.data(), zi.data());
        for (int k = 0; k < nnu; k++) {
            Dual sk(0.0);
            for (int e = 0; e < ne; e++) sk += raw.a[(size_t)e * nnu + k];
            obj += Dual(w_spec[k]) * (sk / Dual((double)ne));
        }
    }
    out[0] = obj.v; out[1] = obj.d; out[2] = MF.v; out[3] = MF.d;
    return 0;
}

}  // extern "C"
