// lyd_adjoint.cuh -- reverse-mode (adjoint) counterparts of the step's device functions, FP64.
//
// Each adj_* function takes the forward inputs (it recomputes what it needs) and the adjoints
// of the forward outputs, and ACCUMULATES the adjoints of the inputs (+=). Non-smooth points
// take the derivative of the branch the forward took (MinMod picks the selected slope, clamps
// and floors pass zero when active, |x| takes sign(x)), so the adjoint is the exact derivative
// of the discrete step wherever that is differentiable.
#pragma once
#include "lyd_physics.cuh"

namespace lyd {

// chi_L84(f) and its derivative together, src/M1Closure.jl:28-33: chi = (3 + 4f^2) / (5 + 2s)
// = (5 - 2s) / 3 with s = sqrt(4 - 3f^2), formed as chi_L84 forms it; chi' = -(2/3) s' = 2f / s.
__device__ __forceinline__ void chi_dchi_L84(double f, double &chi, double &dchi) {
    const double f2 = f * f;
    const double t = 4.0 - 3.0 * f2;
    const double is = rsqrt_nr(t);
    chi = fma(-2.0 * t, is, 5.0) * (1.0 / 3.0);
    dchi = 2.0 * f * is;
}

__device__ __forceinline__ void adj_minmod(double a, double b, double g, double &ga, double &gb) {
    if (a * b <= 0.0) return;
    if (fabs(a) < fabs(b)) ga += g;
    else gb += g;
}

// Compute_D_Edd_from_f_n (src/M1Closure.jl:91-119): (f, nr, nZ) -> (Drr, DZZ, DrZ)
__device__ __forceinline__ void adj_D_from_f_n(double f, double nr, double nZ, double gDrr, double gDZZ,
                                               double gDrZ, double &gf, double &gnr, double &gnZ) {
    if (!(f > kFmin)) return;
    const bool clamped = !(f < kFmax);
    double fc = clamped ? kFmax : f;
    double chi, dchi;
    chi_dchi_L84(fc, chi, dchi);
    double b = (3.0 * chi - 1.0) * 0.5;
    double ga = gDrr + gDZZ;
    double gb = gDrr * nr * nr + gDZZ * nZ * nZ + gDrZ * nr * nZ;
    gnr += 2.0 * b * nr * gDrr + b * nZ * gDrZ;
    gnZ += 2.0 * b * nZ * gDZZ + b * nr * gDrZ;
    double gchi = -0.5 * ga + 1.5 * gb;
    if (!clamped) gf += gchi * dchi;
}

// Compute_D_Edd (src/M1Closure.jl:46-83): (Hr, HZ, J) -> (Drr, DZZ, DrZ)
__device__ __forceinline__ void adj_D_edd(double Hr, double HZ, double J, double jeps, double heps2, double gDrr,
                                          double gDZZ, double gDrZ, double &gHr, double &gHZ, double &gJ) {
    double H2 = Hr * Hr + HZ * HZ;
    const double fmin2 = kFmin * kFmin;
    if (J <= jeps || H2 <= heps2 || H2 <= fmin2 * J * J || !(H2 >= kDblMinNormal)) return;
    const double iH = rsqrt_nr(H2);   // |H| and 1/|H| as D_edd forms them
    const double Hm = H2 * iH;
    const double iJ = rcp<double>(J);
    double fr = Hm * iJ;
    const bool inside = fr > kFmin && fr < kFmax;
    double f = fr < kFmin ? kFmin : (fr > kFmax ? kFmax : fr);
    double chi, dchi;
    chi_dchi_L84(f, chi, dchi);
    double b = (3.0 * chi - 1.0) * 0.5;
    double nr = Hr * iH, nZ = HZ * iH;
    double ga = gDrr + gDZZ;
    double gb = gDrr * nr * nr + gDZZ * nZ * nZ + gDrZ * nr * nZ;
    double gnr = 2.0 * b * nr * gDrr + b * nZ * gDrZ;
    double gnZ = 2.0 * b * nZ * gDZZ + b * nr * gDrZ;
    double gchi = -0.5 * ga + 1.5 * gb;
    double gf = inside ? gchi * dchi : 0.0;
    // f = Hm / J ; n = H / Hm
    double gHm = gf * iJ - (gnr * nr + gnZ * nZ) * iH;
    gJ += -gf * fr * iJ;
    gHr += gnr * iH + gHm * nr;
    gHZ += gnZ * iH + gHm * nZ;
}

// D_colon_grad_u_Cylindrical (src/ConstantsAndFunctions.jl:883-895)
__device__ __forceinline__ void adj_d_colon_grad_u(double Drr, double DrZ, double DZZ, double a, double b, double c,
                                                   double d, double e, double g, double &gDrr, double &gDrZ,
                                                   double &gDZZ, double gu[5]) {
    double Dpp = 1.0 - Drr - DZZ;
    const bool pos = Dpp > 0.0;
    Dpp = pos ? Dpp : 0.0;
    gDrr += g * (a - (pos ? e : 0.0));
    gDZZ += g * (d - (pos ? e : 0.0));
    gDrZ += g * (b + c);
    gu[0] += g * Drr;
    gu[1] += g * DrZ;
    gu[2] += g * DrZ;
    gu[3] += g * DZZ;
    gu[4] += g * Dpp;
}

// Forward intermediates of ReconstructInterface kept for its adjoint.
struct ReconT {
    double dJc, aJL, aJR, dfrc, afrL, afrR, dfZc, afZL, afZR;   // minmod arguments
    double JL, JR;                                               // before the floors
    double frL0, fZL0, frR0, fZR0;                               // before the renormalisation
    double fL0, fR0;                                             // |f| before the renormalisation
    Recon<double> o;
};

__device__ __forceinline__ void recon_fwd(const CellF<double> &cm1, const CellF<double> &ci,
                                          const CellF<double> &cp1, const CellF<double> &cp2, const double iv[5],
                                          double aFi, double aFp, double jeps, ReconT &t) {
    const double dL = iv[0], dR = iv[1];
    Recon<double> &o = t.o;
    o.tau_L = aFi * dL;
    o.tau_R = aFp * dR;
    t.dJc = (cp1.J - ci.J) * iv[3];
    t.aJL = (ci.J - cm1.J) * iv[2];
    t.aJR = (cp2.J - cp1.J) * iv[4];
    t.dfrc = (cp1.fr - ci.fr) * iv[3];
    t.afrL = (ci.fr - cm1.fr) * iv[2];
    t.afrR = (cp2.fr - cp1.fr) * iv[4];
    t.dfZc = (cp1.fZ - ci.fZ) * iv[3];
    t.afZL = (ci.fZ - cm1.fZ) * iv[2];
    t.afZR = (cp2.fZ - cp1.fZ) * iv[4];
    double dJL = minmod(t.aJL, t.dJc), dJR = minmod(t.aJR, t.dJc);
    double dfrL = minmod(t.afrL, t.dfrc), dfrR = minmod(t.afrR, t.dfrc);
    double dfZL = minmod(t.afZL, t.dfZc), dfZR = minmod(t.afZR, t.dfZc);
    t.JL = ci.J + dJL * dL;
    t.JR = cp1.J - dJR * dR;
    o.J_L = t.JL > jeps ? t.JL : jeps;
    o.J_R = t.JR > jeps ? t.JR : jeps;
    t.frL0 = ci.fr + dfrL * dL;
    t.frR0 = cp1.fr - dfrR * dR;
    t.fZL0 = ci.fZ + dfZL * dL;
    t.fZR0 = cp1.fZ - dfZR * dR;
    double frL = t.frL0, fZL = t.fZL0, frR = t.frR0, fZR = t.fZR0;
    // |f| and 1/|f| from one reciprocal square root, as reconstruct_f forms them
    const double sL = frL * frL + fZL * fZL, sR = frR * frR + fZR * fZR;
    double iL = sL >= kDblMinNormal ? rsqrt_nr(sL) : 0.0;
    double iR = sR >= kDblMinNormal ? rsqrt_nr(sR) : 0.0;
    double fL = sL * iL, fR = sR * iR;
    t.fL0 = fL;
    t.fR0 = fR;
    if (fL > 1.0) { frL *= iL; fZL *= iL; fL = 1.0; iL = 1.0; }
    if (fR > 1.0) { frR *= iR; fZR *= iR; fR = 1.0; iR = 1.0; }
    o.Hr_L = frL * o.J_L; o.Hr_R = frR * o.J_R;
    o.HZ_L = fZL * o.J_L; o.HZ_R = fZR * o.J_R;
    o.nr_L = frL * iL; o.nZ_L = fZL * iL;
    o.nr_R = frR * iR; o.nZ_R = fZR * iR;
    o.f_L = fL; o.f_R = fR;
}

// Adjoint of one side's reduced flux: (fr0, fZ0) -> (fr, fZ, |f|, n) with the causality
// renormalisation |f| <= 1; g* are the adjoints of the side's outputs fr, fZ (through H and
// n) and f.
__device__ __forceinline__ void adj_side_f(double fr0, double fZ0, double f0, double J, double gH_r, double gH_Z,
                                           double gf, double gn_r, double gn_Z, double &gfr0, double &gfZ0,
                                           double &gJ) {
    // outputs: H = f_vec * J, n = f_vec / |f_vec|, f = |f_vec| (all after renormalisation)
    double fr = fr0, fZ = fZ0, f = f0;
    const bool ren = f0 > 1.0;
    const double if0 = f0 > 0.0 ? rcp<double>(f0) : 0.0;
    if (ren) { fr = fr0 * if0; fZ = fZ0 * if0; f = 1.0; }
    gJ += gH_r * fr + gH_Z * fZ;
    double gfr = gH_r * J, gfZ = gH_Z * J;
    double gfm = ren ? 0.0 : gf;                  // after renormalisation |f| is the constant 1
    if (f > 0.0) {
        double inv = rcp<double>(f);
        double nr = fr * inv, nZ = fZ * inv;
        gfr += gn_r * inv;
        gfZ += gn_Z * inv;
        gfm += -(gn_r * nr + gn_Z * nZ) * inv;
    }
    if (ren) {
        // v / |v| with v = (fr0, fZ0): d = (g - u (u . g)) / |v|, u = v / |v|
        double ur = fr, uZ = fZ;
        double dot = ur * gfr + uZ * gfZ;
        gfr0 += (gfr - ur * dot) * if0;
        gfZ0 += (gfZ - uZ * dot) * if0;
    } else {
        gfr0 += gfr;
        gfZ0 += gfZ;
        if (f0 > 0.0) {
            gfr0 += gfm * fr0 * if0;
            gfZ0 += gfm * fZ0 * if0;
        }
    }
}

// Adjoint of ReconstructInterface. g.o holds the adjoints of the Recon outputs; the stencil
// adjoints gc[0..3] (J, fr, fZ) and the alpha_F adjoints are accumulated.
__device__ __forceinline__ void adj_recon(const ReconT &t, const CellF<double> cs[4], const double iv[5], double jeps,
                                          const Recon<double> &g, CellF<double> gc[4], double &gaFi, double &gaFp) {
    const double dL = iv[0], dR = iv[1];
    gaFi += g.tau_L * dL;
    gaFp += g.tau_R * dR;
    double gfrL0 = 0.0, gfZL0 = 0.0, gfrR0 = 0.0, gfZR0 = 0.0, gJ_L = g.J_L, gJ_R = g.J_R;
    adj_side_f(t.frL0, t.fZL0, t.fL0, t.o.J_L, g.Hr_L, g.HZ_L, g.f_L, g.nr_L, g.nZ_L, gfrL0, gfZL0, gJ_L);
    adj_side_f(t.frR0, t.fZR0, t.fR0, t.o.J_R, g.Hr_R, g.HZ_R, g.f_R, g.nr_R, g.nZ_R, gfrR0, gfZR0, gJ_R);
    // floors
    double gJL = t.JL > jeps ? gJ_L : 0.0;
    double gJR = t.JR > jeps ? gJ_R : 0.0;
    // JL = ci.J + dJL dL ; JR = cp1.J - dJR dR (and the same for fr, fZ)
    double gdJL = gJL * dL, gdJR = -gJR * dR;
    double gdfrL = gfrL0 * dL, gdfrR = -gfrR0 * dR, gdfZL = gfZL0 * dL, gdfZR = -gfZR0 * dR;
    gc[1].J += gJL; gc[2].J += gJR;
    gc[1].fr += gfrL0; gc[2].fr += gfrR0;
    gc[1].fZ += gfZL0; gc[2].fZ += gfZR0;
    // slopes
    double gaJL = 0, gaJR = 0, gdJc = 0;
    adj_minmod(t.aJL, t.dJc, gdJL, gaJL, gdJc);
    adj_minmod(t.aJR, t.dJc, gdJR, gaJR, gdJc);
    double gafrL = 0, gafrR = 0, gdfrc = 0;
    adj_minmod(t.afrL, t.dfrc, gdfrL, gafrL, gdfrc);
    adj_minmod(t.afrR, t.dfrc, gdfrR, gafrR, gdfrc);
    double gafZL = 0, gafZR = 0, gdfZc = 0;
    adj_minmod(t.afZL, t.dfZc, gdfZL, gafZL, gdfZc);
    adj_minmod(t.afZR, t.dfZc, gdfZR, gafZR, gdfZc);
    // a_L = (ci - cm1) iv2 ; a_R = (cp2 - cp1) iv4 ; c = (cp1 - ci) iv3
    gc[1].J += gaJL * iv[2]; gc[0].J -= gaJL * iv[2];
    gc[3].J += gaJR * iv[4]; gc[2].J -= gaJR * iv[4];
    gc[2].J += gdJc * iv[3]; gc[1].J -= gdJc * iv[3];
    gc[1].fr += gafrL * iv[2]; gc[0].fr -= gafrL * iv[2];
    gc[3].fr += gafrR * iv[4]; gc[2].fr -= gafrR * iv[4];
    gc[2].fr += gdfrc * iv[3]; gc[1].fr -= gdfrc * iv[3];
    gc[1].fZ += gafZL * iv[2]; gc[0].fZ -= gafZL * iv[2];
    gc[3].fZ += gafZR * iv[4]; gc[2].fZ -= gafZR * iv[4];
    gc[2].fZ += gdfZc * iv[3]; gc[1].fZ -= gdfZc * iv[3];
}

// HLL_Eigenvalues (src/M1Closure.jl:273-296) recomputed, with the adjoints gl1, gl3 of the
// clamped outputs taken back to f and mu (+=). The clamps pass a derivative on the branch the
// forward took; sqrt(max(g, 0)) passes none where g <= 0.
__device__ __forceinline__ void adj_hll_eigen(double f0, double mu0, double gl1, double gl3, double &gf,
                                              double &gmu) {
    const bool fin = !(f0 < kFmin) && !(f0 > kFmax);
    const bool muin = !(mu0 < -1.0) && !(mu0 > 1.0);
    double f = f0 < kFmin ? kFmin : (f0 > kFmax ? kFmax : f0);
    double mu = mu0 < -1.0 ? -1.0 : (mu0 > 1.0 ? 1.0 : mu0);
    double f2 = f * f, mu2 = mu * mu, muf = mu * f;
    double t = 4.0 - 3.0 * f2;
    const bool tpos = t > 0.0;      // always (t >= 1): the root and its reciprocal as hll_eigen forms them
    double inv_sq = rsqrt_nr(t);
    double sq = t * inv_sq;
    double g = (2.0 / 3.0) * (4.0 - 3.0 * f2 - sq) + 2.0 * mu2 * (2.0 - f2 - sq);
    const bool gpos = g > 0.0;
    double fac = sqrt(gpos ? g : 0.0);
    double x1 = (muf - fac) * inv_sq, x3 = (muf + fac) * inv_sq;
    double gx1 = (x1 < -1.0 || x1 > 1.0) ? 0.0 : gl1;
    double gx3 = (x3 < -1.0 || x3 > 1.0) ? 0.0 : gl3;
    double gmuf = (gx1 + gx3) * inv_sq;
    double gfac = (gx3 - gx1) * inv_sq;
    double ginv = gx1 * (muf - fac) + gx3 * (muf + fac);
    double gsq = -ginv * inv_sq * inv_sq;
    double gg = gpos && fac > 0.0 ? 0.5 * gfac / fac : 0.0;
    double gf2 = gg * (-2.0 - 2.0 * mu2);
    gsq += gg * (-2.0 / 3.0 - 2.0 * mu2);
    double gmu2 = gg * 2.0 * (2.0 - f2 - sq);
    if (tpos) gf2 += -3.0 * (0.5 * gsq / sq);
    double gfl = gmuf * mu + 2.0 * f * gf2;
    double gml = gmuf * f + 2.0 * mu * gmu2;
    if (fin) gf += gfl;
    if (muin) gmu += gml;
}

// Forward of one face (GLF or HLL flux + upwind advection flux + the K_phiphi face values),
// with its adjoint. Direction ZDIR: false = r face (F_J = H_r, F_Hr = D_rr J, F_HZ = D_rZ J),
// true = Z face (F_J = H_Z, F_Hr = D_rZ J, F_HZ = D_ZZ J). `axis` marks the r = 0 face, whose
// right K_phiphi uses Compute_K_phiphi_InnerAxis. FLUX: 0 = GLF, 1 = HLL.
template <bool ZDIR, int FLUX>
__device__ __forceinline__ void adj_face(const CellF<double> cs[4], const double iv[5], double aFi, double aFp,
                                             double uc, double jeps, bool axis, const double gF[3], double gkL,
                                             double gkR, CellF<double> gc[4], double &gaFi, double &gaFp,
                                             double &guc) {
    ReconT t;
    recon_fwd(cs[0], cs[1], cs[2], cs[3], iv, aFi, aFp, jeps, t);
    const Recon<double> &q = t.o;
    double DrrL, DZZL, DrZL, DrrR, DZZR, DrZR;
    D_from_f_n<double>(q.f_L, q.nr_L, q.nZ_L, DrrL, DZZL, DrZL);
    D_from_f_n<double>(q.f_R, q.nr_R, q.nZ_R, DrrR, DZZR, DrZR);
    Recon<double> g;
    g.J_L = g.J_R = g.Hr_L = g.Hr_R = g.HZ_L = g.HZ_R = g.tau_L = g.tau_R = 0.0;
    g.f_L = g.f_R = g.nr_L = g.nr_R = g.nZ_L = g.nZ_R = 0.0;
    double gDrrL = 0, gDZZL = 0, gDrZL = 0, gDrrR = 0, gDZZR = 0, gDrZR = 0;
    // upwind advection flux: F += uc * (uc < 0 ? Q_R : Q_L)
    {
        const bool up = uc < 0.0;
        guc += gF[0] * (up ? q.J_R : q.J_L) + gF[1] * (up ? q.Hr_R : q.Hr_L) + gF[2] * (up ? q.HZ_R : q.HZ_L);
        if (up) { g.J_R += uc * gF[0]; g.Hr_R += uc * gF[1]; g.HZ_R += uc * gF[2]; }
        else { g.J_L += uc * gF[0]; g.Hr_L += uc * gF[1]; g.HZ_L += uc * gF[2]; }
    }
    // GLF flux with the diffusion-limit blend, src/AdvectJandH.jl:81-118
    if (FLUX == 0) {
        const double FJ_L = ZDIR ? q.HZ_L : q.Hr_L, FJ_R = ZDIR ? q.HZ_R : q.Hr_R;
        const double DaL = ZDIR ? DrZL : DrrL, DaR = ZDIR ? DrZR : DrrR;   // F_Hr = Da J
        const double DbL = ZDIR ? DZZL : DrZL, DbR = ZDIR ? DZZR : DrZR;   // F_HZ = Db J
        double tau = q.tau_L + q.tau_R;
        double num = 0.2 + tau;
        double den = num + tau * tau;
        const double iden = rcp<double>(den);
        double eps = num * iden;
        double ome = 1.0 - eps;
        const bool tpos = tau > Num<double>::tiny();
        double te = tpos ? tau : Num<double>::tiny();
        const double ite = rcp<double>(te);
        double Ji = cs[1].J, Jp = cs[2].J;
        double FJd = -(1.0 / 3.0) * (Jp - Ji) * ite;
        double FJg = 0.5 * (FJ_L + FJ_R) - 0.5 * (q.J_R - q.J_L);
        double he = 0.5 * eps;
        double geps = gF[0] * (FJg - FJd) - 0.5 * (gF[1] * (q.Hr_R - q.Hr_L) + gF[2] * (q.HZ_R - q.HZ_L));
        double gFJg = gF[0] * eps, gFJd = gF[0] * ome;
        double gFJ_L = 0.5 * gFJg, gFJ_R = 0.5 * gFJg;
        g.J_R -= 0.5 * gFJg;
        g.J_L += 0.5 * gFJg;
        // F_Hr = 0.5 (Da_L J_L + Da_R J_R) - he (Hr_R - Hr_L)
        double gDaL = 0.5 * gF[1] * q.J_L, gDaR = 0.5 * gF[1] * q.J_R;
        double gDbL = 0.5 * gF[2] * q.J_L, gDbR = 0.5 * gF[2] * q.J_R;
        g.J_L += 0.5 * (gF[1] * DaL + gF[2] * DbL);
        g.J_R += 0.5 * (gF[1] * DaR + gF[2] * DbR);
        g.Hr_R -= he * gF[1]; g.Hr_L += he * gF[1];
        g.HZ_R -= he * gF[2]; g.HZ_L += he * gF[2];
        if (ZDIR) {
            g.HZ_L += gFJ_L; g.HZ_R += gFJ_R;
            gDrZL += gDaL; gDrZR += gDaR; gDZZL += gDbL; gDZZR += gDbR;
        } else {
            g.Hr_L += gFJ_L; g.Hr_R += gFJ_R;
            gDrrL += gDaL; gDrrR += gDaR; gDrZL += gDbL; gDrZR += gDbR;
        }
        // diffusion term
        double gd = -(1.0 / 3.0) * ite * gFJd;
        gc[2].J += gd;
        gc[1].J -= gd;
        double gte = gFJd * (1.0 / 3.0) * (Jp - Ji) * (ite * ite);
        double gtau = tpos ? gte : 0.0;
        gtau += geps * (tau * tau - 2.0 * tau * num) * (iden * iden);
        g.tau_L += gtau;
        g.tau_R += gtau;
    } else {
        // HLL flux with the diffusion-limit blend, src/AdvectJandH.jl:155-204; wave speeds
        // from M1WaveSpeeds_r/Z, src/M1Closure.jl:301-326
        const double FJ_L = ZDIR ? q.HZ_L : q.Hr_L, FJ_R = ZDIR ? q.HZ_R : q.Hr_R;
        const double DaL = ZDIR ? DrZL : DrrL, DaR = ZDIR ? DrZR : DrrR;   // F_Hr = Da J
        const double DbL = ZDIR ? DZZL : DrZL, DbR = ZDIR ? DZZR : DrZR;   // F_HZ = Db J
        const double FHr_L = DaL * q.J_L, FHr_R = DaR * q.J_R, FHZ_L = DbL * q.J_L, FHZ_R = DbR * q.J_R;
        double tau = q.tau_L + q.tau_R;
        double num = 0.2 + tau;
        double den = num + tau * tau;
        const double iden = rcp<double>(den);
        double eps = num * iden;
        double ome = 1.0 - eps;
        const bool tpos = tau > Num<double>::tiny();
        double te = tpos ? tau : Num<double>::tiny();
        const double ite = rcp<double>(te);
        double Ji = cs[1].J, Jp = cs[2].J;
        double FJd = -(1.0 / 3.0) * (Jp - Ji) * ite;
        const double muL = ZDIR ? q.nZ_L : q.nr_L, muR = ZDIR ? q.nZ_R : q.nr_R;
        double l1L, l3L, l1R, l3R;
        hll_eigen<double>(q.f_L, muL, l1L, l3L);
        hll_eigen<double>(q.f_R, muR, l1R, l3R);
        double m3 = fmax(l3L, l3R), m1 = fmin(l1L, l1R);
        double SR = fmax(m3, 0.0), SL = fmin(m1, 0.0);
        double dS = SR - SL;
        const bool dpos = dS > Num<double>::tiny();
        double inv = rcp<double>(dpos ? dS : Num<double>::tiny());
        double SRSL = SR * SL;
        double dJ = q.J_R - q.J_L, dHr = q.Hr_R - q.Hr_L, dHZ = q.HZ_R - q.HZ_L;
        double nJ = SR * FJ_L - SL * FJ_R + SRSL * dJ;
        double nHr = SR * FHr_L - SL * FHr_R + SRSL * dHr;
        double nHZ = SR * FHZ_L - SL * FHZ_R + SRSL * dHZ;
        double hom = 0.5 * ome;
        double geps = gF[0] * (nJ * inv - FJd) + gF[1] * (nHr * inv - 0.5 * (FHr_L + FHr_R)) +
                      gF[2] * (nHZ * inv - 0.5 * (FHZ_L + FHZ_R));
        double gJh = gF[0] * eps, gHrh = gF[1] * eps, gHZh = gF[2] * eps, gFJd = gF[0] * ome;
        // physical fluxes
        double gFJ_L = gJh * SR * inv, gFJ_R = -gJh * SL * inv;
        double gFHr_L = gHrh * SR * inv + gF[1] * hom, gFHr_R = -gHrh * SL * inv + gF[1] * hom;
        double gFHZ_L = gHZh * SR * inv + gF[2] * hom, gFHZ_R = -gHZh * SL * inv + gF[2] * hom;
        // jumps of the states
        double cJ = gJh * SRSL * inv, cHr = gHrh * SRSL * inv, cHZ = gHZh * SRSL * inv;
        g.J_R += cJ; g.J_L -= cJ;
        g.Hr_R += cHr; g.Hr_L -= cHr;
        g.HZ_R += cHZ; g.HZ_L -= cHZ;
        // wave speeds
        double gSR = (gJh * (FJ_L + SL * dJ) + gHrh * (FHr_L + SL * dHr) + gHZh * (FHZ_L + SL * dHZ)) * inv;
        double gSL = (gJh * (SR * dJ - FJ_R) + gHrh * (SR * dHr - FHr_R) + gHZh * (SR * dHZ - FHZ_R)) * inv;
        if (dpos) {
            double gdS = -(gJh * nJ + gHrh * nHr + gHZh * nHZ) * inv * inv;
            gSR += gdS;
            gSL -= gdS;
        }
        double gl1L = 0.0, gl3L = 0.0, gl1R = 0.0, gl3R = 0.0;
        if (m3 > 0.0) { if (l3L >= l3R) gl3L = gSR; else gl3R = gSR; }
        if (m1 < 0.0) { if (l1L <= l1R) gl1L = gSL; else gl1R = gSL; }
        double gmuL = 0.0, gmuR = 0.0;
        adj_hll_eigen(q.f_L, muL, gl1L, gl3L, g.f_L, gmuL);
        adj_hll_eigen(q.f_R, muR, gl1R, gl3R, g.f_R, gmuR);
        g.J_L += gFHr_L * DaL + gFHZ_L * DbL;
        g.J_R += gFHr_R * DaR + gFHZ_R * DbR;
        double gDaL = gFHr_L * q.J_L, gDaR = gFHr_R * q.J_R, gDbL = gFHZ_L * q.J_L, gDbR = gFHZ_R * q.J_R;
        if (ZDIR) {
            g.nZ_L += gmuL; g.nZ_R += gmuR;
            g.HZ_L += gFJ_L; g.HZ_R += gFJ_R;
            gDrZL += gDaL; gDrZR += gDaR; gDZZL += gDbL; gDZZR += gDbR;
        } else {
            g.nr_L += gmuL; g.nr_R += gmuR;
            g.Hr_L += gFJ_L; g.Hr_R += gFJ_R;
            gDrrL += gDaL; gDrrR += gDaR; gDrZL += gDbL; gDrZR += gDbR;
        }
        // diffusion term and the blend weight, as in the GLF branch
        double gd = -(1.0 / 3.0) * ite * gFJd;
        gc[2].J += gd;
        gc[1].J -= gd;
        double gte = gFJd * (1.0 / 3.0) * (Jp - Ji) * (ite * ite);
        double gtau = tpos ? gte : 0.0;
        gtau += geps * (tau * tau - 2.0 * tau * num) * (iden * iden);
        g.tau_L += gtau;
        g.tau_R += gtau;
    }
    // K_phiphi at the face (r faces only): kL = clamp01(1 - DrrL - DZZL) J_L, kR likewise or
    // the axis form
    if (!ZDIR) {
        double qL = 1.0 - DrrL - DZZL;
        double qLc = qL < 0.0 ? 0.0 : (qL > 1.0 ? 1.0 : qL);
        g.J_L += gkL * qLc;
        if (qL > 0.0 && qL < 1.0) { gDrrL -= gkL * q.J_L; gDZZL -= gkL * q.J_L; }
        if (!axis) {
            double qR = 1.0 - DrrR - DZZR;
            double qRc = qR < 0.0 ? 0.0 : (qR > 1.0 ? 1.0 : qR);
            g.J_R += gkR * qRc;
            if (qR > 0.0 && qR < 1.0) { gDrrR -= gkR * q.J_R; gDZZR -= gkR * q.J_R; }
        } else if (gkR != 0.0) {
            // Compute_K_phiphi_InnerAxis(J_R, HZ_R), src/AdvectJandH.jl:499-522
            const bool jf = q.J_R > jeps;
            double J = jf ? q.J_R : jeps;
            double fZ0 = q.HZ_R / J;
            const bool fin = fZ0 > -1.0 && fZ0 < 1.0;
            double fZ = fZ0 < -1.0 ? -1.0 : (fZ0 > 1.0 ? 1.0 : fZ0);
            double f = fabs(fZ);
            double nZ = f > 0.0 ? (fZ > 0.0 ? 1.0 : -1.0) : 0.0;
            double Dr, DZ, DrZ_;
            D_from_f_n<double>(f, 0.0, nZ, Dr, DZ, DrZ_);
            double kq = 1.0 - Dr - DZ;
            double kqc = kq < 0.0 ? 0.0 : (kq > 1.0 ? 1.0 : kq);
            double gJ = gkR * kqc;
            if (kq > 0.0 && kq < 1.0) {
                double gf = 0, gnr = 0, gnZ = 0;
                adj_D_from_f_n(f, 0.0, nZ, -gkR * J, -gkR * J, 0.0, gf, gnr, gnZ);
                double gfZ = (fZ > 0.0 ? gf : (fZ < 0.0 ? -gf : 0.0));
                if (fin) {
                    g.HZ_R += gfZ / J;
                    gJ += -gfZ * fZ0 / J;
                }
            }
            if (jf) g.J_R += gJ;
        }
    }
    adj_D_from_f_n(q.f_L, q.nr_L, q.nZ_L, gDrrL, gDZZL, gDrZL, g.f_L, g.nr_L, g.nZ_L);
    adj_D_from_f_n(q.f_R, q.nr_R, q.nZ_R, gDrrR, gDZZR, gDrZR, g.f_R, g.nr_R, g.nZ_R);
    adj_recon(t, cs, iv, jeps, g, gc, gaFi, gaFp);
}

// cell_f: (J, Hr, HZ) -> (J, fr = Hr / max(J, jeps), fZ = HZ / max(J, jeps))
__device__ __forceinline__ void adj_cell_f(double J, double Hr, double HZ, double jeps, const CellF<double> &g,
                                           double &gJ, double &gHr, double &gHZ) {
    const bool jf = J > jeps;
    double iJ = rcp<double>(jf ? J : jeps);
    gHr += g.fr * iJ;
    gHZ += g.fZ * iJ;
    gJ += g.J;
    if (jf) gJ += -(g.fr * Hr + g.fZ * HZ) * iJ * iJ;
}

}  // namespace lyd
