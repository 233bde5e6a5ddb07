// lyd_species.cuh -- per-cell Lyman-alpha quantities of the gas state, FP64, for the device:
// the destruction probability, the recombination and collisional emissivities and the line
// opacity at line centre. Each function restates one piece of the LYDION reference (paths
// inside its source tree).
#pragma once
#include "lyd_physics.cuh"

namespace lyd {

// pd_Lya, src/LymanAlphaDestruction.jl:43-97
__device__ __forceinline__ double pd_lya_dev(double nHII, double ne, double nHI, double nHeI, double nH2, double T, double z) {
    T = fmin(fmax(T, 1.0), 1e5);
    double T100 = T / 100.0;
    double lT = log10(T);
    double lT2 = lT * lT, lT3 = lT2 * lT, lT4 = lT3 * lT;
    double Gp2s = 3.1e-6 * (1.0 + z);
    double Gs2p = 3.0 * Gp2s;
    double r25 = 2.5 / T;
    double Ce = 5e-5 * exp(-(r25 * r25)) * ne / (1.0 + pow(T100, 0.45));
    double CHII = (6.98e-3 * (1.0 + 0.933 * lT) * exp(-pow(601.0 / T, 0.406)) / pow(T, 0.5) +
                   pow(10.0, -7.69 + 1.21 * lT + 0.455 * lT2 - 0.199 * lT3 + 0.0182 * lT4)) * nHII;
    double CHeI = 2.6e-9 * pow(T100, 0.315) * nHeI;
    double CH2 = 1.7e-9 * pow(T100, 0.3) * nH2;
    double den = 8.9 * pow(T, -0.55) + 0.078 * pow(T, 0.35);
    double CHI = (4.1e-11 * exp(-pow(1.6 / T, 0.75) - 0.15 * T) + (1.6e-10 + 1.57e-12 * pow(T, 1.1)) / (den * den)) * nHI;
    double Cs2p = Ce + CHII + CHeI + CH2 + CHI;
    double Cp2s = (1.0 / 3.0) * Cs2p;
    double Rp2s = (2.0 / 3.0) * kA2p2s + Cp2s + Gp2s;
    double Rs2p = kA2s2p + Cs2p + Gs2p;
    double pdHI = Rp2s / ((kALya / kA2g) * (kA2g + Rs2p) + Rp2s);
    double pdH2 = 0.0;
    if (nHI > 1e-20) {
        double num = 33.0 * exp(-14540.0 / T) + 13.0 * exp(-15564.0 / T);
        double dd = 46.0 + 1e3 * exp(-pow(1e3 / T, 1.5));
        pdH2 = fmin(num / dd, 1.3e-3) * (nH2 / nHI);
    }
    return fmin(pdHI + pdH2, 1.0);
}

// Line-centre cross-section sigma0(T) (src/ConstantsAndFunctions.jl, Compute_sigma0):
// sqrt(pi) e^2 f_12 / (m_e nu_Lya) / b(T).
constexpr double kEChargeEsu = 4.80320451e-10, kMElec = 9.109382917e-28, kF12Lya = 0.41641;
__host__ __device__ __forceinline__ double compute_sigma0(double T) {
    return (sqrt(kPi) * (kEChargeEsu * kEChargeEsu) * kF12Lya / (kMElec * kNuLya)) / compute_b(T);
}

// Probability of Lyman-alpha emission after a recombination, Storey & Hummer (1995): the
// tables of src/LymanAlphaEmission.jl:36-65 (rows: T = 5e2 .. 3e4 K; columns: n_e = 1e2 ..
// 1e14 cm^-3 for Case B, 1e2 .. 1e10 for Case A), interpolated bilinearly in
// (log10 T, log10 n_e) with the arguments clamped to the grids (src/LymanAlphaEmission.jl:71-90).
__constant__ double kShB[10][13] = {
    {0.80793637, 0.90215197, 0.98157401, 0.9970534, 0.99933853, 0.99934845, 0.99967896, 0.99948547, 0.99931146, 0.99951894, 0.9997498, 0.99864818, 0.99372263},
    {0.78439303, 0.87743841, 0.97423464, 0.99680114, 0.99960243, 0.99967816, 0.9997671, 0.99939133, 0.99922946, 0.99960973, 0.99937386, 0.99906812, 0.9954834},
    {0.74159266, 0.82809599, 0.95734434, 0.99359891, 0.99892162, 0.99927343, 0.99979471, 0.99938909, 0.99899055, 0.99925979, 0.99957955, 0.99923525, 0.99703571},
    {0.71946081, 0.80133228, 0.94581237, 0.99246182, 0.99848958, 0.99940329, 0.99949246, 0.99952048, 0.99981447, 0.99956726, 0.9993515, 0.99952024, 0.99692499},
    {0.70117195, 0.7788453, 0.93441344, 0.99075058, 0.99831301, 0.99960223, 0.99940949, 0.99946884, 0.99948297, 0.99947146, 0.99965311, 0.99918254, 0.99690311},
    {0.68808416, 0.76220739, 0.92503048, 0.9891268, 0.99828523, 0.9994074, 0.99944339, 0.99952601, 0.99932358, 0.99927528, 0.99938987, 0.99904232, 0.9949615},
    {0.6775581, 0.74868826, 0.9176273, 0.98784252, 0.99835238, 0.99903921, 0.99977064, 0.99954296, 0.99930529, 0.99954743, 0.99944997, 0.99874439, 0.9916493},
    {0.66862468, 0.73785038, 0.91033402, 0.98701405, 0.99817046, 0.99892625, 0.99953078, 0.99960556, 0.9993362, 0.99941558, 0.99944365, 0.99828039, 0.98817287},
    {0.65534642, 0.72080463, 0.89823705, 0.98497224, 0.99798854, 0.9988133, 0.99929092, 0.99909416, 0.99933199, 0.9995549, 0.99924446, 0.99764512, 0.97960152},
    {0.63566376, 0.69600394, 0.87952243, 0.98121463, 0.99716593, 0.99896144, 0.99905958, 0.9996252, 0.99953649, 0.99931002, 0.99872497, 0.99561256, 0.96391965}};
__constant__ double kShA[10][9] = {
    {0.58042473, 0.59595911, 0.60335363, 0.58990186, 0.56623927, 0.53426043, 0.492528, 0.44534414, 0.40955195},
    {0.54712958, 0.56465163, 0.57999443, 0.57241623, 0.5541246, 0.5276139, 0.49052298, 0.44606687, 0.4101595},
    {0.48320245, 0.50151448, 0.52818381, 0.53008608, 0.52008701, 0.50298698, 0.47625175, 0.43924427, 0.40696841},
    {0.44933274, 0.46714191, 0.49852558, 0.50475148, 0.49815515, 0.48505756, 0.46319941, 0.43069186, 0.40125666},
    {0.42087234, 0.43810743, 0.47280049, 0.48268151, 0.47821493, 0.46794659, 0.4497736, 0.42097532, 0.39442497},
    {0.40023971, 0.41675887, 0.45373431, 0.46591319, 0.46300415, 0.45454038, 0.43876097, 0.41249415, 0.38810578},
    {0.3840314, 0.40007514, 0.43832241, 0.45257107, 0.45064954, 0.4434932, 0.42939783, 0.40511911, 0.38230403},
    {0.37046215, 0.38617473, 0.42546609, 0.44143608, 0.44049428, 0.43394168, 0.42127472, 0.39854551, 0.37684759},
    {0.34937867, 0.36397106, 0.40484801, 0.42349201, 0.42367822, 0.41860328, 0.40761256, 0.38699493, 0.36739625},
    {0.31960139, 0.33302781, 0.37528203, 0.39805701, 0.39984039, 0.39602958, 0.38718651, 0.36963656, 0.3518518}};

__constant__ double kShT[10] = {5e2, 1e3, 3e3, 5e3, 7.5e3, 1e4, 1.25e4, 1.5e4, 2e4, 3e4};

__device__ __forceinline__ double prob_lya_sh95(double T, double ne, bool caseB) {
    const int nne = caseB ? 13 : 9;
    double lT0 = log10(kShT[0]), lT9 = log10(kShT[9]);
    double x = log10(T), y = log10(ne);
    x = x < lT0 ? lT0 : (x > lT9 ? lT9 : x);
    const double lne0 = 2.0, lneN = caseB ? 14.0 : 10.0;    // the n_e grids are 10^2 .. 10^(nne+1)
    y = y < lne0 ? lne0 : (y > lneN ? lneN : y);
    int i = 0;
    while (i < 8 && x > log10(kShT[i + 1])) i++;
    int j = (int)floor(y - lne0);
    j = j < 0 ? 0 : (j > nne - 2 ? nne - 2 : j);
    const double xi = log10(kShT[i]), xi1 = log10(kShT[i + 1]);
    const double yj = log10(pow(10.0, lne0 + j)), yj1 = log10(pow(10.0, lne0 + j + 1));
    const double t = (x - xi) / (xi1 - xi), u = (y - yj) / (yj1 - yj);
    double v00, v10, v01, v11;
    if (caseB) { v00 = kShB[i][j]; v10 = kShB[i + 1][j]; v01 = kShB[i][j + 1]; v11 = kShB[i + 1][j + 1]; }
    else { v00 = kShA[i][j]; v10 = kShA[i + 1][j]; v01 = kShA[i][j + 1]; v11 = kShA[i + 1][j + 1]; }
    return (1.0 - t) * ((1.0 - u) * v00 + u * v01) + t * ((1.0 - u) * v10 + u * v11);
}

// H II recombination rate, Case B (on-the-spot) or Case A, the fits of
// src/PhotoChemistryAndCooling/GasChemistryRates.jl:166-204
__device__ __forceinline__ double krec_hii(double T, bool ots) {
    T = T < 1.0 ? 1.0 : (T > 1e9 ? 1e9 : T);
    const double lam = 315614.0 / T;
    if (ots) return 2.753e-14 * pow(lam, 1.5) / pow(1.0 + pow(lam / 2.74, 0.407), 2.242);
    return 1.269e-13 * pow(lam, 1.503) / pow(1.0 + pow(lam / 0.522, 0.47), 1.923);
}

constexpr double kNuLyC = 3.289842e15;
constexpr double kELyaOver4Pi = kHPlanck * kNuLya / kFourPi;

// Frequency-integrated emissivity from recombinations, src/LymanAlphaEmission.jl:106-131
__device__ __forceinline__ double js_rec_lya(double T, double nHII, double ne, bool ots) {
    return prob_lya_sh95(T, ne, ots) * krec_hii(T, ots) * nHII * ne * kELyaOver4Pi;
}

// ... from collisional excitation (Smith et al. 2022 fits), src/LymanAlphaEmission.jl:148-175
__device__ __forceinline__ double js_coll_lya(double T, double nHI, double ne) {
    constexpr double Tryd = kHPlanck * kNuLyC / kKBoltz;
    T = T > 1.0 ? T : 1.0;
    const double iT = 1.0 / T;
    const double T6 = (T < 3e5 ? T : 3e5) * 1e-6, T62 = T6 * T6, T63 = T62 * T6;
    const double Y12 = 0.267486 + 1.57257 * T6 - 6.44026 * T62 + 11.5401 * T63;
    const double Y13 = 0.0940821 + 2.90748 * T6 - 6.69528 * T62 + 7.86419 * T63;
    const double Y14 = 0.0415028 + 1.13673 * T6 - 3.97454 * T62 + 6.05941 * T63;
    const double Y15 = 0.032277 + 0.40856 * T6 - 1.34604 * T62 + 2.07558 * T63;
    const double q = (8.63e-6 / (2.0 * sqrt(T))) *
                     (Y12 * exp(-(0.75 * Tryd) * iT) + Y13 * exp(-((8.0 / 9.0) * Tryd) * iT) +
                      Y14 * exp(-((15.0 / 16.0) * Tryd) * iT) + Y15 * exp(-((24.0 / 25.0) * Tryd) * iT));
    return q * nHI * ne * kELyaOver4Pi;
}

}  // namespace lyd
