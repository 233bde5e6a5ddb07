// lyd_kernels.cu -- the hot kernels of the Lyman-alpha M1 step on sm_100a.
//
//  k_advect   AdvectJandH_Cylindrical! (src/AdvectJandH.jl:526-1390) as ONE kernel. A CTA owns a
//             tile of 8 columns (r) x `rows` rows (Z) x 32 bins (one bin per lane, k innermost,
//             so every warp load is a contiguous 256 B / 128 B run) of one cloud and marches up
//             the tile row by row. Face fluxes never touch HBM: the six face-flux arrays and the
//             two K_phiphi arrays of the reference are replaced by shared memory and registers.
//             Ghost cells of the four boundaries are produced on the fly from the boundary
//             conditions.
//  k_freq     LyaEmissionAbsorptionUpdate! + UpdateFreqFactors! + the per-cell tridiagonal solve
//             + the flux correction of FrequencyUpdateJLya_AllCells!, fused per cell: one warp
//             owns one cell's whole spectrum (M contiguous bins per lane), the k +- 1 couplings
//             travel by warp shuffles, and the tridiagonal system is solved in FP64, by parallel
//             cyclic reduction across the warp or by a lane-serial elimination. The epilogue
//             accumulates the next step's FindActiveBins energies and the step diagnostics into
//             per-CTA partials (fixed order, so results are run-to-run deterministic).
//  k_reduce   one CTA per cloud sums that cloud's partials and derives kmin/kmax, M_F, L, f_esc.
#include <cuda_runtime.h>

#include "lyd_internal.h"
#include "lyd_physics.cuh"

namespace lyd {

constexpr int FREQ_THREADS = 256;

// Per-CTA view of one cloud of a batch.
struct View {
    long long o3, oc, orf, ozf;
    int ocol, orow, orint, ozint;
    int nr, nz, bcl, bcr, bzb, bzt;
    int jend;            // end of the rows the tiles update
    double ctdt;
};

__device__ __forceinline__ void load_view(const CloudDesc &d, View &v) {
    v.o3 = d.o3; v.oc = d.oc; v.orf = d.orf; v.ozf = d.ozf;
    v.ocol = d.ocol; v.orow = d.orow; v.orint = d.orint; v.ozint = d.ozint;
    v.nr = d.nr; v.nz = d.nz; v.bcl = d.bc_r_left; v.bcr = d.bc_r_right; v.bzb = d.bc_z_bot; v.bzt = d.bc_z_top;
    v.jend = d.j_own1;
    v.ctdt = d.ctdt;
}

template <typename S, typename R>
__device__ __forceinline__ Cell<R> ld_cell(const AdvArgs<S> &a, const View &v, int i, int j, int k) {
    long long x = v.o3 + (long long)k + (long long)a.nnu * ((long long)i + (long long)v.nr * j);
    Cell<R> c;
    c.J = R(__ldg(a.J + x));
    c.Hr = R(__ldg(a.Hr + x));
    c.HZ = R(__ldg(a.HZ + x));
    return c;
}

// Radial stencil cell with the ghost cells of src/AdvectJandH.jl:662-673 (axis, always
// reflecting) and 853-871 (outer boundary, reflecting or outflow); on a Cartesian grid the
// first X interface reflects or lets flow out (src/AdvectJandH.jl:1528-1545: both ghosts take
// cell 1 with H_X = min(H_X, 0)).
template <typename S, typename R>
__device__ __forceinline__ Cell<R> r_cell(const AdvArgs<S> &a, const View &v, int idx, int j, int k) {
    if (idx < 0) {
        if (v.bcl == 0) {
            Cell<R> c = ld_cell<S, R>(a, v, -1 - idx, j, k);
            c.Hr = -c.Hr;
            return c;
        }
        Cell<R> c = ld_cell<S, R>(a, v, 0, j, k);
        c.Hr = c.Hr < R(0) ? c.Hr : R(0);
        return c;
    }
    if (idx >= v.nr) {
        if (v.bcr == 0) {
            Cell<R> c = ld_cell<S, R>(a, v, 2 * v.nr - 1 - idx, j, k);
            c.Hr = -c.Hr;
            return c;
        }
        Cell<R> c = ld_cell<S, R>(a, v, v.nr - 1, j, k);
        c.Hr = c.Hr > R(0) ? c.Hr : R(0);
        return c;
    }
    return ld_cell<S, R>(a, v, idx, j, k);
}

// Vertical stencil cell with the ghost cells of src/AdvectJandH.jl:1000-1018 (bottom) and
// 1185-1203 (top).
template <typename S, typename R>
__device__ __forceinline__ Cell<R> z_cell(const AdvArgs<S> &a, const View &v, int i, int idx, int k) {
    if (idx < 0) {
        if (v.bzb == 0) {
            Cell<R> c = ld_cell<S, R>(a, v, i, -1 - idx, k);
            c.HZ = -c.HZ;
            return c;
        }
        Cell<R> c = ld_cell<S, R>(a, v, i, 0, k);
        c.HZ = c.HZ < R(0) ? c.HZ : R(0);
        return c;
    }
    if (idx >= v.nz) {
        if (v.bzt == 0) {
            Cell<R> c = ld_cell<S, R>(a, v, i, 2 * v.nz - 1 - idx, k);
            c.HZ = -c.HZ;
            return c;
        }
        Cell<R> c = ld_cell<S, R>(a, v, i, v.nz - 1, k);
        c.HZ = c.HZ > R(0) ? c.HZ : R(0);
        return c;
    }
    return ld_cell<S, R>(a, v, i, idx, k);
}

// alpha_F of an in-grid cell: explicit array, or alpha*H_voigt (+ alpha_cF) as set up by
// src/StaticCloudTest.jl:283-285 and PhotoThermoChemistry.jl:2151.
template <typename S, typename R>
__device__ __forceinline__ R alpha_F(const AdvArgs<S> &a, const View &v, int i, int j, int k) {
    long long c = v.oc + (long long)i + (long long)v.nr * j;
    long long x = v.o3 + (long long)k + (long long)a.nnu * ((long long)i + (long long)v.nr * j);
    if (a.aF) return R(__ldg(a.aF + x));
    R val = R(__ldg(a.alpha + c)) * R(__ldg(a.Hv + x));
    if (a.alpha_cF) val = val + R(__ldg(a.alpha_cF + c));
    return val;
}

// Asynchronous global -> shared copy of one 4- or 8-byte element (cp.async, L1-allocating).
template <typename T>
__device__ __forceinline__ void cp_async_el(T *dst, const T *src) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "element size");
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src) : "memory");
}
// Asynchronous global -> shared copy of 16 bytes (cp.async.cg: L2 only, the rows are streamed).
__device__ __forceinline__ void cp_async_16(void *dst, const void *src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- bulk tensor copies (TMA) into shared memory, completed on an mbarrier -------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// One arrival that also announces `bytes` of copies that will complete on the barrier.
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase `parity` of the barrier to complete; gives up after a bounded number of
// polls (each poll itself returns after a short hardware time limit) and reports false.
constexpr int kMbarPolls = 1 << 20;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity) {
    for (int it = 0; it < kMbarPolls; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Orders this thread's view of earlier generic-proxy shared-memory accesses (made visible to
// it by a barrier) before the bulk copies it issues next into the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// A 3-D tile of a tensor in this GPU's global memory (the map's own buffer) into shared memory;
// x, y, z are the element coordinates of the tile's first element (x * element size a multiple
// of 16 bytes; y may be negative, out-of-range elements read as zero). No multicast.
__device__ __forceinline__ void tma_load_3d(void *dst, const void *map, int x, int y, int z,
                                            unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// ---- k_advect: one CTA = 8 columns (r) x `rows` rows (Z) x 32 bins, marching up in Z --------
//
// A ring of four rows holds, for the 8 own columns and the 2 + 2 halo columns of each row, the
// cell values every face needs: J, the reduced fluxes H/max(J, Jeps) (so the reciprocal of J is
// taken once per cell, not once per face) and alpha_F (formed once per cell, not at each of the
// four face sides that read it); a ring of three rows holds the state of the own columns for
// the cell update. With FP64 arithmetic and per-lane staging the halo columns keep one row and
// every staged input comes a row ahead by cp.async (PFR below): the tile (76 KB) runs at three
// CTAs per SM. Warp w (0..7) owns
// column i0+w; warp 8 stages the halo columns and computes the tile's rightmost r face. Per row: stage row j+2 -> sync -> every warp
// computes the r face on its left (warp 8: the right edge) into shared memory and its Z face
// j+1/2 into registers -> sync -> the cell update of row j uses the two r faces from shared
// memory and the Z faces j-1/2 (carried from the previous row) and j+1/2.
constexpr int MT = 8;                  // own columns per CTA
constexpr int MWARPS = MT + 1;
constexpr int MTHREADS = 32 * MWARPS;
constexpr int MCOL = MT + 4;           // staged columns i0-2 .. i0+MT+1
constexpr int RING = 4;
// staged fields per cell: J, f_r, f_Z and alpha_F (formed once per staged cell; four face sides
// read each cell's)
template <typename R> __host__ __device__ constexpr int nf() { return 4; }
// The own columns' state (J, H_r, H_Z in the storage type) is kept for the rows j .. j+2 only
// (staged at j+2, updated at j): a ring of three slots.
constexpr int HRING = 3;
__host__ __device__ constexpr int hslot(int r) { return ((r % HRING) + HRING) % HRING; }

// The staged-cell ring A: [RING][MCOL][nf][32] (staged column lc, ring slot of the row), or with
// H1 the own columns' ring [RING][MT][nf][32] followed by one row of the four halo columns
// (lc 0, 1, MT+2, MT+3) [4][nf][32]: with per-lane staging the halo of row j is staged for and
// read by row j's r faces alone, so one row of it suffices (12 KB less in FP64).
template <typename R, bool H1>
__device__ __forceinline__ R *a_cell(R *A, int slot, int lc) {
    if constexpr (H1) {
        if (lc >= 2 && lc < MT + 2) return A + ((slot * MT + (lc - 2)) * nf<R>()) * 32;
        return A + ((RING * MT + (lc < 2 ? lc : lc - MT)) * nf<R>()) * 32;
    } else {
        return A + ((slot * MCOL + lc) * nf<R>()) * 32;
    }
}
template <typename R, bool H1> __host__ __device__ constexpr int a_cells() { return H1 ? RING * MT + 4 : RING * MCOL; }

template <typename S, typename R>
__device__ __forceinline__ Cell<R> raw_cell(const AdvArgs<S> &a, const View &v, int col, int row, int k) {
    if (col < 0 || col >= v.nr) return r_cell<S, R>(a, v, col, row, k);
    if (row < 0 || row >= v.nz) return z_cell<S, R>(a, v, col, row, k);
    return ld_cell<S, R>(a, v, col, row, k);
}

// Stage cell (col, row) into ring slot `slot`, staged column lc (= col - i0 + 2): the flux
// inputs in the arithmetic type R, and for the tile's own columns the state (J, H_r, H_Z) in
// the storage type S, which the cell update accumulates into.
template <typename S, typename R, bool H1>
__device__ __forceinline__ void stage_cell(const AdvArgs<S> &a, const View &v, R *A, S *Hh, int slot, int lc,
                                           int col, int row, int k, int lane, R jeps) {
    Cell<S> c = raw_cell<S, S>(a, v, col, row, k);
    // the alpha_F loads are issued together with the state's (one load latency per cell)
    R aF = R(0);
    if (nf<R>() == 4) {
        int cc = col < 0 ? 0 : (col >= v.nr ? v.nr - 1 : col);
        int rr = row < 0 ? 0 : (row >= v.nz ? v.nz - 1 : row);
        aF = alpha_F<S, R>(a, v, cc, rr, k);
    }
    CellF<R> f = cell_f<R>(R(c.J), R(c.Hr), R(c.HZ), jeps);
    R *p = a_cell<R, H1>(A, slot, lc) + lane;
    p[0] = f.J; p[32] = f.fr; p[64] = f.fZ;
    if (nf<R>() == 4) p[96] = aF;
    if (lc >= 2 && lc < 2 + MT) {
        // the state in S; with S == R the ring's J is the state's J
        constexpr int HF = sizeof(S) == sizeof(R) ? 2 : 3;
        S *q = Hh + ((hslot(row) * MT + (lc - 2)) * HF) * 32 + lane;
        q[0] = c.Hr; q[32] = c.HZ;
        if (HF == 3) q[64] = c.J;
    }
}

// ---- a row ahead by cp.async (FP64 arithmetic with per-lane staging) ----
// The cell a staged stencil cell (col, row) copies, and the boundary rules that r_cell / z_cell
// apply to the copy: rr for H_r, rz for H_Z (1: negate; 2: keep the part <= 0; 3: keep the
// part >= 0). A corner cell (ghost in both directions) is never staged.
struct CellSrc { int i, j, rr, rz; };
__device__ __forceinline__ CellSrc cell_src(const View &v, int col, int row) {
    CellSrc s{col, row, 0, 0};
    if (col < 0) {
        if (v.bcl == 0) { s.i = -1 - col; s.rr = 1; } else { s.i = 0; s.rr = 2; }
    } else if (col >= v.nr) {
        if (v.bcr == 0) { s.i = 2 * v.nr - 1 - col; s.rr = 1; } else { s.i = v.nr - 1; s.rr = 3; }
    } else if (row < 0) {
        if (v.bzb == 0) { s.j = -1 - row; s.rz = 1; } else { s.j = 0; s.rz = 2; }
    } else if (row >= v.nz) {
        if (v.bzt == 0) { s.j = 2 * v.nz - 1 - row; s.rz = 1; } else { s.j = v.nz - 1; s.rz = 3; }
    }
    return s;
}
template <typename S>
__device__ __forceinline__ S bc_rule(S h, int rule) {
    if (rule == 1) return -h;
    if (rule == 2) return h < S(0) ? h : S(0);
    if (rule == 3) return h > S(0) ? h : S(0);
    return h;
}
// A raw slot holds one staged cell's inputs as copied: [4][32] values of the storage type
// (J, H_r, H_Z of the cell it mirrors, and alpha_F, or H_voigt when alpha_F is derived, of the
// in-grid cell it clamps to) and two doubles (alpha and alpha_cF of that cell).
constexpr int RAW_SLOT = 4 * 32 + 2;   // doubles (storage FP64)

// Copies of staged cell (col, row)'s inputs into the raw slot `dst` (cp.async, one 8-byte copy
// per value; lanes outside the active bins copy no bin values; lane 0 copies the per-cell ones).
template <typename S>
__device__ __forceinline__ void raw_issue(const AdvArgs<S> &a, const View &v, S *dst, int col, int row, int k,
                                          int lane, bool kact) {
    const CellSrc s = cell_src(v, col, row);
    const int cc = col < 0 ? 0 : (col >= v.nr ? v.nr - 1 : col);
    const int rr = row < 0 ? 0 : (row >= v.nz ? v.nz - 1 : row);
    const long long cla = (long long)cc + (long long)v.nr * rr;
    if (kact) {
        const long long x = v.o3 + (long long)k + (long long)a.nnu * ((long long)s.i + (long long)v.nr * s.j);
        const long long xa = v.o3 + (long long)k + (long long)a.nnu * cla;
        cp_async_el(dst + lane, a.J + x);
        cp_async_el(dst + 32 + lane, a.Hr + x);
        cp_async_el(dst + 64 + lane, a.HZ + x);
        cp_async_el(dst + 96 + lane, a.aF ? a.aF + xa : a.Hv + xa);
    }
    if (lane == 0 && !a.aF) {
        double *dsc = reinterpret_cast<double *>(dst + 128);
        cp_async_el(dsc, a.alpha + v.oc + cla);
        if (a.alpha_cF) cp_async_el(dsc + 1, a.alpha_cF + v.oc + cla);
    }
}
// stage_cell from a raw slot that raw_issue filled (its copies complete and visible to the
// warp): the same values through the same arithmetic.
template <typename S, typename R, bool H1>
__device__ __forceinline__ void stage_raw(const AdvArgs<S> &a, const View &v, const S *src, R *A, S *Hh, int slot,
                                          int lc, int col, int row, int lane, R jeps) {
    const CellSrc s = cell_src(v, col, row);
    Cell<S> c;
    c.J = src[lane];
    c.Hr = bc_rule(src[32 + lane], s.rr);
    c.HZ = bc_rule(src[64 + lane], s.rz);
    R aF;
    if (a.aF) {
        aF = R(src[96 + lane]);
    } else {
        const double *dsc = reinterpret_cast<const double *>(src + 128);
        aF = R(dsc[0]) * R(src[96 + lane]);
        if (a.alpha_cF) aF = aF + R(dsc[1]);
    }
    CellF<R> f = cell_f<R>(R(c.J), R(c.Hr), R(c.HZ), jeps);
    R *p = a_cell<R, H1>(A, slot, lc) + lane;
    p[0] = f.J; p[32] = f.fr; p[64] = f.fZ; p[96] = aF;
    if (lc >= 2 && lc < 2 + MT) {
        constexpr int HF = sizeof(S) == sizeof(R) ? 2 : 3;
        S *q = Hh + ((hslot(row) * MT + (lc - 2)) * HF) * 32 + lane;
        q[0] = c.Hr; q[32] = c.HZ;
        if (HF == 3) q[64] = c.J;
    }
}

// The raw tile a bulk tensor copy lands for one row: J, H_r, H_Z of the staged columns
// i0-2 .. i0+MT+1 and 32 bins, [field][column][bin] (the copy box is 32 bins x MCOL columns).
// Columns outside 0..n_r-1 land as zeros; for a ghost row (row >= n_z) the copy fetched the row
// it mirrors.
template <typename S>
__host__ __device__ constexpr int raw_tile_bytes() { return 3 * MCOL * 32 * (int)sizeof(S); }

// Stage cell (col, row) into ring slot `slot` from the raw tile, applying the ghost-cell rules
// of r_cell / z_cell: a ghost column takes the column it mirrors from the same tile (every such
// column lies in the tile: i0 < n_r), a ghost row's H_Z gets the rule of its boundary.
template <typename S, typename R, bool H1>
__device__ __forceinline__ void stage_from_raw(const AdvArgs<S> &a, const View &v, const S *raw, R *A, S *Hh,
                                               int slot, int lc, int col, int row, int k, int lane, R jeps, int i0) {
    int sc = lc;
    int rule = 0;   // H_r: 1 negate, 2 keep the inward (<= 0) part, 3 keep the outward (>= 0) part
    if (col < 0) {
        if (v.bcl == 0) { sc = (-1 - col) - i0 + 2; rule = 1; }
        else { sc = -i0 + 2; rule = 2; }
    } else if (col >= v.nr) {
        if (v.bcr == 0) { sc = (2 * v.nr - 1 - col) - i0 + 2; rule = 1; }
        else { sc = (v.nr - 1) - i0 + 2; rule = 3; }
    }
    Cell<S> c;
    c.J = raw[(0 * MCOL + sc) * 32 + lane];
    c.Hr = raw[(1 * MCOL + sc) * 32 + lane];
    c.HZ = raw[(2 * MCOL + sc) * 32 + lane];
    if (rule == 1) c.Hr = -c.Hr;
    else if (rule == 2) c.Hr = c.Hr < S(0) ? c.Hr : S(0);
    else if (rule == 3) c.Hr = c.Hr > S(0) ? c.Hr : S(0);
    if (row >= v.nz) {
        if (v.bzt == 0) c.HZ = -c.HZ;
        else c.HZ = c.HZ > S(0) ? c.HZ : S(0);
    }
    R aF = R(0);
    if (nf<R>() == 4) {
        int cc = col < 0 ? 0 : (col >= v.nr ? v.nr - 1 : col);
        int rr = row >= v.nz ? v.nz - 1 : row;
        aF = alpha_F<S, R>(a, v, cc, rr, k);
    }
    CellF<R> f = cell_f<R>(R(c.J), R(c.Hr), R(c.HZ), jeps);
    R *p = a_cell<R, H1>(A, slot, lc) + lane;
    p[0] = f.J; p[32] = f.fr; p[64] = f.fZ;
    if (nf<R>() == 4) p[96] = aF;
    if (lc >= 2 && lc < 2 + MT) {
        constexpr int HF = sizeof(S) == sizeof(R) ? 2 : 3;
        S *q = Hh + ((hslot(row) * MT + (lc - 2)) * HF) * 32 + lane;
        q[0] = c.Hr; q[32] = c.HZ;
        if (HF == 3) q[64] = c.J;
    }
}

// A staged cell; with FP32 arithmetic also its alpha_F from the ring.
template <typename R, bool H1>
__device__ __forceinline__ CellF<R> staged(const R *A, int slot, int lc, int lane, R &aF) {
    const R *p = a_cell<R, H1>(const_cast<R *>(A), slot, lc) + lane;
    CellF<R> c;
    c.J = p[0]; c.fr = p[32]; c.fZ = p[64];
    if (nf<R>() == 4) aF = p[96];
    return c;
}

// With FP32 arithmetic the faces read u* (`up`) and the Z face's PLM intervals (`ivz`) where the
// caller points, the warp's row slot in shared memory (see GEO_N below); with FP64 arithmetic
// they load them from global memory where they are used and ignore the two pointers.
// r face f (between cells f-1 and f) of row j held in ring slot `slot`; wl = f - i0 is the
// staged column of the stencil's first cell (src/AdvectJandH.jl:641-968).
template <typename S, typename R, int FLUX, bool H1>
__device__ __forceinline__ void face_r_staged(const AdvArgs<S> &a, const View &v, const R *A, int slot, int wl,
                                              int f, int j, int k, int lane, R jeps, const double *up,
                                              const double *riv, R *F, R &kL, R &kR) {
    const double us = *up;
    R d0, aFi, aFp, d3;
    CellF<R> cm1 = staged<R, H1>(A, slot, wl, lane, d0);
    CellF<R> ci = staged<R, H1>(A, slot, wl + 1, lane, aFi);
    CellF<R> cp1 = staged<R, H1>(A, slot, wl + 2, lane, aFp);
    CellF<R> cp2 = staged<R, H1>(A, slot, wl + 3, lane, d3);
    R iv[5];
#pragma unroll
    for (int t = 0; t < 5; t++) iv[t] = R(riv[t]);
    Recon<R> q = reconstruct_f<R>(cm1, ci, cp1, cp2, iv, aFi, aFp, jeps);
    R DrrL, DZZL, DrZL, DrrR, DZZR, DrZR;
    D_from_f_n<R>(q.f_L, q.nr_L, q.nZ_L, DrrL, DZZL, DrZL);
    D_from_f_n<R>(q.f_R, q.nr_R, q.nZ_R, DrrR, DZZR, DrZR);
    R FJ, FHr, FHZ;
    m1_flux<R, FLUX, false>(q.Hr_L, q.Hr_R, DrrL * q.J_L, DrrR * q.J_R, DrZL * q.J_L, DrZR * q.J_R, q, ci.J, cp1.J,
                            FJ, FHr, FHZ);
    R uc = R(us * kInvC);
    F[0] = FJ + adv_flux(uc, q.J_L, q.J_R);
    F[1] = FHr + adv_flux(uc, q.Hr_L, q.Hr_R);
    F[2] = FHZ + adv_flux(uc, q.HZ_L, q.HZ_R);
    kL = clamp01(R(1) - DrrL - DZZL) * q.J_L;
    kR = (f == 0) ? k_phiphi_axis<R>(q.J_R, q.HZ_R, jeps) : clamp01(R(1) - DrrR - DZZR) * q.J_R;
}

// Z face f (between rows f-1 and f) of column i, staged column lc (src/AdvectJandH.jl:978-1289).
template <typename S, typename R, int FLUX, bool H1>
__device__ __forceinline__ void face_z_staged(const AdvArgs<S> &a, const View &v, const R *A, int lc, int i, int f,
                                              int k, int lane, R jeps, const double *ivz, const double *up, R *F) {
    const double us = *up;
    R d0, aFi, aFp, d3;
    CellF<R> cm1 = staged<R, H1>(A, (f + 2) & (RING - 1), lc, lane, d0);     // row f-2
    CellF<R> ci = staged<R, H1>(A, (f + 3) & (RING - 1), lc, lane, aFi);     // row f-1
    CellF<R> cp1 = staged<R, H1>(A, f & (RING - 1), lc, lane, aFp);          // row f
    CellF<R> cp2 = staged<R, H1>(A, (f + 1) & (RING - 1), lc, lane, d3);     // row f+1
    R iv[5];
#pragma unroll
    for (int t = 0; t < 5; t++) iv[t] = R(ivz[t]);
    Recon<R> q = reconstruct_f<R>(cm1, ci, cp1, cp2, iv, aFi, aFp, jeps);
    R DrrL, DZZL, DrZL, DrrR, DZZR, DrZR;
    D_from_f_n<R>(q.f_L, q.nr_L, q.nZ_L, DrrL, DZZL, DrZL);
    D_from_f_n<R>(q.f_R, q.nr_R, q.nZ_R, DrrR, DZZR, DrZR);
    R FJ, FHr, FHZ;
    m1_flux<R, FLUX, true>(q.HZ_L, q.HZ_R, DrZL * q.J_L, DrZR * q.J_R, DZZL * q.J_L, DZZR * q.J_R, q, ci.J, cp1.J,
                           FJ, FHr, FHZ);
    R uc = R(us * kInvC);
    F[0] = FJ + adv_flux(uc, q.J_L, q.J_R);
    F[1] = FHr + adv_flux(uc, q.Hr_L, q.Hr_R);
    F[2] = FHZ + adv_flux(uc, q.HZ_L, q.HZ_R);
}

// The per-row scalars a warp needs: the cell's geometry and velocity gradients (0..10), u*_r of
// the warp's r face (11), u*_Z of its Z face above the row (12), that face's PLM intervals
// (13..17). They are copied one per lane a row ahead of their use (cp.async into the other half
// of a per-warp double buffer in shared memory, so no register carries them across the row),
// and their loads overlap a whole row's work instead of stalling the faces and the cell update.
// The r faces' PLM intervals depend on the column only: the tile stages its MT + 1 faces' once.
constexpr int GEO_N = 18;
enum { G_ARL, G_ARR, G_AZL, G_AZR, G_IDV, G_DURDR, G_DURDZ, G_DUZDR, G_DUZDZ, G_UROR, G_IRC, G_UR, G_UZ, G_ZIV };

// Where lane `lane` finds its scalar of row j for warp column `col` (the r face of warp w is
// face col too): src + j * stride, or nowhere (src null). Each lane gets one address, so a row's
// scalars come in with one load instruction per warp. The ranges are those of the consumers:
// the cell update and the Z face run for own columns col < n_r, the r face for faces col <= n_r.
template <typename S>
__device__ __forceinline__ void geo_source(const AdvArgs<S> &a, const View &v, int lane, int col, bool own,
                                           const double *&src, int &stride) {
    src = nullptr;
    stride = 0;
    if (lane == G_UR) {
        if (col <= v.nr) { src = a.u_r_star + v.orf + col; stride = v.nr + 1; }
        return;
    }
    if (!own || col >= v.nr || lane >= GEO_N) return;
    const long long c = v.oc + col;
    stride = v.nr;
    switch (lane) {
        case G_ARL: src = a.A_r + v.orf + col; stride = v.nr + 1; break;
        case G_ARR: src = a.A_r + v.orf + col + 1; stride = v.nr + 1; break;
        case G_AZL: src = a.A_Z + v.ozf + col; break;
        case G_AZR: src = a.A_Z + v.ozf + col + v.nr; break;
        case G_IDV: src = a.inv_dV + c; break;
        case G_DURDR: src = a.dur_dr + c; break;
        case G_DURDZ: src = a.dur_dZ + c; break;
        case G_DUZDR: src = a.duZ_dr + c; break;
        case G_DUZDZ: src = a.duZ_dZ + c; break;
        case G_UROR: src = a.ur_over_r + c; break;
        case G_IRC: src = a.inv_r_cell + v.ocol + col; stride = 0; break;
        case G_UZ: src = a.u_Z_star + v.ozf + col + v.nr; break;                 // face j+1
        default: src = a.zint + v.ozint + 5 + (lane - G_ZIV); stride = 5; break;   // face j+1
    }
}

// Row j's scalar of this lane; rows at or beyond the tile's end j1 (<= n_z) fetch nothing.
__device__ __forceinline__ double geo_fetch(const double *src, int stride, int j, int j1) {
    return (src != nullptr && j < j1) ? __ldg(src + (long long)stride * j) : 0.0;
}

// Shared memory of the advection tile before the bulk-copy staging area, in bytes.
// PFR: every staged input copied a row ahead by per-lane cp.async into raw slots (the own
// column's row j+3 and warp 8's halo cells of row j+1, while row j's faces and update run),
// with the one-row halo ring of a_cell paying for the slots: FP64 arithmetic with per-lane
// staging, 76 KB per CTA, three CTAs per SM. FP64 advection 0.288 -> 0.282 ms at 256^2 x 64,
// 1.219 -> 1.169 ms at 512^2 x 128, 4.82 -> 4.64 ms at 1024^2 x 128; bit for bit unchanged.
template <typename R, bool TMA> __host__ __device__ constexpr bool adv_pfr() { return !TMA && sizeof(R) == 8; }

// Shared memory of the advection tile before the bulk-copy staging area, in bytes (with PFR
// the one-row halo ring and the raw slots).
template <typename S, typename R, bool PFR>
__host__ __device__ constexpr size_t adv_smem_base() {
    return sizeof(R) * 32 * (a_cells<R, PFR>() * nf<R>() + (MT + 1) * 5) +
           sizeof(S) * 32 * HRING * MT * (sizeof(S) == sizeof(R) ? 2 : 3) +
           sizeof(double) * (MWARPS * 2 * GEO_N + (MT + 1) * 5) +
           (PFR ? sizeof(double) * (MT + 4) * RAW_SLOT : 0);
}
__host__ __device__ constexpr size_t adv_tma_off(size_t base) { return (base + 127) / 128 * 128; }

// TMA: rows j0+2 .. of the tile arrive as bulk tensor copies (one 32-bin x MCOL-column box per
// field, issued by one thread a row ahead of their use into one raw tile, completed on an
// mbarrier) instead of per-lane loads; the converting warps apply the ghost-cell rules. The
// first rows (j0-2 .. j0+1) are staged by per-lane loads while the first copy is in flight.
// One tile of the advection (tile `tile` of the work list) by the calling CTA of MTHREADS
// threads, in dynamic shared memory `adv_smem`: the body of k_advect, also run by the persistent
// batch kernel.
template <typename S, typename R, int FLUX, bool TMA>
__device__ __forceinline__ void advect_tile(const AdvArgs<S> &a, int tile, unsigned char *adv_smem) {
    constexpr int HF = sizeof(S) == sizeof(R) ? 2 : 3;
    constexpr int NF = nf<R>();
    constexpr bool PFR = adv_pfr<R, TMA>();
    R *A = reinterpret_cast<R *>(adv_smem);                            // a_cells cells of [NF][32] (a_cell)
    S *Hh = reinterpret_cast<S *>(A + a_cells<R, PFR>() * NF * 32);    // [HRING][MT][HF][32]
    R *Fr = reinterpret_cast<R *>(Hh + HRING * MT * HF * 32);           // [MT+1][5][32]
    double *geo = reinterpret_cast<double *>(Fr + (MT + 1) * 5 * 32);  // [MWARPS][2][GEO_N]: the row slots
    double *riv = geo + MWARPS * 2 * GEO_N;                             // [MT+1][5]: the r faces' intervals
    double *rawp = riv + (MT + 1) * 5;                                  // PFR: [MT + 4][RAW_SLOT] raw slots
    constexpr size_t toff = adv_tma_off(adv_smem_base<S, R, false>());
    S *raw = reinterpret_cast<S *>(adv_smem + toff);                                   // [3][MCOL][32]
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(adv_smem + toff + raw_tile_bytes<S>());
    int *abort_flag = reinterpret_cast<int *>(bar + 1);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int4 t = a.tiles[tile];
    View v;
    load_view(a.cl[t.x], v);
    const int i0 = t.y, j0 = t.z, kb = t.w;
    const int j1 = (j0 + a.rows < v.jend) ? j0 + a.rows : v.jend;
    // the last row a tile stages: the Z face j1 - 1/2 reads rows up to j1 + 1 (ghosts beyond n_z + 1 unused)
    const int rlast = (j1 + 1 < v.nz + 1) ? j1 + 1 : v.nz + 1;
    // one bulk copy per field of row r (a ghost row fetches the row it mirrors)
    auto issue_row = [&](int r) {
        const int src = r < v.nz ? r : (v.bzt == 0 ? 2 * v.nz - 1 - r : v.nz - 1);
        const unsigned char *maps = a.tmaps + (size_t)t.x * 3 * kTensorMapBytes;
        fence_proxy_async_smem();
        mbar_expect_tx(bar, (unsigned)raw_tile_bytes<S>());
#pragma unroll
        for (int f = 0; f < 3; f++) tma_load_3d(raw + f * MCOL * 32, maps + f * kTensorMapBytes, kb, i0 - 2, src, bar);
    };
    const int k = kb + lane;
    const int kmin = a.kwin[2 * t.x], kmax = a.kwin[2 * t.x + 1];
    const bool kact = (k >= kmin) && (k <= kmax) && (k < a.nnu);
    const bool chunk_act = (kb <= kmax) && (kb + 31 >= kmin);
    const R jeps = R(a.jeps);
    const int col = i0 + w;                      // own column (warps 0..7)
    const bool own = (w < MT);

    if (!chunk_act) {
        if (own && col < v.nr && k < a.nnu) {
            for (int j = j0; j < j1; j++) {
                long long x = v.o3 + (long long)k + (long long)a.nnu * ((long long)col + (long long)v.nr * j);
                a.Jo[x] = a.J[x]; a.Hro[x] = a.Hr[x]; a.HZo[x] = a.HZ[x];
            }
        }
        return;
    }

    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            *abort_flag = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0 && j0 + 2 <= rlast) issue_row(j0 + 2);
    }
    // PFR: the first row-ahead copies (the own column's row j0+2, warp 8's halo cells of row j0)
    // go out before the prologue's own loads and are waited for at its end
    S *rawo = reinterpret_cast<S *>(rawp + w * RAW_SLOT);   // own warps; halo cell q: slot MT + q
    const int hl[4] = {0, 1, MT + 2, MT + 3};
    if constexpr (PFR) {
        if (own) {
            const int r = j0 + 2;
            if (r <= j1 + 1 && col <= v.nr + 1 && r <= v.nz + 1 && !(col >= v.nr && r >= v.nz))
                raw_issue<S>(a, v, rawo, col, r, k, lane, kact);
        } else if (j0 < j1) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int c2 = i0 - 2 + hl[q];
                if (c2 <= v.nr + 1) raw_issue<S>(a, v, reinterpret_cast<S *>(rawp + (MT + q) * RAW_SLOT), c2, j0, k, lane, kact);
            }
        }
        cp_async_commit();
    }
    // prologue: own columns, rows j0-2 .. j0+1
    if (own && kact && col <= v.nr + 1) {
        for (int r = j0 - 2; r <= j0 + 1; r++) {
            bool gcol = col >= v.nr, grow = (r < 0 || r >= v.nz);
            if (r < -2 || r > v.nz + 1 || (gcol && grow)) continue;
            stage_cell<S, R, PFR>(a, v, A, Hh, r & (RING - 1), w + 2, col, r, k, lane, jeps);
        }
    }
    if constexpr (TMA) {
        // with bulk copies the halo columns of a row come with its copy, two rows before the
        // r faces read them: the prologue stages those of rows j0 and j0+1
        if (!own && kact) {
            for (int r = j0; r <= j0 + 1 && r < j1 && r < v.nz; r++) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    int c2 = i0 - 2 + hl[q];
                    if (c2 <= v.nr + 1) stage_cell<S, R, PFR>(a, v, A, Hh, r & (RING - 1), hl[q], c2, r, k, lane, jeps);
                }
            }
        }
    }
    // per-row scalars: row j0 now, every next row a row ahead (the buffer of row j is
    // g0 + ((j - j0) & 1) * GEO_N)
    const double *gsrc = nullptr;
    int gstr = 0;
    double *g0 = geo + w * 2 * GEO_N;
    geo_source<S>(a, v, lane, col, own, gsrc, gstr);
    if (lane < GEO_N) g0[lane] = geo_fetch(gsrc, gstr, j0, j1);
    for (int t = threadIdx.x; t < (MT + 1) * 5; t += blockDim.x) {
        const int f = i0 + t / 5;
        riv[t] = f <= v.nr ? __ldg(a.rint + v.orint + 5 * f + t % 5) : 0.0;
    }
    if constexpr (PFR) cp_async_wait<0>();
    __syncthreads();
    R zL[3] = {R(0), R(0), R(0)};
    if (own && kact && col < v.nr)
        face_z_staged<S, R, FLUX, PFR>(a, v, A, w + 2, col, j0, k, lane, jeps, a.zint + v.ozint + 5 * j0,
                                  a.u_Z_star + v.ozf + col + (long long)v.nr * j0, zL);   // face j0

    const double ctdt = v.ctdt;
    const double ctdt_c = ctdt * kInvC;
    // FP32 arithmetic (56 registers at 4 CTAs per SM) holds the next row's scalar in a register
    // and keeps one buffer; FP64 arithmetic, at its register limit, copies it with cp.async into
    // the other buffer (mixed advection 0.183 ms with the register, 0.189 ms with the copy;
    // FP64 advection 0.333 -> 0.320 ms with the copy, at 256^2 x 64)
    constexpr bool GREG = sizeof(R) == 4;
    for (int j = j0; j < j1; j++) {
        double *g = GREG ? g0 : g0 + ((j - j0) & 1) * GEO_N;
        double gnext = 0.0;
        if constexpr (GREG) {
            gnext = geo_fetch(gsrc, gstr, j + 1, j1);
        } else {
            if (lane < GEO_N) {
                double *gn = g0 + ((j + 1 - j0) & 1) * GEO_N;
                if (gsrc != nullptr && j + 1 < j1) cp_async_el(gn + lane, gsrc + (long long)gstr * (j + 1));
                else gn[lane] = 0.0;
            }
            cp_async_commit();
        }
        if constexpr (TMA) {
            // (A) row j+2 from its bulk copy: the own column, and (warp 8) the halo columns
            const int r = j + 2;
            if (r <= rlast) {
                if (!mbar_wait_bounded(bar, (unsigned)((r - (j0 + 2)) & 1))) {
                    *abort_flag = 1;
                    atomicOr(a.err, ERRB_TIMEOUT);
                } else if (kact) {
                    const bool grow = r >= v.nz;
                    if (own) {
                        if (col <= v.nr + 1 && !(col >= v.nr && grow))
                            stage_from_raw<S, R, PFR>(a, v, raw, A, Hh, r & (RING - 1), w + 2, col, r, k, lane, jeps, i0);
                    } else if (!grow && r < j1) {
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            int c2 = i0 - 2 + hl[q];
                            if (c2 <= v.nr + 1)
                                stage_from_raw<S, R, PFR>(a, v, raw, A, Hh, r & (RING - 1), hl[q], c2, r, k, lane, jeps, i0);
                        }
                    }
                }
            }
            __syncthreads();
            if (*reinterpret_cast<volatile int *>(abort_flag)) {
                // a copy never arrived: wait once more (bounded) for it, then leave the tile
                if (threadIdx.x == 0) mbar_wait_bounded(bar, (unsigned)((r - (j0 + 2)) & 1));
                return;
            }
            // the raw tile is free again: fetch row j+3 while this row's faces and update run
            if (threadIdx.x == 0 && j + 3 <= rlast) issue_row(j + 3);
        } else if constexpr (PFR) {
            // (A) from the raw slots: the own column's row j+2 and warp 8's halo cells of row j,
            // copied a row ago; then the copies of the next ones go out and land while this
            // row's faces and update run (the wait at the end of the row)
            if (own) {
                const int r = j + 2;
                if (kact && col <= v.nr + 1 && r <= v.nz + 1 && !(col >= v.nr && r >= v.nz))
                    stage_raw<S, R, PFR>(a, v, rawo, A, Hh, r & (RING - 1), w + 2, col, r, lane, jeps);
                __syncwarp();
                const int rn = r + 1;
                if (rn <= j1 + 1 && col <= v.nr + 1 && rn <= v.nz + 1 && !(col >= v.nr && rn >= v.nz))
                    raw_issue<S>(a, v, rawo, col, rn, k, lane, kact);
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int c2 = i0 - 2 + hl[q];
                    if (kact && c2 <= v.nr + 1)
                        stage_raw<S, R, PFR>(a, v, reinterpret_cast<const S *>(rawp + (MT + q) * RAW_SLOT), A, Hh,
                                             j & (RING - 1), hl[q], c2, j, lane, jeps);
                }
                __syncwarp();
                if (j + 1 < j1) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int c2 = i0 - 2 + hl[q];
                        if (c2 <= v.nr + 1)
                            raw_issue<S>(a, v, reinterpret_cast<S *>(rawp + (MT + q) * RAW_SLOT), c2, j + 1, k, lane, kact);
                    }
                }
            }
            cp_async_commit();
            __syncthreads();
        } else {
            // (A) stage row j+2 of the own column; warp 8 stages the halo columns of row j (spread
            // over four warps instead, one halo cell each, the FP64 advection took 0.336 ms
            // against 0.322 ms at 256^2 x 64, before the row-ahead copies)
            if (kact) {
                if (own) {
                    int r = j + 2;
                    bool gcol = col >= v.nr, grow = r >= v.nz;
                    if (col <= v.nr + 1 && r <= v.nz + 1 && !(gcol && grow))
                        stage_cell<S, R, PFR>(a, v, A, Hh, r & (RING - 1), w + 2, col, r, k, lane, jeps);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        int c2 = i0 - 2 + hl[q];
                        if (c2 <= v.nr + 1)
                            stage_cell<S, R, PFR>(a, v, A, Hh, j & (RING - 1), hl[q], c2, j, k, lane, jeps);
                    }
                }
            }
            __syncthreads();
        }
        // (B) the r face left of the own column (warp 8: the tile's right face), the Z face j+1/2
        const int f = i0 + w;
        R zR[3] = {R(0), R(0), R(0)};
        if (kact && f <= v.nr) {
            R F[3], kL, kR;
            face_r_staged<S, R, FLUX, PFR>(a, v, A, j & (RING - 1), w, f, j, k, lane, jeps, g + G_UR, riv + 5 * w, F,
                                      kL, kR);
            R *p = Fr + (w * 5) * 32 + lane;
            p[0] = F[0]; p[32] = F[1]; p[64] = F[2]; p[96] = kL; p[128] = kR;
        }
        if (own && kact && col < v.nr)
            face_z_staged<S, R, FLUX, PFR>(a, v, A, w + 2, col, j + 1, k, lane, jeps, g + G_ZIV, g + G_UZ, zR);
        __syncthreads();
        // (C) cell update, src/AdvectJandH.jl:1302-1382
        if (own && col < v.nr && k < a.nnu) {
            const int i = col;
            long long cl = (long long)i + (long long)v.nr * j;
            long long x = v.o3 + (long long)k + (long long)a.nnu * cl;
            if (!kact) {
                a.Jo[x] = a.J[x]; a.Hro[x] = a.Hr[x]; a.HZo[x] = a.HZ[x];
            } else {
                const S *pH = Hh + ((hslot(j) * MT + w) * HF) * 32 + lane;
                const S uHr = pH[0], uHZ = pH[32];
                const S uJ = HF == 3 ? pH[64] : S(a_cell<R, PFR>(A, j & (RING - 1), w + 2)[lane]);
                const R sJ = R(uJ), sHr = R(uHr), sHZ = R(uHZ);
                R Drr, DZZ, DrZ;
                D_edd<R>(sHr, sHZ, sJ, jeps, R(a.heps2), Drr, DZZ, DrZ);
                const R *FL = Fr + (w * 5) * 32 + lane;
                const R *FR = FL + 5 * 32;
                const double ArL = g[G_ARL], ArR = g[G_ARR], AZL = g[G_AZL], AZR = g[G_AZR];
                const double fac = ctdt * g[G_IDV];
                // increments in R, accumulated into the state in S
                S Jn, Hrn, HZn;
                const S ujeps = S(a.jeps);
                if (sizeof(R) == 8) {
                    R fr_ = R(fac);
                    Jn = uJ - S(fr_ * ((R(ArR) * FR[0] - R(ArL) * FL[0]) + (R(AZR) * zR[0] - R(AZL) * zL[0])));
                    HZn = uHZ - S(fr_ * ((R(ArR) * FR[64] - R(ArL) * FL[64]) + (R(AZR) * zR[2] - R(AZL) * zL[2])));
                    Hrn = uHr - S(fr_ * ((R(ArR) * FR[32] - R(ArL) * FL[32]) + (R(AZR) * zR[1] - R(AZL) * zL[1])));
                } else {
                    R wrL = R(fac * ArL), wrR = R(fac * ArR), wzL = R(fac * AZL), wzR = R(fac * AZR);
                    Jn = uJ - S((wrR * FR[0] - wrL * FL[0]) + (wzR * zR[0] - wzL * zL[0]));
                    HZn = uHZ - S((wrR * FR[64] - wrL * FL[64]) + (wzR * zR[2] - wzL * zL[2]));
                    Hrn = uHr - S((wrR * FR[32] - wrL * FL[32]) + (wzR * zR[1] - wzL * zL[1]));
                }
                const S Jn0 = Jn;
                Jn = Jn > ujeps ? Jn : ujeps;
                const R ga = R(g[G_DURDR]), gb = R(g[G_DURDZ]), gc = R(g[G_DUZDR]), gd = R(g[G_DUZDZ]);
                const R ge = R(g[G_UROR]);
                R DdU = d_colon_grad_u<R>(Drr, DrZ, DZZ, ga, gb, gc, gd, ge);
                R Kav = R(0.5) * (FL[128] + FR[96]);
                if (sizeof(R) == 8)
                    Hrn += S(R(ctdt) * Kav * R(g[G_IRC]));
                else
                    Hrn += S(R(ctdt * g[G_IRC]) * Kav);
                R cc = R(ctdt_c);
                R dHr = -cc * (sHr * ga + sHZ * gb);
                R dHZ = -cc * (sHr * gc + sHZ * gd);
                Hrn = Hrn + S(dHr);
                HZn = HZn + S(dHZ);
                Jn = Jn - S(cc * DdU * sJ);
                if (a.tape) {
                    // the values before the floors and the causality limiter, for the adjoint
                    a.tape[x] = double(Jn0);
                    a.tape[x + a.tape_stride] = double(Jn);
                    a.tape[x + 2 * a.tape_stride] = double(Hrn);
                    a.tape[x + 3 * a.tape_stride] = double(HZn);
                }
                Jn = Jn > ujeps ? Jn : ujeps;
                S H2 = Hrn * Hrn + HZn * HZn;
                if (H2 > Jn * Jn) {
                    S fsc;
                    if constexpr (sizeof(S) == 4) {
                        // a flushed (zero) root of a subnormal |H|^2 scales H to zero
                        const S Hm = rsq(H2);
                        fsc = Hm > S(0) ? Jn / Hm : S(0);
                    } else {
                        // |H|^2 > J^2 >= jeps^2, far inside the normal range
                        fsc = Jn * rsqrt_nr(H2);
                    }
                    Hrn *= fsc;
                    HZn *= fsc;
                }
                a.Jo[x] = S(Jn);
                a.Hro[x] = S(Hrn);
                a.HZo[x] = S(HZn);
            }
        }
        zL[0] = zR[0]; zL[1] = zR[1]; zL[2] = zR[2];
        if constexpr (GREG) {
            // the next row's scalars replace this row's once every lane of the warp has read them
            __syncwarp();
            if (lane < GEO_N) g[lane] = gnext;
        } else {
            // the next row's scalars have landed (each lane waits for its own copy; the warp
            // barrier shows them to the other lanes and keeps this row's buffer until every lane
            // has read it)
            cp_async_wait<0>();
        }
        __syncwarp();
    }
}

template <typename S, typename R, int FLUX, int MINB, bool TMA>
__global__ void __launch_bounds__(MTHREADS, MINB) k_advect(AdvArgs<S> a) {
    extern __shared__ __align__(128) unsigned char adv_smem[];
    advect_tile<S, R, FLUX, TMA>(a, blockIdx.x, adv_smem);
}

// ------------------------------------------------------------------------------------------
// Frequency kernel helpers
// ------------------------------------------------------------------------------------------
template <int M>
struct Row {
    double a[M], b[M], c[M], d[M];
};

// Fetch, for every owned row r = lane*M + m, the quantity v of row r - s (dir = -1) or r + s
// (dir = +1). Rows outside [0, 32M) read the identity-row value `idv`.
template <int M>
__device__ __forceinline__ void nbr(const double (&v)[M], double (&out)[M], int s, int dir, int lane, double idv) {
    if (s < M) {
#pragma unroll
        for (int m = 0; m < M; m++) {
            int mm = m + dir * s;
            if (mm >= 0 && mm < M) {
                out[m] = v[mm];
            } else {
                int src = mm < 0 ? mm + M : mm - M;
                double w = 0.0;
#pragma unroll
                for (int q = 0; q < M; q++)
                    if (q == src) w = v[q];
                double got = dir < 0 ? __shfl_up_sync(0xffffffffu, w, 1) : __shfl_down_sync(0xffffffffu, w, 1);
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

// Parallel cyclic reduction of the 32*M-row tridiagonal system held by the warp
// (row r = lane*M + m; a = sub-, b = main-, c = super-diagonal, d = right-hand side).
// Decoupled rows are identity rows. Returns x in d.
template <int M>
__device__ __forceinline__ void pcr_solve(Row<M> &R_, int lane) {
#pragma unroll
    for (int s = 1; s < 32 * M; s <<= 1) {
        double ib[M];
#pragma unroll
        for (int m = 0; m < M; m++) ib[m] = rcp<double>(R_.b[m]);
        double am[M], cm[M], dm[M], ibm[M], ap[M], cp[M], dp[M], ibp[M];
        nbr<M>(R_.a, am, s, -1, lane, 0.0);
        nbr<M>(R_.c, cm, s, -1, lane, 0.0);
        nbr<M>(R_.d, dm, s, -1, lane, 0.0);
        nbr<M>(ib, ibm, s, -1, lane, 1.0);
        nbr<M>(R_.a, ap, s, +1, lane, 0.0);
        nbr<M>(R_.c, cp, s, +1, lane, 0.0);
        nbr<M>(R_.d, dp, s, +1, lane, 0.0);
        nbr<M>(ib, ibp, s, +1, lane, 1.0);
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

// Lane-serial elimination of the same system: the warp writes its rows to shared memory and
// lane 0 runs the forward elimination and back substitution of dgtsv's no-interchange branch
// (the Thomas algorithm), then the rows are read back. `sm` holds 4*32*M doubles per warp.
template <int M>
__device__ __forceinline__ void thomas_solve(Row<M> &R_, int lane, double *sm) {
    constexpr int N = 32 * M;
    double *a = sm, *b = sm + N, *c = sm + 2 * N, *d = sm + 3 * N;
#pragma unroll
    for (int m = 0; m < M; m++) {
        int r = lane * M + m;
        a[r] = R_.a[m]; b[r] = R_.b[m]; c[r] = R_.c[m]; d[r] = R_.d[m];
    }
    __syncwarp();
    if (lane == 0) {
        for (int r = 1; r < N; r++) {
            double fact = a[r] / b[r - 1];
            b[r] = b[r] - fact * c[r - 1];
            d[r] = d[r] - fact * d[r - 1];
        }
        d[N - 1] = d[N - 1] / b[N - 1];
        for (int r = N - 2; r >= 0; r--) d[r] = (d[r] - c[r] * d[r + 1]) / b[r];
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < M; m++) {
        int r = lane * M + m;
        R_.d[m] = d[r];
        R_.b[m] = b[r];
    }
    __syncwarp();
}

// Two rows per lane (rows 2l and 2l+1): one cyclic-reduction step eliminates the odd rows,
// leaving one row per lane, which parallel cyclic reduction across the warp solves in five
// levels; the odd rows then follow by back-substitution. Half the divisions and shuffles of
// PCR on all 64 rows, the same arithmetic per eliminated row. Returns x in d.
__device__ __forceinline__ void cr_pcr_solve2(Row<2> &R_, int lane) {
    // odd row o = 2l+1 of this lane; o- = 2l-1 is the previous lane's odd row
    const double ibo = rcp<double>(R_.b[1]);
    double a_om = __shfl_up_sync(0xffffffffu, R_.a[1], 1);
    double c_om = __shfl_up_sync(0xffffffffu, R_.c[1], 1);
    double d_om = __shfl_up_sync(0xffffffffu, R_.d[1], 1);
    double ib_om = __shfl_up_sync(0xffffffffu, ibo, 1);
    if (lane == 0) { a_om = 0.0; c_om = 0.0; d_om = 0.0; ib_om = 1.0; }
    // even row e = 2l: eliminate x_{e-1} (row o-) and x_{e+1} (row o)
    double al = -R_.a[0] * ib_om;
    double ga = -R_.c[0] * ibo;
    double ea = al * a_om;
    double eb = R_.b[0] + al * c_om + ga * R_.a[1];
    double ec = ga * R_.c[1];
    double ed = R_.d[0] + al * d_om + ga * R_.d[1];
    // PCR over the 32 even rows (one per lane), every row scaled to a unit diagonal so that a
    // level fetches three values from each neighbour instead of four (and no reciprocal pivot)
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
    // odd rows: x_o = (d_o - a_o x_e - c_o x_{e+2}) / b_o
    double xe2 = __shfl_down_sync(0xffffffffu, xe, 1);
    if (lane == 31) xe2 = 0.0;
    R_.d[0] = xe;
    R_.d[1] = (R_.d[1] - R_.a[1] * xe - R_.c[1] * xe2) * ibo;
    R_.b[0] = eb;                      // the pivots, for the zero-pivot check (b[1] is b_o)
}

// PCR over one row per lane (lane l holds row l of a 32-row system coupled to lanes l +- s),
// every row scaled to a unit diagonal so that a level fetches three values from each neighbour;
// returns the last level's diagonal (the pivot, before scaling) in eb and x in ed.
__device__ __forceinline__ void pcr_lanes(double &ea, double &eb, double &ec, double &ed, int lane) {
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
    ea = na;
    ec = nc;
    ed = nd;
}

// Four rows per lane (rows 4l .. 4l+3): two cyclic-reduction steps (the odd rows, then rows
// 4l+2) leave row 4l, solved by PCR across the warp; rows 4l+2, then the odd rows follow by
// back-substitution. Returns x in d; b holds the pivots for the zero-pivot check.
__device__ __forceinline__ void cr_pcr_solve4(Row<4> &R_, int lane) {
    const double ib1 = rcp<double>(R_.b[1]), ib3 = rcp<double>(R_.b[3]);
    double a3p = __shfl_up_sync(0xffffffffu, R_.a[3], 1), c3p = __shfl_up_sync(0xffffffffu, R_.c[3], 1);
    double d3p = __shfl_up_sync(0xffffffffu, R_.d[3], 1), ib3p = __shfl_up_sync(0xffffffffu, ib3, 1);
    if (lane == 0) { a3p = 0.0; c3p = 0.0; d3p = 0.0; ib3p = 1.0; }
    // level 1: rows 4l (eliminate 4l-1, 4l+1) and 4l+2 (eliminate 4l+1, 4l+3)
    double al = -R_.a[0] * ib3p, ga = -R_.c[0] * ib1;
    double a0 = al * a3p, b0 = R_.b[0] + al * c3p + ga * R_.a[1], c0 = ga * R_.c[1];
    double d0 = R_.d[0] + al * d3p + ga * R_.d[1];
    al = -R_.a[2] * ib1;
    ga = -R_.c[2] * ib3;
    double a2 = al * R_.a[1], b2 = R_.b[2] + al * R_.c[1] + ga * R_.a[3], c2 = ga * R_.c[3];
    double d2 = R_.d[2] + al * R_.d[1] + ga * R_.d[3];
    // level 2: row 4l eliminates 4l-2 (previous lane's row 2) and 4l+2
    const double ib2 = rcp<double>(b2);
    double a2p = __shfl_up_sync(0xffffffffu, a2, 1), c2p = __shfl_up_sync(0xffffffffu, c2, 1);
    double d2p = __shfl_up_sync(0xffffffffu, d2, 1), ib2p = __shfl_up_sync(0xffffffffu, ib2, 1);
    if (lane == 0) { a2p = 0.0; c2p = 0.0; d2p = 0.0; ib2p = 1.0; }
    al = -a0 * ib2p;
    ga = -c0 * ib2;
    double ea = al * a2p, eb = b0 + al * c2p + ga * a2, ec = ga * c2, ed = d0 + al * d2p + ga * d2;
    pcr_lanes(ea, eb, ec, ed, lane);
    const double x0 = ed;
    double x4 = __shfl_down_sync(0xffffffffu, x0, 1);
    if (lane == 31) x4 = 0.0;
    const double x2 = (d2 - a2 * x0 - c2 * x4) * ib2;
    R_.d[1] = (R_.d[1] - R_.a[1] * x0 - R_.c[1] * x2) * ib1;
    R_.d[3] = (R_.d[3] - R_.a[3] * x2 - R_.c[3] * x4) * ib3;
    R_.d[0] = x0;
    R_.d[2] = x2;
    R_.b[0] = eb;
    R_.b[2] = b2;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-k constants of UpdateFreqFactors! staged in shared memory once per CTA.
// KC_EXP2: the 32 entries of exp_tab's table.
enum { KC_NCK, KC_NCKP, KC_NCKM, KC_DNKP, KC_DNK, KC_DNKM, KC_IDNU, KC_ICK, KC_ICKP, KC_ICKM, KC_DNU, KC_EXP2, KC_N };

// Per-cell inputs staged in shared memory, 32 cells at a time per warp.
// CS_SUM_R / CS_SUM_Z receive each cell's sum over bins of dnu (H_old - H), which the warp's
// lanes turn into the cell's momentum, force and diagnostics once per 32 cells, one cell per lane.
enum { CS_ALPHA, CS_ALPHA_C, CS_PD, CS_JS, CS_PHI_INV, CS_ALPHA_CF, CS_T, CS_DUR_DR, CS_DUR_DZ, CS_DUZ_DR,
       CS_DUZ_DZ, CS_UR_OVER_R, CS_DV, CS_DRU_R, CS_DRU_Z, CS_SUM_R, CS_SUM_Z, CS_N };

// The next cell's bin rows (J, H_r, H_Z, H_voigt, J_old) are prefetched into a per-warp double
// buffer while the current cell computes, up to two bins per lane (four or more would leave
// shared memory for one CTA per SM).
template <int M> __host__ __device__ constexpr bool freq_prefetch() { return M <= 2; }

// Shared memory of the frequency kernel, in doubles: FP64 per-k constants, the per-warp
// reduction rows (without prefetch; with it, each warp's row lies in its own prefetch area,
// free once the warp's cells are done), per-warp staged cell inputs, the per-warp prefetch
// buffers (two slots of `ns` rows: 4, or 5 when J_old is not J's own buffer), and the
// lane-serial solver rows when that solver runs: 72 KB per CTA at two bins per lane with J_old
// aliased (86.5 KB before the overlay and the fourth row), which leaves L1 the difference. A
// third CTA per SM would fit, but its 80-register bound spills in the cell loop (FP64 at
// 256^2 x 64: 0.258 ms against 0.184 ms at two CTAs).
template <int M>
__host__ __device__ constexpr int freq_smem_off_cs(int nwarps) {
    return KC_N * 32 * M + (freq_prefetch<M>() ? 0 : nwarps * (32 * M + 8));
}
template <int M>
__host__ __device__ constexpr int freq_smem_off_pf(int nwarps) { return freq_smem_off_cs<M>(nwarps) + nwarps * CS_N * 32; }
template <int M>
__host__ __device__ constexpr int freq_pf_warp(int ns) { return 2 * ns * 32 * M; }   // doubles per warp
template <int M>
__host__ __device__ constexpr int freq_smem_off_tsm(int nwarps, int ns) {
    return freq_smem_off_pf<M>(nwarps) + (freq_prefetch<M>() ? nwarps * freq_pf_warp<M>(ns) : 0);
}
template <int M>
__host__ __device__ constexpr int freq_smem_doubles(int nwarps, bool thomas, int ns) {
    return freq_smem_off_tsm<M>(nwarps, ns) + (thomas ? nwarps * 4 * 32 * M : 0);
}
template <int M>
__host__ __device__ inline double *freq_red_row(double *fsm, int nwarps, int ns, int w) {
    return freq_prefetch<M>() ? fsm + freq_smem_off_pf<M>(nwarps) + w * freq_pf_warp<M>(ns)
                              : fsm + KC_N * 32 * M + w * (32 * M + 8);
}

// A lane's M contiguous bins of one row as whole 16-byte words, when the row layout allows it
// (k_freq's `vec` path): loads from shared memory and stores to global memory.
template <typename S, int M>
struct LaneRow {
    static constexpr bool ok = (M * sizeof(S)) % 16 == 0;
    static constexpr int words = (M * (int)sizeof(S)) / 16;
    __device__ __forceinline__ static void load(const S *src, S (&v)[M]) {
        if constexpr (ok) {
#pragma unroll
            for (int w = 0; w < words; w++) {
                const float4 t = reinterpret_cast<const float4 *>(src)[w];
                memcpy(&v[w * (16 / sizeof(S))], &t, 16);
            }
        }
    }
    __device__ __forceinline__ static void store(S *dst, const S (&v)[M]) {
        if constexpr (ok) {
#pragma unroll
            for (int w = 0; w < words; w++) {
                float4 t;
                memcpy(&t, &v[w * (16 / sizeof(S))], 16);
                reinterpret_cast<float4 *>(dst)[w] = t;
            }
        }
    }
};

// The cells [wbeg, wend) of a work item that warp `warp` of `nw` handles: one contiguous run
// per warp (k_freq and k_find_active sum their partials in this order).
__device__ __forceinline__ void warp_cell_run(int4 it, int warp, int nw, int &wbeg, int &wend) {
    const int per = (it.z - it.y + nw - 1) / nw;
    wbeg = it.y + warp * per;
    wend = min(it.z, wbeg + per);
}

// Up to four bins per lane the kernel is held to 2 CTAs per SM (128 registers). Four bins:
// ~230 B of spills, measured 1.4x faster than 1 CTA at 172 registers. Two bins: 1.8x faster
// than the 164 registers ptxas picks when only the block size bounds it.
// RC is the arithmetic of the cell-centre closure D(J, H) and of D:grad u that enter the Doppler
// term of the frequency factors: R in the FP64 and FP32-storage forms, FP32 in the mixed form.
// The closure only sets the velocity of the Peclet numbers; every factor is then formed in FP64
// from that one velocity, so its rounding moves the step like a velocity field off by 1e-7
// relative, not like the rounding of F against F+ + F- that the factors themselves cannot take
// (mixed frequency kernel at 256^2 x 64: 0.259 -> 0.246 ms; the mixed form's M_F after 2000
// steps 5.93e-7 -> 5.95e-7 from FP64).
//
// freq_item is one work item (`item` of `nitems`) by the calling CTA, whose first `nw` warps take
// its cells (the others only meet its barriers), in dynamic shared memory `fsm`: the body of
// k_freq, also run by the persistent batch kernel.
template <typename S, typename R, int M, typename RC>
__device__ __forceinline__ void freq_item(const FreqArgs<S> &a, int item, int nitems, double *fsm, int nw) {
    constexpr int NP = 32 * M;
    constexpr bool PF = freq_prefetch<M>();
    const bool jo_alias = a.Jold == a.Jin;
    const int ns = jo_alias ? 4 : 5;               // prefetched rows per cell
    double *kc = fsm;                                  // [KC_N][NP]
    double *tsm = fsm + freq_smem_off_tsm<M>(nw, ns);  // [nwarps][4][NP] (lane-serial solver)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nnu = a.nnu;
    for (int t = threadIdx.x; t < NP; t += blockDim.x) {
        bool in = (t >= 1 && t <= nnu - 2);
        kc[KC_NCK * NP + t] = in ? a.nuC[t] : 0.0;
        kc[KC_NCKP * NP + t] = in ? a.nuC[t + 1] : 0.0;
        kc[KC_NCKM * NP + t] = in ? a.nuC[t - 1] : 0.0;
        kc[KC_DNKP * NP + t] = in ? a.nuC[t + 1] - a.nu[t + 1] : 0.0;
        kc[KC_DNK * NP + t] = in ? a.nu[t + 1] - a.nuC[t] : 0.0;
        kc[KC_DNKM * NP + t] = in ? a.nu[t] - a.nuC[t - 1] : 0.0;
        kc[KC_IDNU * NP + t] = in ? a.inv_dnu[t] : 0.0;
        kc[KC_ICK * NP + t] = in ? a.inv_nuC[t] : 0.0;
        kc[KC_ICKP * NP + t] = in ? a.inv_nuC[t + 1] : 0.0;
        kc[KC_ICKM * NP + t] = in ? a.inv_nuC[t - 1] : 0.0;
        kc[KC_DNU * NP + t] = (t < nnu) ? a.dnu[t] : 0.0;
        kc[KC_EXP2 * NP + t] = (t < 32) ? kExp2Tab[t] : 0.0;
    }
    __syncthreads();

    const int4 it = a.items[item];
    const CloudDesc &cd = a.cl[it.x];
    const long long o3 = cd.o3, oc = cd.oc;
    const int nr = cd.nr, nz = cd.nz, bzb = cd.bc_z_bot;
    const double c_tilde = cd.c_tilde, dt = cd.dt, ctdt = cd.ctdt, z_center = cd.z_center;
    const double jeps = a.jeps;
    const double dw = 1.0 / ctdt;
    double acc_e[M];
#pragma unroll
    for (int m = 0; m < M; m++) acc_e[m] = 0.0;
    double acc_tot = 0.0, acc_mf = 0.0, acc_net = 0.0, acc_out = 0.0, acc_L = 0.0, acc_esc = 0.0;
    int bad = 0;

    int wbeg, wend;
    warp_cell_run(it, warp, nw, wbeg, wend);
    double *cs = fsm + freq_smem_off_cs<M>(nw) + warp * CS_N * 32;      // [CS_N][32]
    S *pf = reinterpret_cast<S *>(fsm + freq_smem_off_pf<M>(nw) + warp * freq_pf_warp<M>(ns));  // [2][ns][NP]
    const bool need_ff = a.do_freq && a.update_ff, need_js = a.do_emission || (a.parts & PART_DIAG);
    // With `vec`, every lane's M bins of a row are whole 16-byte words in global and shared
    // memory (row starts 16-byte aligned, n_nu a multiple of M): rows move as 16-byte copies,
    // loads and stores, bin m of lane l at l*M + m. Otherwise element by element, bin m of
    // lane l at m*32 + l.
    using LR = LaneRow<S, M>;
    const bool vec = LR::ok && a.vec16;
    // copies of cell cl's bin rows into prefetch buffer b
    auto issue = [&](int cl, int b) {
        const long long base = o3 + (long long)cl * nnu;
        S *d = pf + b * ns * NP;
        if constexpr (LR::ok) {
            if (vec) {
                if (lane * M < nnu) {
                    const long long g = base + lane * M;
                    const int q = lane * M;
                    constexpr int per = 16 / sizeof(S);
#pragma unroll
                    for (int w = 0; w < LR::words; w++) {
                        cp_async_16(d + q + w * per, a.Jin + g + w * per);
                        cp_async_16(d + NP + q + w * per, a.Hrin + g + w * per);
                        cp_async_16(d + 2 * NP + q + w * per, a.HZin + g + w * per);
                        cp_async_16(d + 3 * NP + q + w * per, a.Hv + g + w * per);
                        if (!jo_alias) cp_async_16(d + 4 * NP + q + w * per, a.Jold + g + w * per);
                    }
                }
                return;
            }
        }
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int k = lane * M + m, q = m * 32 + lane;
            if (k < nnu) {
                cp_async_el(d + q, a.Jin + base + k);
                cp_async_el(d + NP + q, a.Hrin + base + k);
                cp_async_el(d + 2 * NP + q, a.HZin + base + k);
                cp_async_el(d + 3 * NP + q, a.Hv + base + k);
                if (!jo_alias) cp_async_el(d + 4 * NP + q, a.Jold + base + k);
            }
        }
    };
    const double k4 = kFourPiOverC * (1.0 / c_tilde) * a.j_scale;
    const double inv_dt = 1.0 / dt;
    // the per-cell part of the epilogue for cells [gb, ge) of the run (ge - gb <= 32), one
    // cell per lane: the momentum Delta rho u, this step's force, and the M_F, L and radial
    // partials (Update_f_Lya_MF_L_Lya!, src/ConstantsAndFunctions.jl:588-674)
    auto flush = [&](int gb, int ge) {
        __syncwarp();
        const int cl = gb + lane;
        if (cl >= ge) return;
        const long long c = oc + cl;
        const double drs = cs[CS_SUM_R * 32 + lane], dzs = cs[CS_SUM_Z * 32 + lane];
        if (a.do_emission && a.dru_r) {
            a.dru_r[c] = cs[CS_DRU_R * 32 + lane] + k4 * drs;
            a.dru_Z[c] = cs[CS_DRU_Z * 32 + lane] + k4 * dzs;
        }
        if (a.parts & PART_DIAG) {
            const int i = cl % nr, j = cl / nr;
            const double dV = cs[CS_DV * 32 + lane];
            double fr = (k4 * drs) * inv_dt, fz = (k4 * dzs) * inv_dt;
            if (a.f_r) { a.f_r[c] = fr; a.f_Z[c] = fz; }
            acc_mf += dV * sqrt(fr * fr + fz * fz);
            acc_L += kFourPi * dV * cs[CS_JS * 32 + lane];
            double drr = __ldg(a.rCoM + cd.ocol + i), dzz = __ldg(a.ZCoM + cd.orow + j) - z_center;
            double dist = sqrt(drr * drr + dzz * dzz);
            double frad = 0.0;
            if (dist > 0.0) {
                double id = 1.0 / dist;
                frad = fr * (drr * id) + fz * (dzz * id);
            }
            acc_net += dV * frad;
            acc_out += dV * (frad > 0.0 ? frad : 0.0);
        }
    };
    if constexpr (PF) {
        if (wbeg < wend) issue(wbeg, 0);
        cp_async_commit();
    }
    int g0 = wbeg;
    for (int cl = wbeg; cl < wend; cl++) {
        const int i = cl % nr, j = cl / nr;
        const long long c = oc + cl;
        const long long base = o3 + (long long)cl * nnu;
        if (((cl - wbeg) & 31) == 0) {
            if (cl > wbeg) flush(g0, cl);
            // stage the per-cell inputs of the next 32 cells of the run (one coalesced load per
            // field instead of a dependent load per cell)
            g0 = cl;
            __syncwarp();
            const bool v = cl + lane < wend;
            const long long cc = c + lane;
            auto ld = [&](const double *p, bool need) { return (v && need && p) ? __ldg(p + cc) : 0.0; };
            cs[CS_ALPHA * 32 + lane] = ld(a.alpha, a.do_emission || need_ff);
            cs[CS_ALPHA_C * 32 + lane] = ld(a.alpha_c, a.do_emission);
            cs[CS_PD * 32 + lane] = ld(a.pd, a.do_emission);
            cs[CS_JS * 32 + lane] = ld(a.js, need_js);
            cs[CS_PHI_INV * 32 + lane] = ld(a.phi_inv, a.do_emission && !a.phi);
            cs[CS_ALPHA_CF * 32 + lane] = ld(a.alpha_cF, a.do_emission);
            cs[CS_T * 32 + lane] = ld(a.T, need_ff);
            cs[CS_DUR_DR * 32 + lane] = ld(a.dur_dr, need_ff);
            cs[CS_DUR_DZ * 32 + lane] = ld(a.dur_dZ, need_ff);
            cs[CS_DUZ_DR * 32 + lane] = ld(a.duZ_dr, need_ff);
            cs[CS_DUZ_DZ * 32 + lane] = ld(a.duZ_dZ, need_ff);
            cs[CS_UR_OVER_R * 32 + lane] = ld(a.ur_over_r, need_ff);
            cs[CS_DV * 32 + lane] = ld(a.dV, a.parts != 0);
            cs[CS_DRU_R * 32 + lane] = ld(a.dru_r, a.do_emission);
            cs[CS_DRU_Z * 32 + lane] = ld(a.dru_Z, a.do_emission);
            __syncwarp();
        }
        const double *cv = cs + (cl - g0);        // cv[f * 32]: field f of this cell
        S J[M], Hr[M], HZ[M];
        R Hv[M];
        double Jo[M];
        if constexpr (PF) {
            const int b = (cl - wbeg) & 1;
            if (cl + 1 < wend) issue(cl + 1, b ^ 1);
            cp_async_commit();
            cp_async_wait<1>();                   // this cell's copies (each lane reads its own)
            const S *d = pf + b * ns * NP;
            bool done = false;
            if constexpr (LR::ok) {
                if (vec) {
                    if (lane * M < nnu) {
                        const int q = lane * M;
                        S hv[M], jo[M];
                        LR::load(d + q, J);
                        LR::load(d + NP + q, Hr);
                        LR::load(d + 2 * NP + q, HZ);
                        LR::load(d + 3 * NP + q, hv);
                        LR::load(d + (jo_alias ? 0 : 4 * NP) + q, jo);
#pragma unroll
                        for (int m = 0; m < M; m++) { Hv[m] = R(hv[m]); Jo[m] = double(jo[m]); }
                    } else {
#pragma unroll
                        for (int m = 0; m < M; m++) { J[m] = Hr[m] = HZ[m] = S(0); Hv[m] = R(0); Jo[m] = 0.0; }
                    }
                    done = true;
                }
            }
            if (!done) {
#pragma unroll
                for (int m = 0; m < M; m++) {
                    const int k = lane * M + m, q = m * 32 + lane;
                    const bool vld = k < nnu;
                    J[m] = vld ? d[q] : S(0);
                    Hr[m] = vld ? d[NP + q] : S(0);
                    HZ[m] = vld ? d[2 * NP + q] : S(0);
                    Hv[m] = vld ? R(d[3 * NP + q]) : R(0);
                    Jo[m] = vld ? double(jo_alias ? d[q] : d[4 * NP + q]) : 0.0;
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                bool vld = k < nnu;
                J[m] = vld ? a.Jin[base + k] : S(0);
                Hr[m] = vld ? a.Hrin[base + k] : S(0);
                HZ[m] = vld ? a.HZin[base + k] : S(0);
                Hv[m] = vld ? R(__ldg(a.Hv + base + k)) : R(0);
                Jo[m] = vld ? double(a.Jold[base + k]) : 0.0;
            }
        }
        double dr_sum = 0.0, dz_sum = 0.0;
        // ---- LyaEmissionAbsorptionUpdate! (src/ConstantsAndFunctions.jl:526-567) ----
        if (a.do_emission) {
            const R al = R(cv[CS_ALPHA * 32]), acv = R(cv[CS_ALPHA_C * 32]);
            const R al_pd = al * R(cv[CS_PD * 32]);
            const R js_ct = R(cv[CS_JS * 32] * c_tilde / a.j_scale);
            const R ct = R(c_tilde), dtr = R(dt);
            const R pinv = a.phi ? R(0) : R(cv[CS_PHI_INV * 32]);
            const R acF = a.alpha_cF ? R(cv[CS_ALPHA_CF * 32]) : R(0);
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                if (k >= nnu) continue;
                R phi = a.phi ? R(__ldg(a.phi + base + k))
                              : ((k >= a.phi_kmin && k <= a.phi_kmax) ? Hv[m] * pinv : R(0));
                R aabs = acv + al_pd * Hv[m];
                R dJdt = js_ct * phi;
                R aH = a.aF ? R(__ldg(a.aF + base + k)) : (a.alpha_cF ? al * Hv[m] + acF : al * Hv[m]);
                double dn = kc[KC_DNU * NP + k];
                R Jn = (R(Jo[m]) + dJdt * dtr) * rcp<R>(R(1) + aabs * ct * dtr);
                R iden = rcp<R>(R(1) + aH * ct * dtr);
                R hr = R(Hr[m]) * iden;
                R hz = R(HZ[m]) * iden;
                dr_sum += dn * (double(Hr[m]) - double(hr));
                dz_sum += dn * (double(HZ[m]) - double(hz));
                Hr[m] = S(hr);
                HZ[m] = S(hz);
                J[m] = S(Jn);
                Jo[m] = double(J[m]);
            }
            dr_sum = warp_sum(dr_sum);
            dz_sum = warp_sum(dz_sum);
        }
        if (lane == 0) {     // turned into the cell's momentum and diagnostics by flush()
            cs[CS_SUM_R * 32 + (cl - g0)] = dr_sum;
            cs[CS_SUM_Z * 32 + (cl - g0)] = dz_sum;
        }
        // ---- FrequencyUpdateJLya_AllCells! (src/UpdateLyaJandH.jl:231-391) ----
        if (a.do_freq) {
            Row<M> sys;
            double Fp[M], F0[M], Fm[M];
            if (a.update_ff) {
                // UpdateFreqFactors!, src/FreqFactors.jl:181-275
                const double T = cv[CS_T * 32];
                const double dnuD = compute_dnuD(T);
                const double alv = cv[CS_ALPHA * 32];
                const double pref = 0.5 * (alv > a.alpha_floor ? alv : a.alpha_floor) * (dnuD * dnuD);
                const double rec0 = kHOverKB / T;
                const R ga = R(cv[CS_DUR_DR * 32]), gb = R(cv[CS_DUR_DZ * 32]), gc = R(cv[CS_DUZ_DR * 32]);
                const R gd = R(cv[CS_DUZ_DZ * 32]), ge = R(cv[CS_UR_OVER_R * 32]);
                // K_k = pref H_voigt[k] and 1/K_k once per bin; the k+-1 neighbours come by
                // shuffle (the same products the reference forms at k-1 and k+1)
                // The frequency factors stay FP64 in every precision variant: with F/dw up to
                // ~1e9 at tau0 = 1e8, an FP32 rounding of F0 against Fm + Fp acts as a spurious
                // source or sink tens of times larger than the step's own change.
                double Kb[M], iK[M];
#pragma unroll
                for (int m = 0; m < M; m++) {
                    Kb[m] = pref * double(Hv[m]);
                    iK[m] = rcp<double>(Kb[m]);
                }
                double K_up = __shfl_up_sync(0xffffffffu, Kb[M - 1], 1);
                double K_dn = __shfl_down_sync(0xffffffffu, Kb[0], 1);
                double iK_up = __shfl_up_sync(0xffffffffu, iK[M - 1], 1);
                double iK_dn = __shfl_down_sync(0xffffffffu, iK[0], 1);
#pragma unroll
                for (int m = 0; m < M; m++) {
                    int k = lane * M + m;
                    Fp[m] = 0.0; F0[m] = 0.0; Fm[m] = 0.0;
                    if (k < 1 || k > nnu - 2) continue;
                    RC Drr, DZZ, DrZ;
                    D_edd<RC>(RC(Hr[m]), RC(HZ[m]), RC(J[m]), RC(jeps), RC(a.heps2), Drr, DZZ, DrZ);
                    double vel =
                        double(d_colon_grad_u<RC>(Drr, DrZ, DZZ, RC(ga), RC(gb), RC(gc), RC(gd), RC(ge))) * kInvC;
                    double Kk = Kb[m];
                    double Kkm = (m > 0) ? Kb[m - 1] : K_up;
                    double Kkp = (m < M - 1) ? Kb[m + 1] : K_dn;
                    double iKkm = (m > 0) ? iK[m - 1] : iK_up;
                    double iKkp = (m < M - 1) ? iK[m + 1] : iK_dn;
                    double nCk = kc[KC_NCK * NP + k], nCkp = kc[KC_NCKP * NP + k], nCkm = kc[KC_NCKM * NP + k];
                    double Ckp = vel * nCkp, Ck = vel * nCk, Ckm = vel * nCkm;
                    if (a.recoil) {
                        Ckp += Kkp * (rec0 - 2.0 * kc[KC_ICKP * NP + k]);
                        Ck += Kk * (rec0 - 2.0 * kc[KC_ICK * NP + k]);
                        Ckm += Kkm * (rec0 - 2.0 * kc[KC_ICKM * NP + k]);
                    }
                    double rkp = kc[KC_DNKP * NP + k] * iKkp;
                    double rk = kc[KC_DNK * NP + k] * iK[m];
                    double rkm = kc[KC_DNKM * NP + k] * iKkm;
                    double Pkp = fmin(fmax(Ckp * rkp, -kPmax), kPmax);
                    double Pk = fmin(fmax(Ck * rk, -kPmax), kPmax);
                    double Pkm = fmin(fmax(Ckm * rkm, -kPmax), kPmax);
                    double oRkp, xRkp, oLk, xLk, oRk, xRk, oLkm, xLkm;
                    const double *etab = kc + KC_EXP2 * NP;
                    omphi_R(Pkp, oRkp, xRkp, etab);
                    omphi_LR(Pk, oLk, xLk, oRk, xRk, etab);
                    omphi_L(Pkm, oLkm, xLkm, etab);
                    double idn = kc[KC_IDNU * NP + k];
                    double dkp = idn * rcp<double>(xLk * rk - xRkp * rkp);
                    double dkm = idn * rcp<double>(xLkm * rkm - xRk * rk);
                    Fp[m] = oRkp * dkp;
                    Fm[m] = oLkm * dkm;
                    F0[m] = oLk * dkp + oRk * dkm;
                }
                if (a.Fkp) {
#pragma unroll
                    for (int m = 0; m < M; m++) {
                        int k = lane * M + m;
                        if (k < nnu) { a.Fkp[base + k] = Fp[m]; a.Fk[base + k] = F0[m]; a.Fkm[base + k] = Fm[m]; }
                    }
                }
            } else {
#pragma unroll
                for (int m = 0; m < M; m++) {
                    int k = lane * M + m;
                    bool in = (k >= 1 && k <= nnu - 2);
                    Fp[m] = in ? a.Fkp[base + k] : 0.0;
                    F0[m] = in ? a.Fk[base + k] : 0.0;
                    Fm[m] = in ? a.Fkm[base + k] : 0.0;
                }
            }
            // rows k = 1 .. nnu-2 of src/UpdateLyaJandH.jl:200-214; the couplings of the
            // first and last rows to k = 0 and k = nnu-1 are dropped (TridiagonalSolver.jl:45-46)
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                bool in = (k >= 1 && k <= nnu - 2);
                sys.a[m] = (in && k >= 2) ? Fm[m] : 0.0;
                sys.b[m] = in ? -(F0[m] + dw) : 1.0;
                sys.c[m] = (in && k <= nnu - 3) ? Fp[m] : 0.0;
                sys.d[m] = in ? -dw * Jo[m] : 0.0;
            }
            if (a.solver == SOLVER_THOMAS)
                thomas_solve<M>(sys, lane, tsm + warp * 4 * NP);
            else
                if constexpr (M == 2) cr_pcr_solve2(sys, lane);
                else if constexpr (M == 4) cr_pcr_solve4(sys, lane);
                else pcr_solve<M>(sys, lane);
            // flux correction, src/UpdateLyaJandH.jl:341-377
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                if (k >= nnu) continue;
                bool in = (k >= 1 && k <= nnu - 2);
                double Jn = in ? sys.d[m] : double(J[m]);
                if (!(sys.b[m] != 0.0)) bad |= ERRB_SOLVE;
                double Jf = Jn > jeps ? Jn : jeps;
                double ratio = Jf * rcp<double>(Jo[m] > jeps ? Jo[m] : jeps);
                double hr = double(Hr[m]) * ratio, hz = double(HZ[m]) * ratio;
                double H2 = hr * hr + hz * hz;
                if (H2 > Jf * Jf) {
                    double fsc = Jf * rsqrt_nr(H2);   // |H|^2 > J^2 >= jeps^2: normal
                    hr *= fsc;
                    hz *= fsc;
                }
                J[m] = S(Jf);
                Hr[m] = S(hr);
                HZ[m] = S(hz);
            }
        }
        // ---- store ----
        if (LR::ok && vec) {
            if (lane * M < nnu) {
#pragma unroll
                for (int m = 0; m < M; m++)
                    if (!isfinite(double(J[m])) || !isfinite(double(Hr[m])) || !isfinite(double(HZ[m])))
                        bad |= ERRB_NONFINITE;
                LR::store(a.Jout + base + lane * M, J);
                LR::store(a.Hrout + base + lane * M, Hr);
                LR::store(a.HZout + base + lane * M, HZ);
            }
        } else {
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                if (k >= nnu) continue;
                S js = S(J[m]), hs = S(Hr[m]), zs = S(HZ[m]);
                if (!isfinite(double(js)) || !isfinite(double(hs)) || !isfinite(double(zs))) bad |= ERRB_NONFINITE;
                a.Jout[base + k] = js;
                a.Hrout[base + k] = hs;
                a.HZout[base + k] = zs;
            }
        }
        // ---- epilogue partials ----
        if (a.parts & PART_ACTIVE) {
            const double dV = cv[CS_DV * 32];
#pragma unroll
            for (int m = 0; m < M; m++) {
                int k = lane * M + m;
                if (k >= nnu) continue;
                double dn = kc[KC_DNU * NP + k];
                double Jv = double(S(J[m]));
                double e1 = Jv - 10.0 * jeps, e0 = Jv - jeps;
                acc_e[m] += dn * (e1 > 0.0 ? e1 : 0.0) * dV;
                acc_tot += dn * (e0 > 0.0 ? e0 : 0.0) * dV;
            }
        }
        if (a.parts & PART_DIAG) {
            // escaping flux through the outer r face, the top face and (outflow) the bottom face
            double esc = 0.0;
            const bool rb = (i == nr - 1), zt = (j == nz - 1), zb = (j == 0 && bzb == 1);
            if (rb || zt || zb) {
                const double Arr = rb ? __ldg(a.A_r + cd.orf + nr + (long long)(nr + 1) * j) * kFourPi : 0.0;
                const double AZt = zt ? __ldg(a.A_Z + cd.ozf + i + (long long)nr * nz) * kFourPi : 0.0;
                const double AZb = zb ? __ldg(a.A_Z + cd.ozf + i) * kFourPi : 0.0;
#pragma unroll
                for (int m = 0; m < M; m++) {
                    int k = lane * M + m;
                    if (k >= nnu) continue;
                    double dn = kc[KC_DNU * NP + k];
                    double hr = double(S(Hr[m])) * a.j_scale, hz = double(S(HZ[m])) * a.j_scale;
                    if (rb) esc += dn * (Arr * (hr > 0.0 ? hr : 0.0));
                    if (zt) esc += dn * (AZt * (hz > 0.0 ? hz : 0.0));
                    if (zb) esc += dn * (AZb * (-hz > 0.0 ? -hz : 0.0));
                }
            }
            acc_esc += esc;
        }
    }
    if (wbeg < wend) flush(g0, wend);
    if constexpr (PF) cp_async_wait<0>();
    if (bad) atomicOr(a.err, bad);
    if (!a.parts) return;
    // ---- CTA reduction of the partials, fixed order ----
    // (the warp's own row: with prefetch it overlays the warp's prefetch area, whose last copies
    // landed above)
    double *red = freq_red_row<M>(fsm, nw, ns, warp);
    __syncwarp();
    if (warp < nw) {
#pragma unroll
        for (int m = 0; m < M; m++) red[lane * M + m] = acc_e[m];
    }
    acc_tot = warp_sum(acc_tot);
    acc_esc = warp_sum(acc_esc);
    acc_mf = warp_sum(acc_mf);
    acc_net = warp_sum(acc_net);
    acc_out = warp_sum(acc_out);
    acc_L = warp_sum(acc_L);
    if (lane == 0 && warp < nw) {
        red[NP + 0] = acc_tot;
        red[NP + 1] = acc_mf;
        red[NP + 2] = acc_net;
        red[NP + 3] = acc_out;
        red[NP + 4] = acc_L;
        red[NP + 5] = acc_esc;
    }
    __syncthreads();
    const int ncols = nnu + kExtraCols;
    for (int col = threadIdx.x; col < ncols; col += blockDim.x) {
        int src = col < nnu ? col : NP + (col - nnu);
        double s = 0.0;
        for (int w2 = 0; w2 < nw; w2++) s += freq_red_row<M>(fsm, nw, ns, w2)[src];
        a.partials[(size_t)col * nitems + item] = s;
    }
}

template <typename S, typename R, int M, typename RC = R>
__global__ void __launch_bounds__(FREQ_THREADS, M <= 4 ? 2 : 1) k_freq(FreqArgs<S> a) {
    extern __shared__ __align__(16) double fsm[];
    freq_item<S, R, M, RC>(a, a.item0 + (int)blockIdx.x, a.nitems_all ? a.nitems_all : (int)gridDim.x, fsm,
                           blockDim.x >> 5);
}

// FindActiveBins partials of the current J (src/UpdateLyaJandH.jl:47-97): one warp per cell,
// the same work items (and so the same summation order) as k_freq.
template <typename S, int M>
__global__ void __launch_bounds__(FREQ_THREADS) k_find_active(const S *J, int nnu, const double *dnu,
                                                              const double *dV, const CloudDesc *cl, const int4 *items,
                                                              double jeps, double *partials) {
    extern __shared__ __align__(16) double fsm[];
    constexpr int NP = 32 * M;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int4 it = items[blockIdx.x];
    const long long o3 = cl[it.x].o3, oc = cl[it.x].oc;
    double acc_e[M];
#pragma unroll
    for (int m = 0; m < M; m++) acc_e[m] = 0.0;
    double acc_tot = 0.0;
    int wbeg, wend;
    warp_cell_run(it, warp, nw, wbeg, wend);
    for (int c = wbeg; c < wend; c++) {
        const double v = __ldg(dV + oc + c);
#pragma unroll
        for (int m = 0; m < M; m++) {
            int k = lane * M + m;
            if (k >= nnu) continue;
            double Jv = double(__ldg(J + o3 + (long long)c * nnu + k));
            double dn = __ldg(dnu + k);
            double e1 = Jv - 10.0 * jeps, e0 = Jv - jeps;
            acc_e[m] += dn * (e1 > 0.0 ? e1 : 0.0) * v;
            acc_tot += dn * (e0 > 0.0 ? e0 : 0.0) * v;
        }
    }
    const int stride = NP + 8;
#pragma unroll
    for (int m = 0; m < M; m++) fsm[warp * stride + lane * M + m] = acc_e[m];
    acc_tot = warp_sum(acc_tot);
    if (lane == 0) fsm[warp * stride + NP] = acc_tot;
    __syncthreads();
    for (int col = threadIdx.x; col <= nnu; col += blockDim.x) {
        int src = col < nnu ? col : NP;
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += fsm[w * stride + src];
        partials[(size_t)col * gridDim.x + blockIdx.x] = s;
    }
}

// Column sums of each cloud's partials (one warp per column, a fixed order), then, by one thread
// per cloud, FindActiveBins' decision and the diagnostics of Update_f_Lya_MF_L_Lya! /
// Compute_f_esc_Lya_Cylindrical. With a.cnt set, each cloud's columns are spread over CTAs of
// 8 warps, one column per warp, whose sums go through a.colsum; the last CTA of the cloud to
// finish takes the decision. Without, one CTA per cloud sums every column. The last decision
// of the launch advances the record index.
// reduce_block is block `vb` of that launch by the calling CTA (all its warps): the body of
// k_reduce, also run by the persistent batch kernel.
__device__ __forceinline__ void reduce_block(const RedArgs &a, int vb) {
    __shared__ double col[256 + kExtraCols];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int ncols = a.nnu + kExtraCols;
    const bool split = a.cnt != nullptr;
    const int nchunks = split ? (ncols + nw - 1) / nw : 1;
    const int cloud = vb / nchunks, chunk = vb % nchunks;
    const CloudDesc &cd = a.cl[cloud];
    const int npb = cd.npb;
    const double *pbase = a.partials + cd.pb0;
    const int c0 = split ? chunk * nw : 0, c1 = split ? min(ncols, c0 + nw) : ncols;
    for (int cc = c0 + warp; cc < c1; cc += nw) {
        bool need = (cc < a.nnu + 1) ? (a.parts & PART_ACTIVE) : (a.parts & PART_DIAG);
        double s = 0.0;
        if (need) {
            const double *p = pbase + (size_t)cc * a.nblocks;
            for (int b = lane; b < npb; b += 32) s += p[b];
        }
        s = warp_sum(s);
        if (lane == 0) {
            col[cc] = s;
            if (split) a.colsum[(size_t)cloud * ncols + cc] = s;
        }
    }
    if (split) {
        // the last CTA of this cloud gathers the other CTAs' sums (threadfence reduction)
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) is_last = atomicAdd(a.cnt + cloud, 1) == nchunks - 1;
        __syncthreads();
        if (!is_last) return;
        __threadfence();
        for (int cc = threadIdx.x; cc < ncols; cc += blockDim.x) col[cc] = __ldcg(a.colsum + (size_t)cloud * ncols + cc);
        if (threadIdx.x == 0) a.cnt[cloud] = 0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    int *kw = a.kwin + 2 * cloud;
    int used_kmin = kw[0], used_kmax = kw[1];
    if (a.parts & PART_ACTIVE) {
        double Etot = col[a.nnu];
        int kmin = a.nnu - 1, kmax = 0;
        for (int k = 0; k < a.nnu; k++) {
            if (col[k] > kEpsActive * Etot) {
                kmin = k < kmin ? k : kmin;
                kmax = k > kmax ? k : kmax;
            }
        }
        kmax = kmax > a.kcore_max ? kmax : a.kcore_max;
        kmin = kmin < a.kcore_min ? kmin : a.kcore_min;
        kw[0] = kmin;
        kw[1] = kmax;
        if (a.kwin_copy) {
            a.kwin_copy[2 * cloud] = kmin;
            a.kwin_copy[2 * cloud + 1] = kmax;
        }
    }
    if (a.parts & PART_DIAG) {
        double MF = col[a.nnu + 1], net = col[a.nnu + 2], outw = col[a.nnu + 3];
        double L = col[a.nnu + 4];
        if (L > 0.0) {
            double kk = 1.0 / (L / kC);
            MF *= kk; net *= kk; outw *= kk;
        } else {
            MF = 0.0; net = 0.0; outw = 0.0;
        }
        double Ltot = (cd.bc_z_bot == 0) ? 2.0 * L : L;
        double Lsim = (cd.bc_z_bot == 0) ? 0.5 * Ltot : Ltot;
        double fesc = (Ltot > 0.0 && Lsim > 0.0) ? col[a.nnu + 5] / Lsim : 0.0;
        double rec[7] = {MF, net, outw, Ltot, fesc, (double)used_kmin, (double)used_kmax};
        if (a.last)
            for (int q = 0; q < 7; q++) a.last[(size_t)cloud * 7 + q] = rec[q];
        if (a.diag && a.step_counter) {
            int idx = *a.step_counter;
            if (idx < a.hist_capacity)
                for (int q = 0; q < 7; q++) a.diag[((size_t)idx * a.nclouds + cloud) * 7 + q] = rec[q];
            __threadfence();
            int done = atomicAdd(a.done, 1);
            if (done == a.nclouds - 1) {
                *a.step_counter = idx + 1;
                *a.done = 0;
            }
        }
    }
}

__global__ void __launch_bounds__(1024) k_reduce(RedArgs a) { reduce_block(a, blockIdx.x); }

// ---- the persistent step: one cooperative launch runs the three phases -----------------------
//
// A grid barrier with a bounded wait: the CTAs of the launch arrive on a counter; the last to
// arrive resets it and advances the generation the others wait on. A wait that outlasts `polls`
// polls sets ERRB_TIMEOUT and the CTA leaves the launch (the others then time out at this or
// the next barrier), so a launch never hangs. Fences order each CTA's writes of one phase before
// the other CTAs' reads of the next.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned nblocks, long long polls, int *err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        int good = 1;
        if (atomicAdd(bar, 1u) + 1u == nblocks) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > polls) {
                    good = 0;
                    atomicOr(err, ERRB_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// One fused static step of every cloud of a batch in one launch: the advection tiles, a grid
// barrier, the frequency-kernel items (8 of the CTA's 9 warps take the cells, as in k_freq), a
// grid barrier, the reduction blocks; each CTA walks the work lists with a grid stride. The rows
// are staged by per-lane loads. Within a launch every buffer one phase reads was written by an
// earlier launch or after a barrier, so no read meets a stale copy: the advection reads the set
// the previous launch's frequency phase wrote.
template <typename S>
struct PersistArgs {
    AdvArgs<S> adv;
    FreqArgs<S> freq;
    RedArgs red;
    int ntiles, nitems, nred;
    unsigned *bar;          // [0] arrivals, [1] generation; [0] zero before the launch
    long long polls;
    int *err;
};

// RA: arithmetic of the advection; RF, RC: of the frequency step and its closure (as k_freq).
template <typename S, typename RA, typename RF, typename RC, int FLUX, int M>
__global__ void __launch_bounds__(MTHREADS, 2) k_step_persistent(PersistArgs<S> p) {
    extern __shared__ __align__(128) unsigned char psm[];
    for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
        advect_tile<S, RA, FLUX, false>(p.adv, t, psm);
        __syncthreads();
    }
    if (!grid_barrier(p.bar, gridDim.x, p.polls, p.err)) return;
    for (int it = blockIdx.x; it < p.nitems; it += gridDim.x) {
        freq_item<S, RF, M, RC>(p.freq, it, p.nitems, reinterpret_cast<double *>(psm), FREQ_THREADS / 32);
        __syncthreads();
    }
    if (!grid_barrier(p.bar, gridDim.x, p.polls, p.err)) return;
    for (int vb = blockIdx.x; vb < p.nred; vb += gridDim.x) {
        reduce_block(p.red, vb);
        __syncthreads();
    }
}

// ---- launch wrappers ----------------------------------------------------------------------
template <typename S, typename R, bool TMA>
static size_t adv_smem_bytes() {
    if (!TMA) return adv_smem_base<S, R, adv_pfr<R, TMA>()>();
    return adv_tma_off(adv_smem_base<S, R, false>()) + raw_tile_bytes<S>() + 16;   // raw tile, mbarrier, abort flag
}

template <typename S, typename R, int FLUX, int MINB, bool TMA>
static void adv_launch_t(const void *args, int ntiles, cudaStream_t st) {
    static bool attr = false;
    size_t sm = adv_smem_bytes<S, R, TMA>();
    if (!attr) {
        cudaFuncSetAttribute(k_advect<S, R, FLUX, MINB, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        attr = true;
    }
    k_advect<S, R, FLUX, MINB, TMA><<<ntiles, MTHREADS, sm, st>>>(*static_cast<const AdvArgs<S> *>(args));
}

// the bulk-copy staging runs when the caller encoded tensor maps for this launch's input state
template <typename S, typename R, int FLUX, int MINB>
static void adv_launch(const void *args, int ntiles, cudaStream_t st) {
    if (static_cast<const AdvArgs<S> *>(args)->tmaps) adv_launch_t<S, R, FLUX, MINB, true>(args, ntiles, st);
    else adv_launch_t<S, R, FLUX, MINB, false>(args, ntiles, st);
}

template <typename S, typename R, int FLUX>
static void adv_occ(const void *args, int ntiles, cudaStream_t st, int ctas) {
    if (ctas >= 4) adv_launch<S, R, FLUX, 4>(args, ntiles, st);
    else if (ctas == 2) adv_launch<S, R, FLUX, 2>(args, ntiles, st);
    else adv_launch<S, R, FLUX, 3>(args, ntiles, st);
}

int adv_ctas_per_sm(int prec, int want) {
    if (prec == PREC_K_FP64) return (want == 2) ? 2 : 3;   // FP64: 76 KB of shared memory, 72 registers
    return (want >= 2 && want <= 4) ? want : 4;
}

void launch_advect(int prec, int flux, const void *args, int ntiles, int ctas, cudaStream_t st) {
    if (ntiles <= 0) return;
    ctas = adv_ctas_per_sm(prec, ctas);
    if (prec == PREC_K_FP64) {
        if (ctas == 3) {
            if (flux == 0) adv_launch<double, double, 0, 3>(args, ntiles, st);
            else adv_launch<double, double, 1, 3>(args, ntiles, st);
        } else {
            if (flux == 0) adv_launch<double, double, 0, 2>(args, ntiles, st);
            else adv_launch<double, double, 1, 2>(args, ntiles, st);
        }
    } else if (prec == PREC_K_MIXED) {
        if (flux == 0) adv_occ<double, float, 0>(args, ntiles, st, ctas);
        else adv_occ<double, float, 1>(args, ntiles, st, ctas);
    } else {
        if (flux == 0) adv_occ<float, float, 0>(args, ntiles, st, ctas);
        else adv_occ<float, float, 1>(args, ntiles, st, ctas);
    }
}

int bins_per_lane(int nnu) { return nnu <= 32 ? 1 : nnu <= 64 ? 2 : nnu <= 128 ? 4 : 8; }

int freq_blocks(int ncell, int dev) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int want = (ncell + (FREQ_THREADS / 32) - 1) / (FREQ_THREADS / 32);
    int cap = sms * 4;
    return want < cap ? (want > 0 ? want : 1) : cap;
}

static bool al16(const void *p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename S, typename R, int M, typename RC>
static void freq_launch(const void *args, int nitems, cudaStream_t st) {
    FreqArgs<S> fa = *static_cast<const FreqArgs<S> *>(args);
    // every row of every cloud starts on a 16-byte boundary when the buffers do and a row
    // (n_nu elements) is a multiple of 16 bytes: cloud offsets are sums of whole rows
    fa.vec16 = LaneRow<S, M>::ok && fa.nnu % M == 0 && (fa.nnu * sizeof(S)) % 16 == 0 && al16(fa.Jin) &&
               al16(fa.Hrin) && al16(fa.HZin) && al16(fa.Jold) && al16(fa.Hv) && al16(fa.Jout) && al16(fa.Hrout) &&
               al16(fa.HZout);
    const int ns = fa.Jold == fa.Jin ? 4 : 5;
    const size_t sm = sizeof(double) * freq_smem_doubles<M>(FREQ_THREADS / 32, fa.solver == SOLVER_THOMAS, ns);
    static bool attr = false;
    if (!attr) {
        const size_t smax = sizeof(double) * freq_smem_doubles<M>(FREQ_THREADS / 32, true, 5);
        cudaFuncSetAttribute(k_freq<S, R, M, RC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
        attr = true;
    }
    k_freq<S, R, M, RC><<<nitems, FREQ_THREADS, sm, st>>>(fa);
}

void launch_freq(int prec, const void *args, int nnu, int nitems, cudaStream_t st) {
    if (nitems <= 0) return;
    int M = bins_per_lane(nnu);
#define LYD_FQ(S_, R_, RC_)                                              \
    switch (M) {                                                         \
    case 1: freq_launch<S_, R_, 1, RC_>(args, nitems, st); break;        \
    case 2: freq_launch<S_, R_, 2, RC_>(args, nitems, st); break;        \
    case 4: freq_launch<S_, R_, 4, RC_>(args, nitems, st); break;        \
    default: freq_launch<S_, R_, 8, RC_>(args, nitems, st); break;       \
    }
    // the mixed variant keeps the frequency step in FP64 (its state, factors and solve need
    // it) except the closure that sets the Doppler velocity (see k_freq)
    if (prec == PREC_K_FP32) {
        LYD_FQ(float, float, float)
    } else if (prec == PREC_K_MIXED) {
        LYD_FQ(double, double, float)
    } else {
        LYD_FQ(double, double, double)
    }
#undef LYD_FQ
}

template <typename S, int M>
static void active_launch(const S *J, int nnu, const double *dnu, const double *dV, const CloudDesc *cl,
                          const int4 *items, int nitems, double jeps, double *partials, cudaStream_t st) {
    size_t sm = sizeof(double) * (FREQ_THREADS / 32) * (32 * M + 8);
    k_find_active<S, M><<<nitems, FREQ_THREADS, sm, st>>>(J, nnu, dnu, dV, cl, items, jeps, partials);
}

void launch_find_active(int sprec, const void *J, int nnu, const double *dnu, const double *dV, const CloudDesc *cl,
                        const int4 *items, int nitems, double jeps, double *partials, cudaStream_t st) {
    if (nitems <= 0) return;
    int M = bins_per_lane(nnu);
#define LYD_ACT(T, MM) \
    active_launch<T, MM>(static_cast<const T *>(J), nnu, dnu, dV, cl, items, nitems, jeps, partials, st)
    if (sprec == 0) {
        switch (M) { case 1: LYD_ACT(double, 1); break; case 2: LYD_ACT(double, 2); break;
                     case 4: LYD_ACT(double, 4); break; default: LYD_ACT(double, 8); break; }
    } else {
        switch (M) { case 1: LYD_ACT(float, 1); break; case 2: LYD_ACT(float, 2); break;
                     case 4: LYD_ACT(float, 4); break; default: LYD_ACT(float, 8); break; }
    }
#undef LYD_ACT
}

template <typename S, typename RA, typename RF, typename RC, int FLUX, int M>
static cudaError_t persist_launch(const void *adv, const void *freq, const RedArgs &red, int ntiles, int nitems,
                                  unsigned *bar, long long polls, int *err, cudaStream_t st) {
    PersistArgs<S> p;
    p.adv = *static_cast<const AdvArgs<S> *>(adv);
    p.adv.tmaps = nullptr;
    p.freq = *static_cast<const FreqArgs<S> *>(freq);
    p.freq.vec16 = LaneRow<S, M>::ok && p.freq.nnu % M == 0 && (p.freq.nnu * sizeof(S)) % 16 == 0 && al16(p.freq.Jin) &&
                   al16(p.freq.Hrin) && al16(p.freq.HZin) && al16(p.freq.Jold) && al16(p.freq.Hv) &&
                   al16(p.freq.Jout) && al16(p.freq.Hrout) && al16(p.freq.HZout);
    p.red = red;
    if (!red.colsum) p.red.cnt = nullptr;
    const int ncols = red.nnu + kExtraCols, rw = MTHREADS / 32;
    p.ntiles = ntiles;
    p.nitems = nitems;
    p.nred = p.red.cnt ? red.nclouds * ((ncols + rw - 1) / rw) : red.nclouds;
    p.bar = bar;
    p.polls = polls;
    p.err = err;
    auto kern = k_step_persistent<S, RA, RF, RC, FLUX, M>;
    const size_t sa = adv_smem_bytes<S, RA, false>();
    const size_t sf = sizeof(double) * freq_smem_doubles<M>(FREQ_THREADS / 32, p.freq.solver == SOLVER_THOMAS,
                                                            p.freq.Jold == p.freq.Jin ? 4 : 5);
    const size_t sm = sa > sf ? sa : sf;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, MTHREADS, sm);
    if (e != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(per * sms));
    cfg.blockDim = dim3(MTHREADS);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, kern, p);
}

cudaError_t launch_persistent(int prec, int flux, const void *adv, const void *freq, const RedArgs &red, int nnu,
                              int ntiles, int nitems, unsigned *bar, long long polls, int *err, cudaStream_t st) {
    const int M = bins_per_lane(nnu);
#define LYD_PS1(S_, RA_, RF_, RC_, M_)                                                                     \
    return flux == 0 ? persist_launch<S_, RA_, RF_, RC_, 0, M_>(adv, freq, red, ntiles, nitems, bar, polls, err, st) \
                     : persist_launch<S_, RA_, RF_, RC_, 1, M_>(adv, freq, red, ntiles, nitems, bar, polls, err, st);
#define LYD_PS(S_, RA_, RF_, RC_)                                                                         \
    switch (M) {                                                                                          \
    case 1: LYD_PS1(S_, RA_, RF_, RC_, 1)                                                                 \
    case 2: LYD_PS1(S_, RA_, RF_, RC_, 2)                                                                 \
    case 4: LYD_PS1(S_, RA_, RF_, RC_, 4)                                                                 \
    default: LYD_PS1(S_, RA_, RF_, RC_, 8)                                                                \
    }
    // the arithmetic of each phase as in launch_advect and launch_freq
    if (prec == PREC_K_FP32) {
        LYD_PS(float, float, float, float)
    } else if (prec == PREC_K_MIXED) {
        LYD_PS(double, float, double, float)
    } else {
        LYD_PS(double, double, double, double)
    }
#undef LYD_PS
#undef LYD_PS1
}

void launch_reduce(const RedArgs &a, cudaStream_t st) {
    if (a.nclouds <= 0) return;
    if (a.cnt && a.colsum) {
        const int nchunks = (a.nnu + kExtraCols + 7) / 8;
        k_reduce<<<a.nclouds * nchunks, 256, 0, st>>>(a);
    } else {
        RedArgs b = a;
        b.cnt = nullptr;
        k_reduce<<<a.nclouds, 1024, 0, st>>>(b);
    }
}

}  // namespace lyd
