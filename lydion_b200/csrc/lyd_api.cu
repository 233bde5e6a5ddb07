// lyd_api.cu -- the C ABI (include/lydion_m1.h): context, device state, and the drop-in
// entry points of the Lyman-alpha M1 step.
//
// A context holds a batch of independent clouds (one cloud for lyd_create). Every field of
// every cloud lives in one concatenated device array per field, cloud after cloud; the
// per-cloud offsets, sizes, boundary conditions and time step are CloudDesc records in
// device memory that the kernels read, so changing a time step is a 100-byte copy and the
// captured step graph stays valid.
//
// Device state. J, H_r, H_Z live in two buffer sets. `cur` holds the current values; the
// other set holds J_old, H_r_old, H_Z_old unless `old_alias` is set, in which case the old
// values equal the current ones (true after every step phase of the reference:
// AdvectLya! copies J_old = J and H_old = H, the emission and frequency updates end by
// setting the old arrays to the new ones). The advection writes into the spare set and the
// sets swap; the emission and frequency kernels work per cell in place. The fused
// static-cloud step advects cur -> spare and then runs emission + frequency spare -> cur,
// so a step starts and ends in the same set and one CUDA graph replays every step.
#include <cuda.h>   // CUtensorMap and its enums (types only: the driver entry point is fetched at run time)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <functional>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "lyd_adjoint.h"
#include "lyd_internal.h"
#include "lyd_physics.cuh"
#include "lydion_m1.h"

using namespace lyd;

namespace {
constexpr int kLutN = 200001;        // src/FastInterpolations.jl:175-176
constexpr double kLutXmax = 1000.0;
constexpr int kTileCols = 8;         // columns per advection tile (the kernel's MT)
constexpr int kDefaultRows = 16;

// per-cloud "was provided" bits: per-cell fields use their index (field - LYD_F_ALPHA)
enum { CF_ALPHA = 0, CF_ALPHA_C, CF_ALPHA_CF, CF_PD, CF_JS, CF_T, CF_DUR_DR, CF_DUR_DZ, CF_DUZ_DR, CF_DUZ_DZ,
       CF_UR_OVER_R, CF_DRU_R, CF_DRU_Z, CF_F_R, CF_F_Z, CF_E_LYA, CF_N };
enum : unsigned { BIT_HV = 1u << 16, BIT_PHI = 1u << 17, BIT_AF = 1u << 18, BIT_GEOM = 1u << 19 };
}  // namespace

struct lyd_ctx {
    int dev = 0;
    cudaStream_t st = nullptr;
    int nnu = 0, ncl = 0, sms = 148;
    std::vector<int> nr, nz;
    std::vector<CloudDesc> desc;       // host copy of the descriptors
    std::vector<CloudDesc> desc_dev;   // what the device holds (to skip unchanged uploads)
    CloudDesc *cl = nullptr;
    std::vector<unsigned> have;        // per-cloud provided bits
    size_t ncell = 0, n3 = 0, nrf = 0, nzf = 0, ncol = 0, nrow = 0, nrint = 0, nzint = 0, nrif = 0, nzif = 0;
    lyd_config cfg{};
    int prec = 0;                      // kernel variant (LYD_PREC_*)
    int sprec = 0;                     // storage of the state arrays: 0 double, 1 float
    size_t ssz = 8;
    double jscale = 1.0, jeps_s = kJeps, heps2_s = kHeps * kHeps;
    void *set[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int cur = 0;
    bool old_alias = true;
    void *Hv = nullptr;
    bool hv_from_T = false;            // H_voigt last computed on the device from T
    void *phi = nullptr;
    double *phi_inv = nullptr;
    int phi_kmin = 0, phi_kmax = -1;
    bool phi_inv_ready = false;
    void *aF = nullptr;
    double *Ff[3] = {nullptr, nullptr, nullptr};
    bool ff_valid = false;
    double *cellf[CF_N] = {};
    CloudDesc *dd_cl = nullptr;    // device record of lyd_dd_finish (the all-reduced columns)
    double *dust_F = nullptr;      // [3][ncell] dust flux opacities of the RHD Lya block (set by
                                   // lyd_rhd_lya_prepare)
    double *u_r_star = nullptr, *u_Z_star = nullptr;
    double *dV = nullptr, *inv_dV = nullptr, *A_r = nullptr, *A_Z = nullptr, *inv_r_cell = nullptr;
    double *rCoM = nullptr, *ZCoM = nullptr, *rint = nullptr, *zint = nullptr, *r_if = nullptr, *Z_if = nullptr;
    double *nu = nullptr, *nuC = nullptr, *dnu = nullptr, *inv_dnu = nullptr, *inv_nuC = nullptr;
    bool freq_set = false;
    // work lists
    lyd_tuning tune{kDefaultRows, 0, SOLVER_PCR, 0, LYD_STAGING_AUTO};
    unsigned char *tmaps = nullptr;    // tensor maps of J, H_r, H_Z: [set][cloud][3] (TMA staging)
    bool tma_ok = false;               // every map encoded (the layout allows bulk tensor copies)
    int4 *tiles = nullptr, *items = nullptr;
    int ntiles = 0, nitems = 0;
    double *partials = nullptr;
    int *kwin = nullptr;
    bool active_valid = false;
    double *hist = nullptr;
    int hist_cap = 0;                  // steps
    int *step_ctr = nullptr;           // [0] record index, [1] completion counter
    double *red_cols = nullptr;        // column sums of the reduction [cloud][N_nu + kExtraCols]
    int *red_cnt = nullptr;            // per-cloud CTA counters of the reduction (zero between launches)
    double *last = nullptr;
    int *err = nullptr;
    double *lut = nullptr;
    double *stage = nullptr;           // device FP64 staging buffer
    size_t stage_n = 0;
    double *small = nullptr;           // device scratch (512 doubles)
    cudaGraphExec_t gexec = nullptr;
    int gkey_cur = -1;
    long long gkey_polls = 0;          // 0: the three-launch step graph; else the persistent step's poll limit
    // the host-state step (lyd_static_step_host): the state as uploaded, the window check, the
    // work lists grouped by row chunk, its copy streams and events
    double *hin = nullptr;             // [3][n3] J, H_r, H_Z as uploaded
    double *part_chk = nullptr;        // FindActiveBins partials of the uploaded J
    int *kwin_chk = nullptr;           // the window the step used, then the window of the uploaded J
    int4 *ctiles = nullptr;            // advection tiles, chunk after chunk
    std::vector<int> ct_off, it_off, row_off;
    int hs_req = 0, hs_chunks = 0, hs_rows = 0, hs_cpb = 0, hs_pchk = 0;
    cudaStream_t st_up = nullptr, st_dn = nullptr, st_fq = nullptr;
    cudaEvent_t hs_ev[3 * 16 + 2] = {};
    // the adjoint's recomputation stream, and its events: recomputed (2), reversed (2), start
    cudaStream_t st_rec = nullptr;
    cudaEvent_t adj_ev[5] = {};
    unsigned *bar = nullptr;           // grid barrier of the persistent step: arrivals, generation
    int persist_graph = 0;             // persistent step replayed from a graph: 1 yes, -1 no (capture refused)
    bool timing = false;
    cudaEvent_t ev[8] = {};
    double ms[3] = {0, 0, 0};
    double adj_ms[5] = {0, 0, 0, 0, 0};
    void *adj_ws = nullptr;            // adjoint workspace, kept between calls (grow only)
    size_t adj_ws_bytes = 0;
    std::string msg;
};

static int fail(lyd_ctx *c, int code, const std::string &m) {
    if (c) c->msg = m;
    return code;
}

#define LYD_CU(ctx, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(ctx, LYD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

static int dalloc(lyd_ctx *c, void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, LYD_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    e = cudaMemsetAsync(*p, 0, bytes ? bytes : 16, c->st);
    if (e != cudaSuccess) return fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
    return LYD_OK;
}
#define LYD_TRY(x)              \
    do {                        \
        int r_ = (x);           \
        if (r_ != LYD_OK) return r_; \
    } while (0)

static void *Jc(lyd_ctx *c, int q) { return c->set[c->cur][q]; }
static void *Jold(lyd_ctx *c, int q) { return c->old_alias ? c->set[c->cur][q] : c->set[1 - c->cur][q]; }
static char *at(void *p, size_t elems, size_t esz) { return static_cast<char *>(p) + elems * esz; }

static bool all_have(const lyd_ctx *c, unsigned bit) {
    for (unsigned h : c->have)
        if (!(h & bit)) return false;
    return true;
}
static bool any_have(const lyd_ctx *c, unsigned bit) {
    for (unsigned h : c->have)
        if (h & bit) return true;
    return false;
}
static void set_all(lyd_ctx *c, unsigned bit) {
    for (unsigned &h : c->have) h |= bit;
}

static int check_err(lyd_ctx *c) {
    int h = 0;
    LYD_CU(c, cudaMemcpyAsync(&h, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    if (h) {
        LYD_CU(c, cudaMemsetAsync(c->err, 0, sizeof(int), c->st));
        if (h & ERRB_TIMEOUT) {
            // a persistent step whose CTAs left early may leave the reduction's counters part-way
            LYD_CU(c, cudaMemsetAsync(c->red_cnt, 0, (size_t)c->ncl * sizeof(int), c->st));
            LYD_CU(c, cudaMemsetAsync(c->step_ctr + 1, 0, sizeof(int), c->st));
            LYD_CU(c, cudaStreamSynchronize(c->st));
            c->active_valid = false;
            return fail(c, LYD_ERR_TIMEOUT,
                        "a bounded wait ran out (a bulk copy of the advection's staging or a grid barrier of the "
                        "persistent step)");
        }
        if (h & ERRB_NONFINITE) return fail(c, LYD_ERR_NONFINITE, "non-finite value in J or H");
        return fail(c, LYD_ERR_SOLVE, "zero pivot in a frequency tridiagonal system");
    }
    return LYD_OK;
}

// Copy the host descriptors to the device when they changed. A pageable host-to-device
// cudaMemcpyAsync returns once the source is staged, so the host copy may change right after.
static int sync_desc(lyd_ctx *c) {
    if (c->desc_dev.size() == c->desc.size() &&
        memcmp(c->desc_dev.data(), c->desc.data(), c->desc.size() * sizeof(CloudDesc)) == 0)
        return LYD_OK;
    LYD_CU(c, cudaMemcpyAsync(c->cl, c->desc.data(), c->desc.size() * sizeof(CloudDesc), cudaMemcpyHostToDevice,
                              c->st));
    c->desc_dev = c->desc;
    return LYD_OK;
}

static void drop_graph(lyd_ctx *c) {
    if (c->gexec) {
        cudaGraphExecDestroy(c->gexec);
        c->gexec = nullptr;
    }
}

// Work lists. Advection: tiles of 8 columns x rows x 32 bins, column tile fastest, per cloud.
// Frequency kernel: runs of `cpb` consecutive cells of one cloud per block.
static int cells_per_block(const lyd_ctx *c) {
    if (c->tune.cells_per_block > 0) return c->tune.cells_per_block;
    long long want = (long long)(c->ncell + 4 * c->sms - 1) / (4 * c->sms);
    want = (want + 7) / 8 * 8;
    return (int)std::min<long long>(1024, std::max<long long>(8, want));
}

static int build_work(lyd_ctx *c) {
    const int rows = c->tune.rows_per_tile;
    std::vector<int4> t, it;
    const int nkb = (c->nnu + 31) / 32;
    for (int q = 0; q < c->ncl; q++)
        for (int kb = 0; kb < nkb; kb++)
            for (int j0 = c->desc[q].j_own0; j0 < c->desc[q].j_own1; j0 += rows)
                for (int i0 = 0; i0 < c->nr[q]; i0 += kTileCols) t.push_back(make_int4(q, i0, j0, 32 * kb));
    const int cpb = cells_per_block(c);
    for (int q = 0; q < c->ncl; q++) {
        const int b0 = c->nr[q] * c->desc[q].j_own0, nc = c->nr[q] * c->desc[q].j_own1;   // owned cells
        c->desc[q].pb0 = (int)it.size();
        for (int b = b0; b < nc; b += cpb) it.push_back(make_int4(q, b, std::min(nc, b + cpb), 0));
        c->desc[q].npb = (int)it.size() - c->desc[q].pb0;
    }
    cudaFree(c->tiles);
    cudaFree(c->items);
    cudaFree(c->partials);
    c->tiles = c->items = nullptr;
    c->partials = nullptr;
    LYD_TRY(dalloc(c, (void **)&c->tiles, t.size() * sizeof(int4)));
    LYD_TRY(dalloc(c, (void **)&c->items, it.size() * sizeof(int4)));
    LYD_TRY(dalloc(c, (void **)&c->partials, it.size() * (size_t)(c->nnu + kExtraCols) * 8));
    LYD_CU(c, cudaMemcpyAsync(c->tiles, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice, c->st));
    LYD_CU(c, cudaMemcpyAsync(c->items, it.data(), it.size() * sizeof(int4), cudaMemcpyHostToDevice, c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    c->ntiles = (int)t.size();
    c->nitems = (int)it.size();
    drop_graph(c);
    return sync_desc(c);
}

static int ensure_stage(lyd_ctx *c, size_t n) {
    if (n <= c->stage_n) return LYD_OK;
    LYD_CU(c, cudaStreamSynchronize(c->st));
    cudaFree(c->stage);
    c->stage = nullptr;
    c->stage_n = 0;
    LYD_TRY(dalloc(c, (void **)&c->stage, n * 8));
    c->stage_n = n;
    return LYD_OK;
}

// Every lyd_* definition below has C linkage through its declaration in lydion_m1.h.

int lyd_abi_version(void) { return LYD_ABI_VERSION; }

// cuTensorMapEncodeTiled, fetched from the driver at run time (the library links no libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// Tensor maps for the advection's bulk-copy staging: one per cloud, field (J, H_r, H_Z) and
// buffer set, over the cloud's [n_nu][n_r][n_z] block with a box of 32 bins x (tile columns + 4
// halo columns) x 1 row. A map needs its block to start on a 16-byte boundary and a row of
// n_nu elements to be a multiple of 16 bytes; cloud blocks are sums of whole rows, so the
// second implies the first. When that fails, or the driver lacks the encoder, the advection
// stages with per-lane loads.
static int encode_tmaps(lyd_ctx *c) {
    static_assert(sizeof(CUtensorMap) == kTensorMapBytes, "tensor map size");
    c->tma_ok = false;
    const size_t es = c->ssz;
    if ((c->nnu * es) % 16 != 0) return LYD_OK;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return LYD_OK;
    std::vector<CUtensorMap> maps((size_t)2 * c->ncl * 3);
    for (int s = 0; s < 2; s++)
        for (int q = 0; q < c->ncl; q++)
            for (int f = 0; f < 3; f++) {
                const CloudDesc &d = c->desc[q];
                void *base = static_cast<char *>(c->set[s][f]) + (size_t)d.o3 * es;
                const cuuint64_t dims[3] = {(cuuint64_t)c->nnu, (cuuint64_t)d.nr, (cuuint64_t)d.nz};
                const cuuint64_t strides[2] = {(cuuint64_t)c->nnu * es, (cuuint64_t)c->nnu * d.nr * es};
                const cuuint32_t box[3] = {32u, (cuuint32_t)(kTileCols + 4), 1u};
                const cuuint32_t estr[3] = {1u, 1u, 1u};
                CUresult e = fn(&maps[((size_t)s * c->ncl + q) * 3 + f],
                                es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base,
                                dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (e != CUDA_SUCCESS) return LYD_OK;
            }
    LYD_TRY(dalloc(c, (void **)&c->tmaps, maps.size() * sizeof(CUtensorMap)));
    LYD_CU(c, cudaMemcpyAsync(c->tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                              c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    c->tma_ok = true;
    return LYD_OK;
}

// The staging the advection uses: bulk copies when asked for, or by default with FP32 storage,
// and the maps exist. Measured at 256^2 x 64 (per launch): FP32 storage 0.171 ms with per-lane
// loads, 0.167 ms with bulk copies; FP64 arithmetic at 3 CTAs per SM 0.333 / 0.341 ms (the row
// loads are not what stalls it); FP32 arithmetic over FP64 storage 0.183 / 0.215 ms (the raw
// tile leaves room for 3 CTAs per SM instead of 4).
static int staging_used(const lyd_ctx *c) {
    const int want = c->tune.adv_staging != LYD_STAGING_AUTO
                         ? c->tune.adv_staging
                         : (c->prec == LYD_PREC_FP32 ? LYD_STAGING_TMA : LYD_STAGING_LANES);
    return (want == LYD_STAGING_TMA && c->tma_ok) ? LYD_STAGING_TMA : LYD_STAGING_LANES;
}

const char *lyd_last_error(const lyd_ctx *c) { return c ? c->msg.c_str() : "null context"; }

int lyd_edge_count(int32_t n_r, int32_t n_z) { return (n_z - 2) + 2 * (n_r - 3); }

int lyd_host_alloc(size_t bytes, void **out) {
    if (!out) return LYD_ERR_ARG;
    *out = nullptr;
    return cudaHostAlloc(out, bytes ? bytes : 16, cudaHostAllocPortable) == cudaSuccess ? LYD_OK : LYD_ERR_NOMEM;
}

int lyd_host_free(void *p) {
    if (!p) return LYD_OK;
    return cudaFreeHost(p) == cudaSuccess ? LYD_OK : LYD_ERR_CUDA;
}

int lyd_math_check(int32_t fn, const double *x, double *y, size_t n) {
    if (fn < 0 || fn > 4 || !x || !y) return LYD_ERR_ARG;
    if (n == 0) return LYD_OK;
    double *d = nullptr;
    if (cudaMalloc(&d, 2 * n * sizeof(double)) != cudaSuccess) return LYD_ERR_NOMEM;
    cudaError_t e = cudaMemcpy(d, x, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        launch_math(fn, d, d + n, n, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + n, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? LYD_OK : LYD_ERR_CUDA;
}

int lyd_batch_create(lyd_ctx **out, int32_t ncl, const int32_t *n_r, const int32_t *n_z, int32_t n_nu,
                     const lyd_config *cfg) {
    if (!out || !cfg || !n_r || !n_z) return LYD_ERR_ARG;
    *out = nullptr;
    if (ncl < 1 || n_nu < 4 || n_nu > 256) return LYD_ERR_ARG;
    for (int q = 0; q < ncl; q++) {
        if (n_r[q] < 3 || n_z[q] < 3) return LYD_ERR_ARG;
        if ((long long)n_r[q] * n_z[q] * n_nu >= (1LL << 31)) return LYD_ERR_ARG;   // per-cloud int indices
    }
    if (cfg->precision != LYD_PREC_FP64 && cfg->precision != LYD_PREC_MIXED && cfg->precision != LYD_PREC_FP32)
        return LYD_ERR_ARG;
    if (cfg->flux_method != LYD_FLUX_GLF && cfg->flux_method != LYD_FLUX_HLL) return LYD_ERR_ARG;
    if (cfg->kcore_min < 0 || cfg->kcore_max >= n_nu || cfg->kcore_min > cfg->kcore_max) return LYD_ERR_ARG;
    if (cfg->geometry != LYD_GEOM_CYLINDRICAL && cfg->geometry != LYD_GEOM_CARTESIAN) return LYD_ERR_ARG;
    if (cfg->bc_r_left != LYD_BC_REFLECT && cfg->bc_r_left != LYD_BC_OUTFLOW) return LYD_ERR_ARG;
    if (cfg->geometry == LYD_GEOM_CYLINDRICAL && cfg->bc_r_left != LYD_BC_REFLECT) return LYD_ERR_ARG;
    lyd_ctx *c = new lyd_ctx();
    c->cfg = *cfg;
    c->dev = cfg->device;
    if (cudaSetDevice(c->dev) != cudaSuccess) { delete c; return LYD_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) { delete c; return LYD_ERR_CUDA; }
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev);
    c->nnu = n_nu;
    c->ncl = ncl;
    c->nr.assign(n_r, n_r + ncl);
    c->nz.assign(n_z, n_z + ncl);
    c->have.assign(ncl, 0u);
    c->desc.assign(ncl, CloudDesc{});
    for (int q = 0; q < ncl; q++) {
        CloudDesc &d = c->desc[q];
        const int nr = n_r[q], nz = n_z[q];
        d.o3 = (long long)c->n3; d.oc = (long long)c->ncell;
        d.orf = (long long)c->nrf; d.ozf = (long long)c->nzf;
        d.ocol = (int)c->ncol; d.orow = (int)c->nrow;
        d.orint = (int)c->nrint; d.ozint = (int)c->nzint;
        d.orif = (int)c->nrif; d.ozif = (int)c->nzif;
        d.nr = nr; d.nz = nz;
        d.j_own0 = 0; d.j_own1 = nz;
        d.ctdt = d.dt = d.c_tilde = 1.0;
        c->ncell += (size_t)nr * nz;
        c->n3 += (size_t)nr * nz * n_nu;
        c->nrf += (size_t)(nr + 1) * nz;
        c->nzf += (size_t)nr * (nz + 1);
        c->ncol += nr; c->nrow += nz;
        c->nrint += (size_t)(nr + 1) * 5; c->nzint += (size_t)(nz + 1) * 5;
        c->nrif += nr + 1; c->nzif += nz + 1;
    }
    if (c->nrint >= (1u << 31) || c->nzint >= (1u << 31)) { lyd_destroy(c); return LYD_ERR_ARG; }
    c->prec = cfg->precision;
    c->sprec = c->prec == LYD_PREC_FP32 ? 1 : 0;
    c->ssz = c->sprec == 0 ? sizeof(double) : sizeof(float);
    if (c->prec != LYD_PREC_FP64) {
        c->jscale = cfg->j_scale > 0.0 ? cfg->j_scale : 1e-12;
        c->jeps_s = 1e-30;
        c->heps2_s = 0.0;
    }
    int r = LYD_OK;
    auto A = [&](void **p, size_t b) { if (r == LYD_OK) r = dalloc(c, p, b); };
    for (int s = 0; s < 2; s++)
        for (int q = 0; q < 3; q++) A(&c->set[s][q], c->n3 * c->ssz);
    A(&c->Hv, c->n3 * c->ssz);
    A((void **)&c->phi_inv, c->ncell * 8);
    for (int q = 0; q < CF_N; q++) A((void **)&c->cellf[q], c->ncell * 8);
    A((void **)&c->u_r_star, c->nrf * 8);
    A((void **)&c->u_Z_star, c->nzf * 8);
    A((void **)&c->dV, c->ncell * 8); A((void **)&c->inv_dV, c->ncell * 8);
    A((void **)&c->A_r, c->nrf * 8); A((void **)&c->A_Z, c->nzf * 8);
    A((void **)&c->inv_r_cell, c->ncol * 8); A((void **)&c->rCoM, c->ncol * 8); A((void **)&c->ZCoM, c->nrow * 8);
    A((void **)&c->rint, c->nrint * 8); A((void **)&c->zint, c->nzint * 8);
    A((void **)&c->r_if, c->nrif * 8); A((void **)&c->Z_if, c->nzif * 8);
    A((void **)&c->nu, (c->nnu + 1) * 8); A((void **)&c->nuC, c->nnu * 8); A((void **)&c->dnu, c->nnu * 8);
    A((void **)&c->inv_dnu, c->nnu * 8); A((void **)&c->inv_nuC, c->nnu * 8);
    A((void **)&c->cl, (size_t)ncl * sizeof(CloudDesc));
    A((void **)&c->kwin, (size_t)2 * ncl * sizeof(int));
    A((void **)&c->step_ctr, 2 * sizeof(int));
    A((void **)&c->red_cols, (size_t)ncl * (c->nnu + kExtraCols) * sizeof(double));
    A((void **)&c->red_cnt, (size_t)ncl * sizeof(int));
    A((void **)&c->last, (size_t)7 * ncl * sizeof(double));
    A((void **)&c->err, sizeof(int));
    A((void **)&c->small, 512 * 8);
    A((void **)&c->bar, 2 * sizeof(unsigned));
    if (cfg->keep_freq_factors)
        for (int q = 0; q < 3; q++) A((void **)&c->Ff[q], c->n3 * 8);
    if (r == LYD_OK) r = build_work(c);
    if (r == LYD_OK) r = encode_tmaps(c);
    if (r != LYD_OK) {
        lyd_destroy(c);
        return r;
    }
    for (int q = 0; q < 8; q++) cudaEventCreate(&c->ev[q]);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) { lyd_destroy(c); return LYD_ERR_CUDA; }
    *out = c;
    return LYD_OK;
}

int lyd_create(lyd_ctx **out, const lyd_dims *d, const lyd_config *cfg) {
    if (!out || !d || !cfg) return LYD_ERR_ARG;
    *out = nullptr;
    if (d->n_nu < 4 || d->n_nu > 256 || d->n_r < 3 || d->n_z < 3) return LYD_ERR_ARG;
    int32_t nr = d->n_r, nz = d->n_z;
    return lyd_batch_create(out, 1, &nr, &nz, d->n_nu, cfg);
}

int lyd_destroy(lyd_ctx *c) {
    if (!c) return LYD_OK;
    cudaSetDevice(c->dev);
    if (c->st) cudaStreamSynchronize(c->st);
    drop_graph(c);
    for (int s = 0; s < 2; s++)
        for (int q = 0; q < 3; q++) cudaFree(c->set[s][q]);
    cudaFree(c->tmaps);
    void *ps[] = {c->Hv, c->phi, c->phi_inv, c->aF, c->Ff[0], c->Ff[1], c->Ff[2], c->u_r_star, c->u_Z_star, c->dV,
                  c->inv_dV, c->A_r, c->A_Z, c->inv_r_cell, c->rCoM, c->ZCoM, c->rint, c->zint, c->r_if, c->Z_if,
                  c->nu, c->nuC, c->dnu, c->inv_dnu, c->inv_nuC, c->partials, c->kwin, c->hist, c->step_ctr,
                  c->last, c->err, c->lut, c->stage, c->small, c->cl, c->tiles, c->items, c->adj_ws,
                  c->red_cols, c->red_cnt, c->bar, c->hin, c->part_chk, c->kwin_chk, c->ctiles};
    for (void *p : ps) cudaFree(p);
    for (int q = 0; q < CF_N; q++) cudaFree(c->cellf[q]);
    cudaFree(c->dust_F);
    cudaFree(c->dd_cl);
    for (int q = 0; q < 8; q++)
        if (c->ev[q]) cudaEventDestroy(c->ev[q]);
    for (cudaEvent_t e : c->hs_ev)
        if (e) cudaEventDestroy(e);
    if (c->st_up) cudaStreamDestroy(c->st_up);
    if (c->st_dn) cudaStreamDestroy(c->st_dn);
    if (c->st_fq) cudaStreamDestroy(c->st_fq);
    for (cudaEvent_t e : c->adj_ev)
        if (e) cudaEventDestroy(e);
    if (c->st_rec) cudaStreamDestroy(c->st_rec);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return LYD_OK;
}

int lyd_batch_info(lyd_ctx *c, int32_t *ncl, int64_t *cell_bins) {
    if (!c) return LYD_ERR_ARG;
    if (ncl) *ncl = c->ncl;
    if (cell_bins) *cell_bins = (int64_t)c->n3;
    return LYD_OK;
}

int lyd_get_stream(lyd_ctx *c, void **s) {
    if (!c || !s) return LYD_ERR_ARG;
    *s = (void *)c->st;
    return LYD_OK;
}

int lyd_synchronize(lyd_ctx *c) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    return check_err(c);
}

int lyd_set_tuning(lyd_ctx *c, const lyd_tuning *t) {
    if (!c || !t) return LYD_ERR_ARG;
    if (t->rows_per_tile < 4 || t->rows_per_tile > 64) return fail(c, LYD_ERR_ARG, "rows_per_tile outside 4..64");
    if (t->cells_per_block != 0 && (t->cells_per_block < 8 || t->cells_per_block > 1024))
        return fail(c, LYD_ERR_ARG, "cells_per_block outside 8..1024");
    if (t->solver != SOLVER_PCR && t->solver != SOLVER_THOMAS) return fail(c, LYD_ERR_ARG, "unknown solver");
    if (t->adv_ctas_per_sm != 0 && (t->adv_ctas_per_sm < 2 || t->adv_ctas_per_sm > 4))
        return fail(c, LYD_ERR_ARG, "adv_ctas_per_sm outside 2..4");
    if (t->adv_staging < LYD_STAGING_AUTO || t->adv_staging > LYD_STAGING_TMA)
        return fail(c, LYD_ERR_ARG, "unknown adv_staging");
    cudaSetDevice(c->dev);
    LYD_CU(c, cudaStreamSynchronize(c->st));
    c->tune = *t;
    return build_work(c);
}

int lyd_get_tuning(lyd_ctx *c, lyd_tuning *t) {
    if (!c || !t) return LYD_ERR_ARG;
    *t = c->tune;
    if (t->cells_per_block == 0) t->cells_per_block = -cells_per_block(c);   // negative: chosen automatically
    t->adv_ctas_per_sm = adv_ctas_per_sm(c->prec, t->adv_ctas_per_sm);
    t->adv_staging = staging_used(c);
    return LYD_OK;
}

static int h2d(lyd_ctx *c, void *dst, const double *src, size_t n) {
    if (!src) return fail(c, LYD_ERR_ARG, "null host pointer");
    LYD_CU(c, cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyHostToDevice, c->st));
    return LYD_OK;
}

static int bad_cloud(lyd_ctx *c, int q) {
    return (q < 0 || q >= c->ncl) ? fail(c, LYD_ERR_ARG, "cloud index out of range") : LYD_OK;
}

int lyd_set_geometry_cloud(lyd_ctx *c, int32_t q, const lyd_geometry *g) {
    if (!c || !g) return LYD_ERR_ARG;
    LYD_TRY(bad_cloud(c, q));
    cudaSetDevice(c->dev);
    const CloudDesc &d = c->desc[q];
    const int nr = d.nr, nz = d.nz;
    const size_t nc = (size_t)nr * nz;
    LYD_TRY(h2d(c, c->dV + d.oc, g->dV, nc));
    LYD_TRY(h2d(c, c->inv_dV + d.oc, g->inv_dV, nc));
    LYD_TRY(h2d(c, c->A_r + d.orf, g->A_r, (size_t)(nr + 1) * nz));
    LYD_TRY(h2d(c, c->A_Z + d.ozf, g->A_Z, (size_t)nr * (nz + 1)));
    if (c->cfg.geometry == LYD_GEOM_CARTESIAN)   // no K_phiphi source on a Cartesian grid
        LYD_CU(c, cudaMemsetAsync(c->inv_r_cell + d.ocol, 0, (size_t)nr * 8, c->st));
    else
        LYD_TRY(h2d(c, c->inv_r_cell + d.ocol, g->inv_r_cell, nr));
    LYD_TRY(h2d(c, c->rCoM + d.ocol, g->rCoM, nr));
    LYD_TRY(h2d(c, c->ZCoM + d.orow, g->ZCoM, nz));
    LYD_TRY(h2d(c, c->r_if + d.orif, g->r, nr + 1));
    LYD_TRY(h2d(c, c->Z_if + d.ozif, g->Z, nz + 1));
    // PLM intervals per face: face 0 = inner boundary, face n = outer boundary, face f in
    // between uses the cell arrays at f-1 (src/AdvectJandH.jl:628-638, 775-779, 884-887).
    auto pack = [](int n, const double *L, const double *R, const double *a, const double *b, const double *cc,
                   const double *bnd, std::vector<double> &o) {
        o.assign((size_t)(n + 1) * 5, 0.0);
        for (int t = 0; t < 5; t++) o[t] = bnd[t];
        for (int f = 1; f < n; f++) {
            o[5 * f + 0] = L[f - 1]; o[5 * f + 1] = R[f - 1]; o[5 * f + 2] = a[f - 1];
            o[5 * f + 3] = b[f - 1]; o[5 * f + 4] = cc[f - 1];
        }
        for (int t = 0; t < 5; t++) o[5 * n + t] = bnd[5 + t];
    };
    if (!g->dr_L || !g->dr_R || !g->inv_dr_i_im1 || !g->inv_dr_ip1_i || !g->inv_dr_ip2_ip1 || !g->dZ_L ||
        !g->dZ_R || !g->inv_dZ_j_jm1 || !g->inv_dZ_jp1_j || !g->inv_dZ_jp2_jp1)
        return fail(c, LYD_ERR_ARG, "missing interval arrays");
    std::vector<double> pr, pz;
    pack(nr, g->dr_L, g->dr_R, g->inv_dr_i_im1, g->inv_dr_ip1_i, g->inv_dr_ip2_ip1, g->dr_bnd, pr);
    pack(nz, g->dZ_L, g->dZ_R, g->inv_dZ_j_jm1, g->inv_dZ_jp1_j, g->inv_dZ_jp2_jp1, g->dZ_bnd, pz);
    LYD_CU(c, cudaMemcpyAsync(c->rint + d.orint, pr.data(), pr.size() * 8, cudaMemcpyHostToDevice, c->st));
    LYD_CU(c, cudaMemcpyAsync(c->zint + d.ozint, pz.data(), pz.size() * 8, cudaMemcpyHostToDevice, c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    c->have[q] |= BIT_GEOM;
    return LYD_OK;
}

int lyd_set_geometry(lyd_ctx *c, const lyd_geometry *g) {
    if (!c || !g) return LYD_ERR_ARG;
    if (c->ncl != 1) return fail(c, LYD_ERR_STATE, "a batch context takes lyd_set_geometry_cloud");
    return lyd_set_geometry_cloud(c, 0, g);
}

int lyd_set_freq_grid(lyd_ctx *c, const lyd_freq_grid *f) {
    if (!c || !f) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(h2d(c, c->nu, f->nu, c->nnu + 1));
    LYD_TRY(h2d(c, c->nuC, f->nuC, c->nnu));
    LYD_TRY(h2d(c, c->dnu, f->dnu, c->nnu));
    LYD_TRY(h2d(c, c->inv_dnu, f->inv_dnu, c->nnu));
    LYD_TRY(h2d(c, c->inv_nuC, f->inv_nuC, c->nnu));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    c->freq_set = true;
    c->active_valid = false;
    return LYD_OK;
}

// Make the old set a real copy before one of J/H or J_old/H_old is overwritten alone.
static int materialize_old(lyd_ctx *c) {
    if (!c->old_alias) return LYD_OK;
    for (int q = 0; q < 3; q++)
        LYD_CU(c, cudaMemcpyAsync(c->set[1 - c->cur][q], c->set[c->cur][q], c->n3 * c->ssz, cudaMemcpyDeviceToDevice,
                                  c->st));
    c->old_alias = false;
    return LYD_OK;
}

static int upload3(lyd_ctx *c, void *dst, const double *host, size_t n, double scale) {
    LYD_TRY(ensure_stage(c, n));
    LYD_CU(c, cudaMemcpyAsync(c->stage, host, n * 8, cudaMemcpyHostToDevice, c->st));
    launch_convert_in(c->sprec, c->stage, dst, n, scale, c->st);
    LYD_CU(c, cudaGetLastError());
    return LYD_OK;
}

// One field of cloud q (q < 0: every cloud, concatenated).
static int upload_field(lyd_ctx *c, int q, int32_t field, const double *host, size_t count) {
    if (!host) return fail(c, LYD_ERR_ARG, "null host pointer");
    cudaSetDevice(c->dev);
    const bool one = q >= 0;
    const CloudDesc d0{};
    const CloudDesc &d = one ? c->desc[q] : d0;
    const size_t n3 = one ? (size_t)d.nr * d.nz * c->nnu : c->n3;
    const size_t nc = one ? (size_t)d.nr * d.nz : c->ncell;
    auto mark = [&](unsigned bit) {
        if (one) c->have[q] |= bit;
        else set_all(c, bit);
    };
    if (field <= LYD_F_H_Z_OLD && field >= 0) {
        if (count != n3) return fail(c, LYD_ERR_ARG, "wrong element count for a (n_nu, n_r, n_z) field");
        LYD_TRY(materialize_old(c));
        int k = (field == LYD_F_J || field == LYD_F_J_OLD) ? 0 : ((field == LYD_F_H_R || field == LYD_F_H_R_OLD) ? 1 : 2);
        bool old = field == LYD_F_J_OLD || field == LYD_F_H_R_OLD || field == LYD_F_H_Z_OLD;
        void *dst = old ? c->set[1 - c->cur][k] : c->set[c->cur][k];
        LYD_TRY(upload3(c, at(dst, d.o3, c->ssz), host, n3, c->jscale));
        if (k == 0 && !old) c->active_valid = false;
    } else if (field == LYD_F_HVOIGT) {
        if (count != n3) return fail(c, LYD_ERR_ARG, "wrong element count for H_voigt");
        LYD_TRY(upload3(c, at(c->Hv, d.o3, c->ssz), host, n3, 1.0));
        mark(BIT_HV);
        c->hv_from_T = false;
        c->phi_inv_ready = false;
    } else if (field == LYD_F_PHI_NU || field == LYD_F_ALPHA_F) {
        if (count != n3) return fail(c, LYD_ERR_ARG, "wrong element count");
        void **p = field == LYD_F_PHI_NU ? &c->phi : &c->aF;
        if (!*p) LYD_TRY(dalloc(c, p, c->n3 * c->ssz));
        LYD_TRY(upload3(c, at(*p, d.o3, c->ssz), host, n3, 1.0));
        mark(field == LYD_F_PHI_NU ? BIT_PHI : BIT_AF);
    } else if (field >= LYD_F_ALPHA && field <= LYD_F_E_LYA) {
        if (count != nc) return fail(c, LYD_ERR_ARG, "wrong element count for a per-cell field");
        if (field == LYD_F_UR_OVER_R && c->cfg.geometry == LYD_GEOM_CARTESIAN)
            return fail(c, LYD_ERR_ARG, "a Cartesian grid has no u_r / r term");
        int k = field - LYD_F_ALPHA;
        LYD_TRY(h2d(c, c->cellf[k] + d.oc, host, nc));
        mark(1u << k);
    } else if (field == LYD_F_U_R_STAR) {
        size_t n = one ? (size_t)(d.nr + 1) * d.nz : c->nrf;
        if (count != n) return fail(c, LYD_ERR_ARG, "wrong element count for u_r_star");
        LYD_TRY(h2d(c, c->u_r_star + d.orf, host, n));
    } else if (field == LYD_F_U_Z_STAR) {
        size_t n = one ? (size_t)d.nr * (d.nz + 1) : c->nzf;
        if (count != n) return fail(c, LYD_ERR_ARG, "wrong element count for u_Z_star");
        LYD_TRY(h2d(c, c->u_Z_star + d.ozf, host, n));
    } else {
        return fail(c, LYD_ERR_ARG, "unknown field");
    }
    LYD_CU(c, cudaStreamSynchronize(c->st));
    return LYD_OK;
}

static int download_field(lyd_ctx *c, int q, int32_t field, double *host, size_t count) {
    if (!host) return fail(c, LYD_ERR_ARG, "null host pointer");
    cudaSetDevice(c->dev);
    const bool one = q >= 0;
    const CloudDesc d0{};
    const CloudDesc &d = one ? c->desc[q] : d0;
    const size_t n3 = one ? (size_t)d.nr * d.nz * c->nnu : c->n3;
    const size_t nc = one ? (size_t)d.nr * d.nz : c->ncell;
    const void *src = nullptr;
    size_t n = 0;
    double scale = 1.0;
    bool is3 = false;
    if (field <= LYD_F_H_Z_OLD && field >= 0) {
        int k = (field == LYD_F_J || field == LYD_F_J_OLD) ? 0 : ((field == LYD_F_H_R || field == LYD_F_H_R_OLD) ? 1 : 2);
        bool old = field == LYD_F_J_OLD || field == LYD_F_H_R_OLD || field == LYD_F_H_Z_OLD;
        src = old ? Jold(c, k) : Jc(c, k);
        n = n3; scale = c->jscale; is3 = true;
    } else if (field == LYD_F_HVOIGT) {
        src = c->Hv; n = n3; is3 = true;
    } else if (field == LYD_F_PHI_NU || field == LYD_F_ALPHA_F) {
        src = field == LYD_F_PHI_NU ? c->phi : c->aF;
        if (!src) return fail(c, LYD_ERR_STATE, "field is derived on the device and was never uploaded");
        n = n3; is3 = true;
    } else if (field >= LYD_F_ALPHA && field <= LYD_F_E_LYA) {
        src = c->cellf[field - LYD_F_ALPHA] + d.oc; n = nc;
    } else if (field == LYD_F_U_R_STAR) {
        src = c->u_r_star + d.orf; n = one ? (size_t)(d.nr + 1) * d.nz : c->nrf;
    } else if (field == LYD_F_U_Z_STAR) {
        src = c->u_Z_star + d.ozf; n = one ? (size_t)d.nr * (d.nz + 1) : c->nzf;
    } else {
        return fail(c, LYD_ERR_ARG, "unknown field");
    }
    if (count != n) return fail(c, LYD_ERR_ARG, "wrong element count");
    if (is3) {
        LYD_TRY(ensure_stage(c, n));
        launch_convert_out(c->sprec, at(const_cast<void *>(src), d.o3, c->ssz), c->stage, n, scale, c->st);
        LYD_CU(c, cudaGetLastError());
        LYD_CU(c, cudaMemcpyAsync(host, c->stage, n * 8, cudaMemcpyDeviceToHost, c->st));
    } else {
        LYD_CU(c, cudaMemcpyAsync(host, src, n * 8, cudaMemcpyDeviceToHost, c->st));
    }
    return check_err(c);
}

int lyd_upload(lyd_ctx *c, int32_t field, const double *host, size_t count) {
    if (!c) return LYD_ERR_ARG;
    return upload_field(c, -1, field, host, count);
}
int lyd_download(lyd_ctx *c, int32_t field, double *host, size_t count) {
    if (!c) return LYD_ERR_ARG;
    return download_field(c, -1, field, host, count);
}
int lyd_upload_cloud(lyd_ctx *c, int32_t q, int32_t field, const double *host, size_t count) {
    if (!c) return LYD_ERR_ARG;
    LYD_TRY(bad_cloud(c, q));
    return upload_field(c, q, field, host, count);
}
int lyd_download_cloud(lyd_ctx *c, int32_t q, int32_t field, double *host, size_t count) {
    if (!c) return LYD_ERR_ARG;
    LYD_TRY(bad_cloud(c, q));
    return download_field(c, q, field, host, count);
}

// ---- argument blocks -------------------------------------------------------------------------
template <typename S>
static void fill_adv(lyd_ctx *c, AdvArgs<S> &a, int in_set, int out_set) {
    memset(&a, 0, sizeof(a));
    a.J = (const S *)c->set[in_set][0]; a.Hr = (const S *)c->set[in_set][1]; a.HZ = (const S *)c->set[in_set][2];
    a.Jo = (S *)c->set[out_set][0]; a.Hro = (S *)c->set[out_set][1]; a.HZo = (S *)c->set[out_set][2];
    a.aF = c->aF ? (const S *)c->aF : nullptr;
    a.Hv = (const S *)c->Hv;
    a.alpha = c->cellf[CF_ALPHA];
    a.alpha_cF = any_have(c, 1u << CF_ALPHA_CF) ? c->cellf[CF_ALPHA_CF] : nullptr;
    a.A_r = c->A_r; a.A_Z = c->A_Z; a.inv_dV = c->inv_dV; a.inv_r_cell = c->inv_r_cell;
    a.rint = c->rint; a.zint = c->zint;
    a.u_r_star = c->u_r_star; a.u_Z_star = c->u_Z_star;
    a.dur_dr = c->cellf[CF_DUR_DR]; a.dur_dZ = c->cellf[CF_DUR_DZ]; a.duZ_dr = c->cellf[CF_DUZ_DR];
    a.duZ_dZ = c->cellf[CF_DUZ_DZ]; a.ur_over_r = c->cellf[CF_UR_OVER_R];
    a.kwin = c->kwin;
    a.cl = c->cl;
    a.tiles = c->tiles;
    a.rows = c->tune.rows_per_tile;
    a.nnu = c->nnu;
    a.jeps = c->jeps_s; a.heps2 = c->heps2_s;
    a.err = c->err;
    a.tmaps = staging_used(c) == LYD_STAGING_TMA ? c->tmaps + (size_t)in_set * c->ncl * 3 * kTensorMapBytes : nullptr;
}

template <typename S>
static void fill_freq(lyd_ctx *c, FreqArgs<S> &a, const void *Jin, const void *Hrin, const void *HZin, const void *Jo,
                      void *Jout, void *Hrout, void *HZout) {
    memset(&a, 0, sizeof(a));
    a.Jin = (const S *)Jin; a.Hrin = (const S *)Hrin; a.HZin = (const S *)HZin; a.Jold = (const S *)Jo;
    a.Jout = (S *)Jout; a.Hrout = (S *)Hrout; a.HZout = (S *)HZout;
    a.Hv = (const S *)c->Hv;
    a.phi = c->phi ? (const S *)c->phi : nullptr;
    a.phi_inv = c->phi_inv; a.phi_kmin = c->phi_kmin; a.phi_kmax = c->phi_kmax;
    a.aF = c->aF ? (const S *)c->aF : nullptr;
    a.alpha = c->cellf[CF_ALPHA]; a.alpha_c = c->cellf[CF_ALPHA_C];
    a.alpha_cF = any_have(c, 1u << CF_ALPHA_CF) ? c->cellf[CF_ALPHA_CF] : nullptr;
    a.pd = c->cellf[CF_PD]; a.js = c->cellf[CF_JS]; a.T = c->cellf[CF_T];
    a.dur_dr = c->cellf[CF_DUR_DR]; a.dur_dZ = c->cellf[CF_DUR_DZ]; a.duZ_dr = c->cellf[CF_DUZ_DR];
    a.duZ_dZ = c->cellf[CF_DUZ_DZ]; a.ur_over_r = c->cellf[CF_UR_OVER_R];
    a.nu = c->nu; a.nuC = c->nuC; a.dnu = c->dnu; a.inv_dnu = c->inv_dnu; a.inv_nuC = c->inv_nuC;
    a.dV = c->dV; a.A_r = c->A_r; a.A_Z = c->A_Z; a.rCoM = c->rCoM; a.ZCoM = c->ZCoM;
    a.cl = c->cl;
    a.items = c->items;
    a.alpha_floor = c->cfg.alpha_floor;
    a.jeps = c->jeps_s; a.heps2 = c->heps2_s; a.j_scale = c->jscale;
    a.recoil = c->cfg.recoil;
    a.partials = c->partials; a.err = c->err;
    a.nnu = c->nnu;
    a.solver = c->tune.solver;
}

static int need_inputs(lyd_ctx *c, bool emission, bool freq) {
    if (!all_have(c, BIT_GEOM)) return fail(c, LYD_ERR_STATE, "geometry not set (lyd_set_geometry)");
    if (!c->freq_set) return fail(c, LYD_ERR_STATE, "frequency grid not set (lyd_set_freq_grid)");
    if ((emission || freq) && !all_have(c, BIT_HV)) return fail(c, LYD_ERR_STATE, "H_voigt not set");
    if (c->phi && !all_have(c, BIT_PHI))
        return fail(c, LYD_ERR_STATE, "phi_nu was uploaded for some clouds only");
    if (c->aF && !all_have(c, BIT_AF))
        return fail(c, LYD_ERR_STATE, "alpha_F was uploaded for some clouds only");
    if (emission && !c->phi && !c->phi_inv_ready)
        return fail(c, LYD_ERR_STATE, "phi_nu not set (upload it or call lyd_update_phi_nu)");
    if (freq && !all_have(c, 1u << CF_T)) return fail(c, LYD_ERR_STATE, "temperature T not uploaded");
    return LYD_OK;
}

static RedArgs red_args(lyd_ctx *c, int parts) {
    RedArgs r;
    memset(&r, 0, sizeof(r));
    r.partials = c->partials; r.nblocks = c->nitems; r.nnu = c->nnu; r.nclouds = c->ncl; r.parts = parts;
    r.kcore_min = c->cfg.kcore_min; r.kcore_max = c->cfg.kcore_max;
    r.j_scale = c->jscale; r.cl = c->cl; r.kwin = c->kwin; r.last = c->last;
    r.colsum = c->red_cols; r.cnt = c->red_cnt;
    return r;
}

static int run_find_active(lyd_ctx *c) {
    LYD_TRY(sync_desc(c));
    launch_find_active(c->sprec, Jc(c, 0), c->nnu, c->dnu, c->dV, c->cl, c->items, c->nitems, c->jeps_s, c->partials,
                       c->st);
    launch_reduce(red_args(c, PART_ACTIVE), c->st);
    LYD_CU(c, cudaGetLastError());
    c->active_valid = true;
    return LYD_OK;
}

int lyd_find_active_bins(lyd_ctx *c, int32_t *kmin, int32_t *kmax) {
    if (!c || !kmin || !kmax) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(need_inputs(c, false, false));
    LYD_TRY(run_find_active(c));
    std::vector<int> h((size_t)2 * c->ncl);
    LYD_CU(c, cudaMemcpyAsync(h.data(), c->kwin, h.size() * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    LYD_TRY(check_err(c));
    for (int q = 0; q < c->ncl; q++) {
        kmin[q] = h[2 * q];
        kmax[q] = h[2 * q + 1];
    }
    return LYD_OK;
}

static int check_bcs(lyd_ctx *c, int l, int r, int b, int t) {
    auto ok = [](int v) { return v == LYD_BC_REFLECT || v == LYD_BC_OUTFLOW; };
    if (c->cfg.geometry == LYD_GEOM_CYLINDRICAL && l != LYD_BC_REFLECT)
        return fail(c, LYD_ERR_ARG, "the r = 0 boundary of a cylindrical grid is always reflecting");
    if (!ok(l) || !ok(r) || !ok(b) || !ok(t)) return fail(c, LYD_ERR_ARG, "unknown boundary condition");
    return LYD_OK;
}

// Parameters of every cloud for the per-phase calls (one c~, dt and boundary set for all).
static void params_all(lyd_ctx *c, double ct, double dt, double ctdt) {
    for (CloudDesc &d : c->desc) {
        d.c_tilde = ct; d.dt = dt; d.ctdt = ctdt;
    }
}
static void bcs_all(lyd_ctx *c, int bcl, int bcr, int bzb, int bzt) {
    for (CloudDesc &d : c->desc) {
        d.bc_r_left = bcl; d.bc_r_right = bcr; d.bc_z_bot = bzb; d.bc_z_top = bzt;
    }
}

static int do_advect(lyd_ctx *c) {
    if (!c->active_valid) LYD_TRY(run_find_active(c));
    LYD_TRY(sync_desc(c));
    int in = c->cur, out = 1 - c->cur;
    if (c->sprec == 0) {
        AdvArgs<double> a;
        fill_adv<double>(c, a, in, out);
        launch_advect(c->prec, c->cfg.flux_method, &a, c->ntiles, c->tune.adv_ctas_per_sm, c->st);
    } else {
        AdvArgs<float> a;
        fill_adv<float>(c, a, in, out);
        launch_advect(c->prec, c->cfg.flux_method, &a, c->ntiles, c->tune.adv_ctas_per_sm, c->st);
    }
    LYD_CU(c, cudaGetLastError());
    c->cur = out;
    c->old_alias = true;
    c->active_valid = false;
    return LYD_OK;
}

int lyd_advect(lyd_ctx *c, double ctdt, int32_t bl, int32_t br, int32_t bb, int32_t bt) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(check_bcs(c, bl, br, bb, bt));
    LYD_TRY(need_inputs(c, false, false));
    if (!(ctdt > 0.0)) return fail(c, LYD_ERR_ARG, "c~ dt must be positive");
    for (CloudDesc &d : c->desc) d.ctdt = ctdt;
    bcs_all(c, bl, br, bb, bt);
    return do_advect(c);
}

// AdvectJandH! with its own bin range and J_old rule (src/AdvectJandH.jl:2227-2464): the
// stellar/IR bands and any caller that does not want FindActiveBins. J_old becomes the new J
// when update_jold is set and is otherwise left as it was; H_old is never touched.
int lyd_advect_jh(lyd_ctx *c, double ctdt, int32_t kmin, int32_t kmax, int32_t update_jold, int32_t bl, int32_t br,
                  int32_t bb, int32_t bt) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(check_bcs(c, bl, br, bb, bt));
    LYD_TRY(need_inputs(c, false, false));
    if (!(ctdt > 0.0)) return fail(c, LYD_ERR_ARG, "c~ dt must be positive");
    if (kmin < 0 || kmax >= c->nnu || kmin > kmax) return fail(c, LYD_ERR_ARG, "bad bin range");
    for (CloudDesc &d : c->desc) d.ctdt = ctdt;
    bcs_all(c, bl, br, bb, bt);
    LYD_TRY(sync_desc(c));
    const bool alias = c->old_alias;
    const size_t bytes = c->n3 * c->ssz;
    void *saved = nullptr;
    if (!alias) {
        // the old set is about to receive the advected state: keep J_old and H_old
        LYD_TRY(dalloc(c, &saved, 3 * bytes));
        for (int q = 0; q < 3; q++)
            LYD_CU(c, cudaMemcpyAsync(at(saved, q * c->n3, c->ssz), c->set[1 - c->cur][q], bytes,
                                      cudaMemcpyDeviceToDevice, c->st));
    }
    std::vector<int> w((size_t)2 * c->ncl);
    for (int q = 0; q < c->ncl; q++) { w[2 * q] = kmin; w[2 * q + 1] = kmax; }
    LYD_CU(c, cudaMemcpyAsync(c->kwin, w.data(), w.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
    const int in = c->cur, out = 1 - c->cur;
    if (c->sprec == 0) {
        AdvArgs<double> a;
        fill_adv<double>(c, a, in, out);
        launch_advect(c->prec, c->cfg.flux_method, &a, c->ntiles, c->tune.adv_ctas_per_sm, c->st);
    } else {
        AdvArgs<float> a;
        fill_adv<float>(c, a, in, out);
        launch_advect(c->prec, c->cfg.flux_method, &a, c->ntiles, c->tune.adv_ctas_per_sm, c->st);
    }
    cudaError_t e = cudaGetLastError();
    c->cur = out;
    // the set `in` now holds the state before the advection: make it J_old / H_old
    if (e == cudaSuccess && saved)
        for (int q = 0; q < 3 && e == cudaSuccess; q++)
            e = cudaMemcpyAsync(c->set[in][q], at(saved, q * c->n3, c->ssz), bytes, cudaMemcpyDeviceToDevice, c->st);
    if (e == cudaSuccess && update_jold)
        e = cudaMemcpyAsync(c->set[in][0], c->set[out][0], bytes, cudaMemcpyDeviceToDevice, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(saved);
    if (e != cudaSuccess) return fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
    c->old_alias = false;
    c->active_valid = false;
    return LYD_OK;
}

template <typename S>
static int freq_call(lyd_ctx *c, bool emission, bool freq, int update_ff, int parts) {
    LYD_TRY(sync_desc(c));
    FreqArgs<S> a;
    fill_freq<S>(c, a, Jc(c, 0), Jc(c, 1), Jc(c, 2), Jold(c, 0), Jc(c, 0), Jc(c, 1), Jc(c, 2));
    a.do_emission = emission; a.do_freq = freq; a.update_ff = update_ff;
    a.dru_r = c->cellf[CF_DRU_R]; a.dru_Z = c->cellf[CF_DRU_Z];
    if (c->cfg.keep_freq_factors) { a.Fkp = c->Ff[0]; a.Fk = c->Ff[1]; a.Fkm = c->Ff[2]; }
    a.parts = parts;
    launch_freq(c->prec, &a, c->nnu, c->nitems, c->st);
    LYD_CU(c, cudaGetLastError());
    return LYD_OK;
}

int lyd_emission_absorption(lyd_ctx *c, double ct, double dt) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(need_inputs(c, true, false));
    if (!(ct > 0.0) || !(dt > 0.0)) return fail(c, LYD_ERR_ARG, "c~ and dt must be positive");
    params_all(c, ct, dt, ct * dt);
    int r = c->sprec == 0 ? freq_call<double>(c, true, false, 1, 0) : freq_call<float>(c, true, false, 1, 0);
    if (r != LYD_OK) return r;
    c->old_alias = true;
    c->active_valid = false;
    return LYD_OK;
}

int lyd_frequency_update(lyd_ctx *c, double ctdt, int32_t update_ff) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(need_inputs(c, false, true));
    if (!(ctdt > 0.0)) return fail(c, LYD_ERR_ARG, "c~ dt must be positive");
    if (!update_ff && !(c->cfg.keep_freq_factors && c->ff_valid))
        return fail(c, LYD_ERR_STATE, "update_freq_factors = 0 needs keep_freq_factors and a previous update");
    for (CloudDesc &d : c->desc) d.ctdt = ctdt;
    int uf = update_ff ? 1 : 0;
    int r = c->sprec == 0 ? freq_call<double>(c, false, true, uf, PART_ACTIVE)
                         : freq_call<float>(c, false, true, uf, PART_ACTIVE);
    if (r != LYD_OK) return r;
    launch_reduce(red_args(c, PART_ACTIVE), c->st);
    LYD_CU(c, cudaGetLastError());
    if (update_ff && c->cfg.keep_freq_factors) c->ff_valid = true;
    c->old_alias = true;
    c->active_valid = true;
    return LYD_OK;
}

int lyd_update_J_and_H(lyd_ctx *c, double dt, double ct, int32_t update_ff, int32_t bl, int32_t br, int32_t bb,
                       int32_t bt) {
    if (!c) return LYD_ERR_ARG;
    double ctdt = ct * dt;
    LYD_TRY(lyd_advect(c, ctdt, bl, br, bb, bt));
    return lyd_frequency_update(c, ctdt, update_ff);
}

int lyd_reset_dru(lyd_ctx *c) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_R], 0, c->ncell * 8, c->st));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_Z], 0, c->ncell * 8, c->st));
    return LYD_OK;
}

static int single_cloud(lyd_ctx *c, const char *what) {
    if (c->ncl != 1)
        return fail(c, LYD_ERR_STATE, std::string(what) + " acts on a single-cloud context; a batch reports it per cloud");
    return LYD_OK;
}

// Update_f_Lya_MF_L_Lya!, src/ConstantsAndFunctions.jl:588-674, and (g_r != nullptr, host
// arrays) its gravity variant, :691-804.
static int force_multiplier(lyd_ctx *c, double dt, double zc, int32_t bc_z_bot, const double *g_r,
                            const double *g_Z, double *out) {
    LYD_TRY(single_cloud(c, "lyd_force_multiplier"));
    cudaSetDevice(c->dev);
    if (!all_have(c, BIT_GEOM)) return fail(c, LYD_ERR_STATE, "geometry not set");
    if (!(dt > 0.0)) return fail(c, LYD_ERR_ARG, "dt must be positive");
    const int nr = c->nr[0], nz = c->nz[0];
    const int nb = std::min(c->nitems, 4 * c->sms);
    double *dg = nullptr;
    if (g_r) {
        LYD_TRY(dalloc(c, (void **)&dg, 2 * c->ncell * 8));
        int r = h2d(c, dg, g_r, c->ncell);
        if (r == LYD_OK) r = h2d(c, dg + c->ncell, g_Z, c->ncell);
        if (r != LYD_OK) { cudaFree(dg); return r; }
    }
    launch_mf(c->cellf[CF_DRU_R], c->cellf[CF_DRU_Z], c->cellf[CF_F_R], c->cellf[CF_F_Z], c->cellf[CF_JS], c->dV,
              c->rCoM, c->ZCoM, nr, nz, dt, zc, dg, dg ? dg + c->ncell : nullptr, c->partials, nb, c->st);
    launch_column_sums(c->partials, 5, nb, c->small, c->st);
    double h[5];
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, c->small, sizeof(h), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(dg);
    if (e != cudaSuccess) return fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
    LYD_TRY(check_err(c));
    set_all(c, (1u << CF_F_R) | (1u << CF_F_Z));
    // normalisation, src/ConstantsAndFunctions.jl:652-673 / 780-795
    double MF = h[0], net = h[1], outw = h[2], L = h[3], anti = h[4];
    if (L > 0.0) {
        double k = 1.0 / (L / kC);
        MF *= k; net *= k; outw *= k; anti *= k;
    } else {
        MF = net = outw = anti = 0.0;
    }
    double Ltot = (bc_z_bot == LYD_BC_REFLECT) ? 2.0 * L : L;
    if (g_r) {
        out[0] = MF; out[1] = anti; out[2] = net; out[3] = outw; out[4] = Ltot;
    } else {
        out[0] = MF; out[1] = net; out[2] = outw; out[3] = Ltot;
    }
    return LYD_OK;
}

int lyd_force_multiplier(lyd_ctx *c, double dt, double zc, int32_t bc_z_bot, double out[4]) {
    if (!c || !out) return LYD_ERR_ARG;
    return force_multiplier(c, dt, zc, bc_z_bot, nullptr, nullptr, out);
}

int lyd_force_multiplier_gravity(lyd_ctx *c, double dt, const double *g_r, const double *g_Z, double zc,
                                 int32_t bc_z_bot, double out[5]) {
    if (!c || !out || !g_r || !g_Z) return LYD_ERR_ARG;
    return force_multiplier(c, dt, zc, bc_z_bot, g_r, g_Z, out);
}

int lyd_f_esc(lyd_ctx *c, double L_all, int32_t bc_z_bot, double *f) {
    if (!c || !f) return LYD_ERR_ARG;
    LYD_TRY(single_cloud(c, "lyd_f_esc"));
    cudaSetDevice(c->dev);
    if (!all_have(c, BIT_GEOM) || !c->freq_set) return fail(c, LYD_ERR_STATE, "geometry / frequency grid not set");
    if (L_all <= 0.0) { *f = 0.0; return LYD_OK; }
    launch_fesc(c->sprec, Jc(c, 1), Jc(c, 2), c->A_r, c->A_Z, c->dnu, c->nnu, c->nr[0], c->nz[0], bc_z_bot, c->jscale,
                c->small, c->st);
    LYD_CU(c, cudaGetLastError());
    double num;
    LYD_CU(c, cudaMemcpyAsync(&num, c->small, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    LYD_TRY(check_err(c));
    double Lsim = (bc_z_bot == LYD_BC_REFLECT) ? 0.5 * L_all : L_all;
    *f = Lsim > 0.0 ? num / Lsim : 0.0;
    return LYD_OK;
}

// ---- fused static-cloud step -----------------------------------------------------------------
template <typename S>
// One step from set[cur] back into set[cur] (x_A in the other set). The adjoint's forward sweep
// passes `tape` to record the advection's tape, `in` / `out` (three fields each, n3 apart) to
// read s_n from and write s_{n+1} into its own storage instead, and `ff` to keep the frequency
// factors F+, F, F- (n3 apart), and `win_next` to receive the window the step decides for the
// next one.
// `polls` > 0 runs the step as one cooperative launch of the persistent kernel whose grid
// barriers give up after that many polls.
static int enqueue_step(lyd_ctx *c, bool timed, double *tape = nullptr, const S *in = nullptr, S *out = nullptr,
                        double *ff = nullptr, bool reduce = true, int *win_next = nullptr, long long polls = 0) {
    const int A = c->cur, B = 1 - c->cur;
    AdvArgs<S> aa;
    fill_adv<S>(c, aa, A, B);
    aa.tape = tape;
    aa.tape_stride = (long long)c->n3;
    if (in) { aa.J = in; aa.Hr = in + c->n3; aa.HZ = in + 2 * c->n3; aa.tmaps = nullptr; }
    FreqArgs<S> fa;
    if (out)
        fill_freq<S>(c, fa, c->set[B][0], c->set[B][1], c->set[B][2], c->set[B][0], out, out + c->n3,
                     out + 2 * c->n3);
    else
        fill_freq<S>(c, fa, c->set[B][0], c->set[B][1], c->set[B][2], c->set[B][0], c->set[A][0], c->set[A][1],
                     c->set[A][2]);
    fa.do_emission = 1; fa.do_freq = 1; fa.update_ff = 1;
    fa.parts = PART_ACTIVE | PART_DIAG;
    fa.f_r = c->cellf[CF_F_R]; fa.f_Z = c->cellf[CF_F_Z];
    if (ff) { fa.Fkp = ff; fa.Fk = ff + c->n3; fa.Fkm = ff + 2 * c->n3; }
    RedArgs ra = red_args(c, PART_ACTIVE | PART_DIAG);
    ra.diag = c->hist; ra.step_counter = c->step_ctr; ra.done = c->step_ctr + 1; ra.hist_capacity = c->hist_cap;
    ra.kwin_copy = win_next;
    const int prec = c->prec;
    if (polls > 0) {
        if (timed) cudaEventRecord(c->ev[0], c->st);
        cudaError_t e = launch_persistent(prec, c->cfg.flux_method, &aa, &fa, ra, c->nnu, c->ntiles, c->nitems, c->bar,
                                          polls, c->err, c->st);
        if (timed)
            for (int q = 1; q < 4; q++) cudaEventRecord(c->ev[q], c->st);
        if (e != cudaSuccess) return fail(c, LYD_ERR_CUDA, std::string("persistent step: ") + cudaGetErrorString(e));
        LYD_CU(c, cudaGetLastError());
        return LYD_OK;
    }
    if (timed) cudaEventRecord(c->ev[0], c->st);
    launch_advect(prec, c->cfg.flux_method, &aa, c->ntiles, c->tune.adv_ctas_per_sm, c->st);
    if (timed) cudaEventRecord(c->ev[1], c->st);
    launch_freq(prec, &fa, c->nnu, c->nitems, c->st);
    if (timed) cudaEventRecord(c->ev[2], c->st);
    if (reduce) launch_reduce(ra, c->st);
    if (timed) cudaEventRecord(c->ev[3], c->st);
    LYD_CU(c, cudaGetLastError());
    return LYD_OK;
}

int lyd_set_timing(lyd_ctx *c, int32_t enable) {
    if (!c) return LYD_ERR_ARG;
    c->timing = enable != 0;
    return LYD_OK;
}

int lyd_get_timing(lyd_ctx *c, double ms[3]) {
    if (!c || !ms) return LYD_ERR_ARG;
    for (int q = 0; q < 3; q++) ms[q] = c->ms[q];
    return LYD_OK;
}

// n_steps fused steps with the parameters already in the host descriptors; `polls` > 0 runs
// each step as one persistent cooperative launch (see enqueue_step).
static int run_steps(lyd_ctx *c, int n_steps, lyd_diag *hist_out, long long polls = 0) {
    LYD_TRY(need_inputs(c, true, true));
    if (n_steps == 0) return LYD_OK;
    if (n_steps > c->hist_cap) {
        LYD_CU(c, cudaStreamSynchronize(c->st));
        cudaFree(c->hist);
        c->hist = nullptr;
        c->hist_cap = 0;
        int cap = n_steps < 1024 ? 1024 : n_steps;
        LYD_TRY(dalloc(c, (void **)&c->hist, (size_t)cap * c->ncl * 7 * 8));
        c->hist_cap = cap;
        drop_graph(c);
    }
    LYD_TRY(sync_desc(c));
    LYD_CU(c, cudaMemsetAsync(c->step_ctr, 0, 2 * sizeof(int), c->st));
    // the fused step keeps no Delta rho u between steps (Reset_Delta_rho_u! ends each step)
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_R], 0, c->ncell * 8, c->st));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_Z], 0, c->ncell * 8, c->st));
    if (!c->active_valid) LYD_TRY(run_find_active(c));
    if (c->timing) {
        double acc[3] = {0, 0, 0};
        for (int n = 0; n < n_steps; n++) {
            int r = c->sprec == 0 ? enqueue_step<double>(c, true, nullptr, nullptr, nullptr, nullptr, true, nullptr, polls)
                                  : enqueue_step<float>(c, true, nullptr, nullptr, nullptr, nullptr, true, nullptr, polls);
            if (r != LYD_OK) return r;
            LYD_CU(c, cudaEventSynchronize(c->ev[3]));
            for (int q = 0; q < 3; q++) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, c->ev[q], c->ev[q + 1]);
                acc[q] += ms;
            }
        }
        for (int q = 0; q < 3; q++) c->ms[q] = acc[q];
    } else if (polls > 0 && c->persist_graph < 0) {
        // the runtime refused to capture the cooperative launch: one launch per step
        for (int n = 0; n < n_steps; n++) {
            int r = c->sprec == 0 ? enqueue_step<double>(c, false, nullptr, nullptr, nullptr, nullptr, true, nullptr, polls)
                                  : enqueue_step<float>(c, false, nullptr, nullptr, nullptr, nullptr, true, nullptr, polls);
            if (r != LYD_OK) return r;
        }
    } else {
        if (!c->gexec || c->gkey_cur != c->cur || c->gkey_polls != polls) {
            drop_graph(c);
            cudaGraph_t g = nullptr;
            LYD_CU(c, cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
            int r = c->sprec == 0 ? enqueue_step<double>(c, false, nullptr, nullptr, nullptr, nullptr, true, nullptr, polls)
                                  : enqueue_step<float>(c, false, nullptr, nullptr, nullptr, nullptr, true, nullptr, polls);
            cudaError_t e = cudaStreamEndCapture(c->st, &g);
            if (e == cudaSuccess && r == LYD_OK) {
                e = cudaGraphInstantiate(&c->gexec, g, 0);
                if (e != cudaSuccess) c->gexec = nullptr;
            }
            if (g) cudaGraphDestroy(g);
            if (polls > 0 && (r != LYD_OK || e != cudaSuccess)) {
                // capture of the cooperative launch refused: launch it directly from now on
                cudaGetLastError();
                c->persist_graph = -1;
                return run_steps(c, n_steps, hist_out, polls);
            }
            if (r != LYD_OK) return r;
            if (e != cudaSuccess) return fail(c, LYD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            c->gkey_cur = c->cur;
            c->gkey_polls = polls;
            if (polls > 0) c->persist_graph = 1;
        }
        for (int n = 0; n < n_steps; n++) LYD_CU(c, cudaGraphLaunch(c->gexec, c->st));
    }
    c->old_alias = true;
    c->active_valid = true;
    if (hist_out) {
        std::vector<double> h((size_t)n_steps * c->ncl * 7);
        LYD_CU(c, cudaMemcpyAsync(h.data(), c->hist, h.size() * 8, cudaMemcpyDeviceToHost, c->st));
        LYD_TRY(check_err(c));
        for (size_t n = 0; n < (size_t)n_steps * c->ncl; n++) {
            const double *r = &h[n * 7];
            hist_out[n].M_F = r[0]; hist_out[n].M_F_radial_net = r[1]; hist_out[n].M_F_radial_out = r[2];
            hist_out[n].L_tot = r[3]; hist_out[n].f_esc = r[4];
            hist_out[n].kmin = (int32_t)r[5]; hist_out[n].kmax = (int32_t)r[6];
        }
        return LYD_OK;
    }
    // without a history buffer the call only enqueues; errors surface at the next
    // synchronising call (lyd_synchronize, a download or a diagnostic)
    LYD_CU(c, cudaGetLastError());
    return LYD_OK;
}

int lyd_static_steps(lyd_ctx *c, const lyd_step_params *p, lyd_diag *hist_out) {
    if (!c || !p) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(check_bcs(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top));
    if (!(p->c_tilde > 0.0) || !(p->dt > 0.0) || p->n_steps < 0) return fail(c, LYD_ERR_ARG, "bad step parameters");
    params_all(c, p->c_tilde, p->dt, p->c_tilde * p->dt);
    for (CloudDesc &d : c->desc) d.z_center = p->z_center;
    bcs_all(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top);
    return run_steps(c, p->n_steps, hist_out);
}

// ---- one step on host state, pipelined over row chunks -----------------------------------------
constexpr int kMaxHostChunks = 16;

// The work lists grouped by row chunk: chunk q covers a run of the T tile rows, its advection
// tiles (every bin chunk of those rows), and the frequency items whose cells all lie below the
// chunk's last row (the last chunk takes the rest). The first and the last chunk get half the
// rows of the others: the first chunk's upload runs before anything else can start, and the
// last chunk's download after everything else has ended.
static int build_host_chunks(lyd_ctx *c, int chunks) {
    const int rows = c->tune.rows_per_tile, nr = c->nr[0], nz = c->nz[0];
    const int ntr = (nz + rows - 1) / rows, nkb = (c->nnu + 31) / 32, cpb = cells_per_block(c);
    if (c->hs_req == chunks && c->hs_rows == rows && c->hs_cpb == cpb && c->ctiles) return LYD_OK;
    c->hs_req = chunks;
    if (chunks > ntr) chunks = ntr;
    std::vector<int4> t;
    c->ct_off.assign(chunks + 1, 0);
    c->it_off.assign(chunks + 1, 0);
    c->row_off.assign(chunks + 1, 0);
    // boundary q (0 < q < n) at tile row T (q - 1/2) / (n - 1), rounded; at least one tile row each
    auto bound = [&](int q) {
        if (q <= 0) return 0;
        if (q >= chunks) return ntr;
        const int b = (int)(((long long)ntr * (2 * q - 1) + (chunks - 1)) / (2 * (chunks - 1)));
        return std::min(std::max(b, q), ntr - (chunks - q));
    };
    for (int q = 0; q < chunks; q++) {
        const int tr0 = bound(q), tr1 = bound(q + 1);
        c->ct_off[q] = (int)t.size();
        for (int kb = 0; kb < nkb; kb++)
            for (int tr = tr0; tr < tr1; tr++)
                for (int i0 = 0; i0 < nr; i0 += kTileCols) t.push_back(make_int4(0, i0, tr * rows, 32 * kb));
        c->row_off[q] = std::min(nz, tr0 * rows);
        c->it_off[q] = (int)std::min<long long>(c->nitems, (long long)c->row_off[q] * nr / cpb);
    }
    c->ct_off[chunks] = (int)t.size();
    c->row_off[chunks] = nz;
    c->it_off[chunks] = c->nitems;
    cudaFree(c->ctiles);
    c->ctiles = nullptr;
    LYD_TRY(dalloc(c, (void **)&c->ctiles, t.size() * sizeof(int4)));
    LYD_CU(c, cudaMemcpyAsync(c->ctiles, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice, c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    c->hs_chunks = chunks;
    c->hs_rows = rows;
    c->hs_cpb = cpb;
    return LYD_OK;
}

// Drains the context's streams when a call that spreads its work over several of them leaves
// early: no copy into or out of the caller's arrays (the host-state step), and no recomputation
// into the workspace (the adjoint), may still run after the call returns.
struct StreamDrain {
    lyd_ctx *c;
    bool armed = false;
    ~StreamDrain() {
        if (!armed) return;
        for (cudaStream_t s : {c->st_up, c->st_fq, c->st_dn, c->st_rec, c->st})
            if (s) cudaStreamSynchronize(s);
    }
};

int lyd_static_step_host(lyd_ctx *c, const lyd_step_params *p, const double *J, const double *Hr, const double *HZ,
                         double *J_out, double *Hr_out, double *HZ_out, int32_t chunks, lyd_diag *diag) {
    if (!c || !p || !J || !Hr || !HZ || !J_out || !Hr_out || !HZ_out) return LYD_ERR_ARG;
    LYD_TRY(single_cloud(c, "lyd_static_step_host"));
    cudaSetDevice(c->dev);
    if (chunks < 1 || chunks > kMaxHostChunks) return fail(c, LYD_ERR_ARG, "chunks outside 1..16");
    if (c->prec != LYD_PREC_FP64 || c->jscale != 1.0)
        return fail(c, LYD_ERR_STATE, "the host-state step runs the FP64 form (state in the caller's units)");
    if (c->desc[0].j_own0 != 0 || c->desc[0].j_own1 != c->nz[0])
        return fail(c, LYD_ERR_STATE, "the host-state step runs on a whole field, not a Z slab");
    LYD_TRY(check_bcs(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top));
    if (!(p->c_tilde > 0.0) || !(p->dt > 0.0)) return fail(c, LYD_ERR_ARG, "bad step parameters");
    params_all(c, p->c_tilde, p->dt, p->c_tilde * p->dt);
    c->desc[0].z_center = p->z_center;
    bcs_all(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top);
    LYD_TRY(need_inputs(c, true, true));
    LYD_TRY(sync_desc(c));
    const size_t n3 = c->n3, nnu = c->nnu, nr = c->nr[0];
    if (!c->hin) LYD_TRY(dalloc(c, (void **)&c->hin, 3 * n3 * 8));
    if (!c->kwin_chk) LYD_TRY(dalloc(c, (void **)&c->kwin_chk, 4 * sizeof(int)));
    if (c->hs_pchk != c->nitems) {
        cudaFree(c->part_chk);
        c->part_chk = nullptr;
        c->hs_pchk = 0;
        LYD_TRY(dalloc(c, (void **)&c->part_chk, (size_t)c->nitems * (c->nnu + kExtraCols) * 8));
        c->hs_pchk = c->nitems;
    }
    if (!c->st_up) {
        LYD_CU(c, cudaStreamCreateWithFlags(&c->st_up, cudaStreamNonBlocking));
        LYD_CU(c, cudaStreamCreateWithFlags(&c->st_dn, cudaStreamNonBlocking));
        LYD_CU(c, cudaStreamCreateWithFlags(&c->st_fq, cudaStreamNonBlocking));
        for (cudaEvent_t &e : c->hs_ev) LYD_CU(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    LYD_TRY(build_host_chunks(c, chunks));
    const int nch = c->hs_chunks;
    cudaEvent_t *ev_up = c->hs_ev, *ev_fq = c->hs_ev + kMaxHostChunks, *ev_adv = c->hs_ev + 2 * kMaxHostChunks;
    cudaEvent_t ev_start = c->hs_ev[3 * kMaxHostChunks], ev_chk = c->hs_ev[3 * kMaxHostChunks + 1];
    const double *src[3] = {J, Hr, HZ};
    double *dst[3] = {J_out, Hr_out, HZ_out};
    StreamDrain drain{c};
    drain.armed = true;
    // whatever ran before on the context's stream is done with the reduction's counters first
    LYD_CU(c, cudaEventRecord(ev_start, c->st));
    LYD_CU(c, cudaStreamWaitEvent(c->st_up, ev_start, 0));
    // the step keeps no Delta rho u between steps; the window it uses is the previous step's
    const bool spec = c->active_valid;
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_R], 0, c->ncell * 8, c->st));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_Z], 0, c->ncell * 8, c->st));
    // uploads, chunk after chunk, then the window of the uploaded J (FindActiveBins) for the check.
    // A chunk's advection reads two rows past its last row (the Z face of its last row reads rows
    // up to one beyond, the reconstruction one more), so chunk q's upload ends two rows into
    // chunk q+1 and the advection of q waits for q's upload alone.
    const int nzr = c->nz[0];
    auto up_row = [&](int q) { return q <= 0 ? 0 : q >= nch ? nzr : std::min(nzr, c->row_off[q] + 2); };
    for (int q = 0; q < nch; q++) {
        const size_t off = (size_t)up_row(q) * nr * nnu, len = (size_t)(up_row(q + 1) - up_row(q)) * nr * nnu;
        if (len > 0)
            for (int f = 0; f < 3; f++)
                LYD_CU(c, cudaMemcpyAsync(c->hin + f * n3 + off, src[f] + off, len * 8, cudaMemcpyHostToDevice, c->st_up));
        LYD_CU(c, cudaEventRecord(ev_up[q], c->st_up));
    }
    launch_find_active(0, c->hin, c->nnu, c->dnu, c->dV, c->cl, c->items, c->nitems, c->jeps_s, c->part_chk, c->st_up);
    RedArgs rc = red_args(c, PART_ACTIVE);
    rc.partials = c->part_chk;
    rc.kwin = c->kwin_chk + 2;
    rc.last = nullptr;
    launch_reduce(rc, c->st_up);
    LYD_CU(c, cudaEventRecord(ev_chk, c->st_up));
    if (!spec) {
        // no window yet: the step waits for that of the uploaded J
        LYD_CU(c, cudaStreamWaitEvent(c->st, ev_chk, 0));
        LYD_CU(c, cudaMemcpyAsync(c->kwin, c->kwin_chk + 2, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    }
    LYD_CU(c, cudaMemcpyAsync(c->kwin_chk, c->kwin, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    // per chunk: the advection of its rows (once they and the two rows above them have landed)
    // from the uploaded state into the other buffer set, then on a
    // second stream the frequency step of its items back into the state's set, then its rows
    // down. A chunk's launches fill a fraction of the GPU, so the frequency step of chunk q runs
    // beside the advection of chunk q+1 (they touch different rows).
    const int A = c->cur, B = 1 - c->cur;
    AdvArgs<double> aa;
    fill_adv<double>(c, aa, A, B);
    aa.J = c->hin; aa.Hr = c->hin + n3; aa.HZ = c->hin + 2 * n3;
    aa.tmaps = nullptr;
    FreqArgs<double> fa;
    fill_freq<double>(c, fa, c->set[B][0], c->set[B][1], c->set[B][2], c->set[B][0], c->set[A][0], c->set[A][1],
                      c->set[A][2]);
    fa.do_emission = 1; fa.do_freq = 1; fa.update_ff = 1;
    fa.parts = PART_ACTIVE | PART_DIAG;
    fa.f_r = c->cellf[CF_F_R]; fa.f_Z = c->cellf[CF_F_Z];
    fa.nitems_all = c->nitems;
    for (int q = 0; q < nch; q++) {
        LYD_CU(c, cudaStreamWaitEvent(c->st, ev_up[q], 0));
        aa.tiles = c->ctiles + c->ct_off[q];
        if (c->ct_off[q + 1] > c->ct_off[q])
            launch_advect(c->prec, c->cfg.flux_method, &aa, c->ct_off[q + 1] - c->ct_off[q], c->tune.adv_ctas_per_sm,
                          c->st);
        LYD_CU(c, cudaEventRecord(ev_adv[q], c->st));
        LYD_CU(c, cudaStreamWaitEvent(c->st_fq, ev_adv[q], 0));
        fa.item0 = c->it_off[q];
        if (c->it_off[q + 1] > c->it_off[q])
            launch_freq(c->prec, &fa, c->nnu, c->it_off[q + 1] - c->it_off[q], c->st_fq);
        LYD_CU(c, cudaEventRecord(ev_fq[q], c->st_fq));
        LYD_CU(c, cudaStreamWaitEvent(c->st_dn, ev_fq[q], 0));
        const size_t b0 = (size_t)c->it_off[q] * c->hs_cpb;
        const size_t b1 = std::min<size_t>((size_t)c->it_off[q + 1] * c->hs_cpb, (size_t)c->ncell);
        if (b1 > b0)
            for (int f = 0; f < 3; f++)
                LYD_CU(c, cudaMemcpyAsync(dst[f] + b0 * nnu, static_cast<const double *>(c->set[A][f]) + b0 * nnu,
                                          (b1 - b0) * nnu * 8, cudaMemcpyDeviceToHost, c->st_dn));
    }
    LYD_CU(c, cudaGetLastError());
    // the diagnostics and the next window, after the check (the two share the reduction's counters)
    LYD_CU(c, cudaStreamWaitEvent(c->st, ev_fq[nch - 1], 0));
    LYD_CU(c, cudaStreamWaitEvent(c->st, ev_chk, 0));
    launch_reduce(red_args(c, PART_ACTIVE | PART_DIAG), c->st);
    double rec[7];
    int kw[4];
    LYD_CU(c, cudaMemcpyAsync(rec, c->last, sizeof(rec), cudaMemcpyDeviceToHost, c->st));
    LYD_CU(c, cudaMemcpyAsync(kw, c->kwin_chk, sizeof(kw), cudaMemcpyDeviceToHost, c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st_dn));
    LYD_CU(c, cudaStreamSynchronize(c->st_up));
    LYD_TRY(check_err(c));
    c->old_alias = true;
    c->active_valid = true;
    if (kw[0] != kw[2] || kw[1] != kw[3]) {
        // the uploaded J was not the state the previous step left: its window differs from the
        // one the step used. Step again from the uploaded state with its own window, unpipelined.
        for (int f = 0; f < 3; f++)
            LYD_CU(c, cudaMemcpyAsync(c->set[A][f], c->hin + f * n3, n3 * 8, cudaMemcpyDeviceToDevice, c->st));
        LYD_CU(c, cudaMemcpyAsync(c->kwin, c->kwin_chk + 2, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
        LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_R], 0, c->ncell * 8, c->st));
        LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_Z], 0, c->ncell * 8, c->st));
        LYD_TRY(enqueue_step<double>(c, false, nullptr, nullptr, nullptr, nullptr, false));
        launch_reduce(red_args(c, PART_ACTIVE | PART_DIAG), c->st);
        for (int f = 0; f < 3; f++)
            LYD_CU(c, cudaMemcpyAsync(dst[f], c->set[A][f], n3 * 8, cudaMemcpyDeviceToHost, c->st));
        LYD_CU(c, cudaMemcpyAsync(rec, c->last, sizeof(rec), cudaMemcpyDeviceToHost, c->st));
        LYD_TRY(check_err(c));
    }
    if (diag) {
        diag->M_F = rec[0]; diag->M_F_radial_net = rec[1]; diag->M_F_radial_out = rec[2];
        diag->L_tot = rec[3]; diag->f_esc = rec[4];
        diag->kmin = (int32_t)rec[5]; diag->kmax = (int32_t)rec[6];
    }
    return LYD_OK;
}

// ---- Z-slab domain decomposition -------------------------------------------------------------
int lyd_dd_set_halo(lyd_ctx *c, int32_t h_bot, int32_t h_top) {
    if (!c) return LYD_ERR_ARG;
    LYD_TRY(single_cloud(c, "lyd_dd_set_halo"));
    cudaSetDevice(c->dev);
    const int nz = c->nz[0];
    if ((h_bot != 0 && h_bot != 2) || (h_top != 0 && h_top != 2) || nz - h_bot - h_top < 2)
        return fail(c, LYD_ERR_ARG, "halos are 0 or 2 rows and at least 2 rows must be owned");
    c->desc[0].j_own0 = h_bot;
    c->desc[0].j_own1 = nz - h_top;
    c->active_valid = false;
    return build_work(c);
}

int lyd_dd_columns(lyd_ctx *c) { return c ? c->nnu + kExtraCols : LYD_ERR_ARG; }

int lyd_dd_find_active_partials(lyd_ctx *c, double *colsum) {
    if (!c || !colsum) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(need_inputs(c, false, false));
    LYD_TRY(sync_desc(c));
    launch_find_active(c->sprec, Jc(c, 0), c->nnu, c->dnu, c->dV, c->cl, c->items, c->nitems, c->jeps_s, c->partials,
                       c->st);
    launch_column_sums(c->partials, c->nnu + kExtraCols, c->nitems, colsum, c->st);
    LYD_CU(c, cudaGetLastError());
    return LYD_OK;
}

int lyd_dd_step_partials(lyd_ctx *c, const lyd_step_params *p, double *colsum) {
    if (!c || !p || !colsum) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    LYD_TRY(check_bcs(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top));
    if (!(p->c_tilde > 0.0) || !(p->dt > 0.0)) return fail(c, LYD_ERR_ARG, "bad step parameters");
    if (!c->active_valid) return fail(c, LYD_ERR_STATE, "no active window: run lyd_dd_find_active_partials and lyd_dd_finish first");
    LYD_TRY(need_inputs(c, true, true));
    params_all(c, p->c_tilde, p->dt, p->c_tilde * p->dt);
    for (CloudDesc &d : c->desc) d.z_center = p->z_center;
    bcs_all(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top);
    LYD_TRY(sync_desc(c));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_R], 0, c->ncell * 8, c->st));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_Z], 0, c->ncell * 8, c->st));
    int r = c->sprec == 0 ? enqueue_step<double>(c, false, nullptr, nullptr, nullptr, nullptr, false)
                          : enqueue_step<float>(c, false, nullptr, nullptr, nullptr, nullptr, false);
    if (r != LYD_OK) return r;
    launch_column_sums(c->partials, c->nnu + kExtraCols, c->nitems, colsum, c->st);
    LYD_CU(c, cudaGetLastError());
    c->active_valid = false;   // until lyd_dd_finish decides the next window
    return LYD_OK;
}

int lyd_dd_finish(lyd_ctx *c, const double *colsum, int32_t step, lyd_diag *rec) {
    if (!c || !colsum) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    if (!c->dd_cl) LYD_TRY(dalloc(c, (void **)&c->dd_cl, sizeof(CloudDesc)));
    CloudDesc d = c->desc[0];
    d.pb0 = 0;
    d.npb = 1;                 // the all-reduced column sums: one "block"
    LYD_CU(c, cudaMemcpyAsync(c->dd_cl, &d, sizeof(d), cudaMemcpyHostToDevice, c->st));
    RedArgs ra = red_args(c, step ? (PART_ACTIVE | PART_DIAG) : PART_ACTIVE);
    ra.partials = colsum;
    ra.nblocks = 1;
    ra.cl = c->dd_cl;
    ra.colsum = nullptr;   // the input is already the column sums: one CTA reads them
    ra.cnt = nullptr;
    launch_reduce(ra, c->st);
    LYD_CU(c, cudaGetLastError());
    c->active_valid = true;
    if (rec) {
        double h[7];
        int kw[2];
        LYD_CU(c, cudaMemcpyAsync(h, c->last, sizeof(h), cudaMemcpyDeviceToHost, c->st));
        LYD_CU(c, cudaMemcpyAsync(kw, c->kwin, sizeof(kw), cudaMemcpyDeviceToHost, c->st));
        LYD_CU(c, cudaStreamSynchronize(c->st));
        rec->M_F = h[0]; rec->M_F_radial_net = h[1]; rec->M_F_radial_out = h[2]; rec->L_tot = h[3]; rec->f_esc = h[4];
        if (step) { rec->kmin = (int32_t)h[5]; rec->kmax = (int32_t)h[6]; }
        else { rec->kmin = kw[0]; rec->kmax = kw[1]; }
    }
    return check_err(c);
}

int lyd_dd_halo(lyd_ctx *c, int32_t side, int32_t pack, void *buf) {
    if (!c || !buf || (side != 0 && side != 1)) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    const CloudDesc &d = c->desc[0];
    const int hb = d.j_own0, ht = d.nz - d.j_own1;
    if ((side == 0 && hb != 2) || (side == 1 && ht != 2)) return fail(c, LYD_ERR_STATE, "no halo on that side");
    // pack: the two owned rows next to the neighbour; unpack: the two halo rows
    const int row = pack ? (side == 0 ? d.j_own0 : d.j_own1 - 2) : (side == 0 ? d.j_own0 - 2 : d.j_own1);
    const size_t n2 = (size_t)2 * d.nr * c->nnu, off = (size_t)row * d.nr * c->nnu;
    for (int q = 0; q < 3; q++) {
        char *dev = static_cast<char *>(Jc(c, q)) + off * c->ssz;
        char *b = static_cast<char *>(buf) + (size_t)q * n2 * c->ssz;
        if (pack) LYD_CU(c, cudaMemcpyAsync(b, dev, n2 * c->ssz, cudaMemcpyDeviceToDevice, c->st));
        else LYD_CU(c, cudaMemcpyAsync(dev, b, n2 * c->ssz, cudaMemcpyDeviceToDevice, c->st));
    }
    return LYD_OK;
}

// per-cloud step parameters into the host descriptors
static int batch_params(lyd_ctx *c, const lyd_cloud_params *p) {
    for (int q = 0; q < c->ncl; q++) {
        LYD_TRY(check_bcs(c, c->cfg.bc_r_left, p[q].bc_r_right, p[q].bc_z_bot, p[q].bc_z_top));
        if (!(p[q].c_tilde > 0.0) || !(p[q].dt > 0.0)) return fail(c, LYD_ERR_ARG, "bad step parameters");
    }
    for (int q = 0; q < c->ncl; q++) {
        CloudDesc &d = c->desc[q];
        d.c_tilde = p[q].c_tilde; d.dt = p[q].dt; d.ctdt = p[q].c_tilde * p[q].dt; d.z_center = p[q].z_center;
        d.bc_r_left = c->cfg.bc_r_left;
        d.bc_r_right = p[q].bc_r_right; d.bc_z_bot = p[q].bc_z_bot; d.bc_z_top = p[q].bc_z_top;
    }
    return LYD_OK;
}

int lyd_batch_steps(lyd_ctx *c, const lyd_cloud_params *p, int32_t n_steps, lyd_diag *hist_out) {
    if (!c || !p) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    if (n_steps < 0) return fail(c, LYD_ERR_ARG, "bad step count");
    LYD_TRY(batch_params(c, p));
    return run_steps(c, n_steps, hist_out);
}

int lyd_batch_steps_persistent(lyd_ctx *c, const lyd_cloud_params *p, int32_t n_steps, int64_t barrier_polls,
                               lyd_diag *hist_out) {
    if (!c || !p) return LYD_ERR_ARG;
    if (barrier_polls < 1) return fail(c, LYD_ERR_ARG, "barrier_polls must be positive");
    cudaSetDevice(c->dev);
    if (n_steps < 0) return fail(c, LYD_ERR_ARG, "bad step count");
    LYD_TRY(batch_params(c, p));
    return run_steps(c, n_steps, hist_out, (long long)barrier_polls);
}

int lyd_persistent_info(lyd_ctx *c, int32_t *graph) {
    if (!c || !graph) return LYD_ERR_ARG;
    *graph = c->persist_graph;
    return LYD_OK;
}

// ---- set-up helpers ------------------------------------------------------------------------------
int lyd_update_hvoigt(lyd_ctx *c) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    if (!c->freq_set) return fail(c, LYD_ERR_STATE, "frequency grid not set");
    if (!all_have(c, 1u << CF_T)) return fail(c, LYD_ERR_STATE, "temperature T not uploaded");
    if (!c->lut) {
        std::vector<double> h((size_t)5 * kLutN);
        build_voigt_lut(h.data(), kLutN, kLutXmax);
        LYD_TRY(dalloc(c, (void **)&c->lut, h.size() * 8));
        LYD_CU(c, cudaMemcpyAsync(c->lut, h.data(), h.size() * 8, cudaMemcpyHostToDevice, c->st));
        LYD_CU(c, cudaStreamSynchronize(c->st));
    }
    launch_hvoigt(c->sprec, c->Hv, c->cellf[CF_T], c->nu, c->nuC, c->nnu, c->ncell, c->lut, kLutN, kLutXmax, c->st);
    LYD_CU(c, cudaGetLastError());
    set_all(c, BIT_HV);
    c->hv_from_T = true;
    c->phi_inv_ready = false;
    return check_err(c);
}

int lyd_update_phi_nu(lyd_ctx *c, int32_t kmin, int32_t kmax) {
    if (!c) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    if (kmin < 0 || kmax >= c->nnu || kmin > kmax) return fail(c, LYD_ERR_ARG, "bad bin range");
    if (!all_have(c, BIT_HV) || !c->freq_set) return fail(c, LYD_ERR_STATE, "H_voigt / frequency grid not set");
    launch_phi_inv(c->sprec, c->Hv, c->dnu, c->nnu, c->ncell, kmin, kmax, c->phi_inv, c->st);
    LYD_CU(c, cudaGetLastError());
    c->phi_kmin = kmin;
    c->phi_kmax = kmax;
    // a derived phi_nu replaces an uploaded one
    cudaFree(c->phi);
    c->phi = nullptr;
    for (unsigned &h : c->have) h &= ~BIT_PHI;
    c->phi_inv_ready = true;
    return check_err(c);
}

// ---- RHD-side Lyman-alpha block ---------------------------------------------------------------
int lyd_rhd_lya_prepare(lyd_ctx *c, const double *T, const double *nHI, const double *nH2, const double *nHII,
                        const double *nHeI, const double *ne, const double *nOHx, const double *nCHx,
                        const double *rho_d, const lyd_dust_lya *dust, double z, int32_t ots, int32_t destruction) {
    if (!c) return LYD_ERR_ARG;
    if (!T || !nHI || !nH2 || !nHII || !nHeI || !ne || !nOHx || !nCHx || !rho_d || !dust)
        return fail(c, LYD_ERR_ARG, "null input");
    cudaSetDevice(c->dev);
    if (!c->freq_set) return fail(c, LYD_ERR_STATE, "frequency grid not set");
    const size_t nc = c->ncell;
    LYD_TRY(ensure_stage(c, 11 * nc));
    double *d = c->stage;
    const double *src[8] = {T, nHI, nH2, nHII, nHeI, ne, nOHx, nCHx};
    for (int q = 0; q < 8; q++) LYD_TRY(h2d(c, d + q * nc, src[q], nc));
    LYD_TRY(h2d(c, d + 8 * nc, rho_d, 3 * nc));
    RhdPrepArgs a;
    memset(&a, 0, sizeof(a));
    a.T = d; a.nHI = d + nc; a.nH2 = d + 2 * nc; a.nHII = d + 3 * nc; a.nHeI = d + 4 * nc; a.ne = d + 5 * nc;
    a.nOHx = d + 6 * nc; a.nCHx = d + 7 * nc; a.rho_d = d + 8 * nc;
    for (int q = 0; q < 3; q++) { a.kabs[q] = dust->kappa_abs[q]; a.kF[q] = dust->kappa_F[q]; }
    a.rho_ignore = dust->rho_ignore; a.z = z; a.ots = ots; a.destruction = destruction; a.ncell = nc;
    a.alpha = c->cellf[CF_ALPHA]; a.alpha_c = c->cellf[CF_ALPHA_C]; a.alpha_cF = c->cellf[CF_ALPHA_CF];
    a.pd = c->cellf[CF_PD]; a.js = c->cellf[CF_JS]; a.T_out = c->cellf[CF_T];
    if (!c->dust_F) LYD_TRY(dalloc(c, (void **)&c->dust_F, 3 * nc * 8));
    a.dust_F = c->dust_F;
    launch_rhd_prep(a, c->st);
    LYD_CU(c, cudaGetLastError());
    set_all(c, (1u << CF_ALPHA) | (1u << CF_ALPHA_C) | (1u << CF_ALPHA_CF) | (1u << CF_PD) | (1u << CF_JS) |
                   (1u << CF_T));
    LYD_TRY(lyd_update_hvoigt(c));
    return lyd_update_phi_nu(c, 0, c->nnu - 1);
}

int lyd_rhd_lya_absorb(lyd_ctx *c, const double *dt, double c_tilde, int32_t commit, lyd_rhd_lya_out *out) {
    if (!c) return LYD_ERR_ARG;
    if (!dt) return fail(c, LYD_ERR_ARG, "null dt");
    if (!(c_tilde > 0.0)) return fail(c, LYD_ERR_ARG, "c_tilde must be positive");
    cudaSetDevice(c->dev);
    if (!c->dust_F || !c->phi_inv_ready || c->phi || c->phi_kmin != 0 || c->phi_kmax != c->nnu - 1)
        return fail(c, LYD_ERR_STATE, "call lyd_rhd_lya_prepare first (it sets phi_nu over all bins)");
    const size_t nc = c->ncell;
    LYD_TRY(materialize_old(c));
    LYD_TRY(ensure_stage(c, 15 * nc));
    double *d = c->stage;                     // [0, nc): dt ; [nc, 15 nc): outputs
    LYD_TRY(h2d(c, d, dt, nc));
    const void *args = nullptr;
    RhdAbsorbArgs<double> a64;
    RhdAbsorbArgs<float> a32;
    auto fill = [&](auto &a, auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        memset(&a, 0, sizeof(a));
        a.dt = d;
        a.alpha = c->cellf[CF_ALPHA]; a.alpha_c = c->cellf[CF_ALPHA_C]; a.alpha_cF = c->cellf[CF_ALPHA_CF];
        a.pd = c->cellf[CF_PD]; a.js = c->cellf[CF_JS]; a.phi_inv = c->phi_inv; a.dust_F = c->dust_F;
        a.dnu = c->dnu;
        a.Hv = (const S *)c->Hv;
        a.J = (S *)Jc(c, 0); a.Hr = (S *)Jc(c, 1); a.HZ = (S *)Jc(c, 2);
        a.Jold = (S *)Jold(c, 0); a.Hrold = (S *)Jold(c, 1); a.HZold = (S *)Jold(c, 2);
        a.e_lya = c->cellf[CF_E_LYA];
        a.out = d + nc;
        a.c_tilde = c_tilde; a.jeps = c->jeps_s; a.j_scale = c->jscale;
        a.nnu = c->nnu; a.commit = commit ? 1 : 0; a.ncell = nc;
    };
    if (c->sprec == 0) { fill(a64, (double *)nullptr); args = &a64; }
    else { fill(a32, (float *)nullptr); args = &a32; }
    launch_rhd_absorb(c->sprec, args, c->st);
    LYD_CU(c, cudaGetLastError());
    c->active_valid = false;
    if (out) {
        std::vector<double> flag;
        const double *o = d + nc;
        if (out->reject) {
            flag.resize(nc);
            LYD_CU(c, cudaMemcpyAsync(flag.data(), o, nc * 8, cudaMemcpyDeviceToHost, c->st));
        }
        if (out->de) LYD_CU(c, cudaMemcpyAsync(out->de, o + nc, nc * 8, cudaMemcpyDeviceToHost, c->st));
        if (out->e_new) LYD_CU(c, cudaMemcpyAsync(out->e_new, o + 2 * nc, nc * 8, cudaMemcpyDeviceToHost, c->st));
        if (out->dru_r) LYD_CU(c, cudaMemcpyAsync(out->dru_r, o + 3 * nc, nc * 8, cudaMemcpyDeviceToHost, c->st));
        if (out->dru_Z) LYD_CU(c, cudaMemcpyAsync(out->dru_Z, o + 4 * nc, nc * 8, cudaMemcpyDeviceToHost, c->st));
        if (out->split) LYD_CU(c, cudaMemcpyAsync(out->split, o + 5 * nc, 8 * nc * 8, cudaMemcpyDeviceToHost, c->st));
        if (out->dt_lya) LYD_CU(c, cudaMemcpyAsync(out->dt_lya, o + 13 * nc, nc * 8, cudaMemcpyDeviceToHost, c->st));
        LYD_CU(c, cudaStreamSynchronize(c->st));
        if (out->reject)
            for (size_t q = 0; q < nc; q++) out->reject[q] = flag[q] != 0.0 ? 1 : 0;
    }
    return check_err(c);
}

int lyd_find_rsl_lya(lyd_ctx *c, double ct_old, double ct_min, const double *u_r, const double *u_Z, const double *P,
                     const double *rho, const double *gamma_ad, const double *T, const double *xHII,
                     const double *xH2, const double *rho_d, const lyd_dust_lya *dust, double eps_rsl,
                     double X_over_mH, double *ct_new) {
    if (!c) return LYD_ERR_ARG;
    if (!u_r || !u_Z || !P || !rho || !gamma_ad || !T || !xHII || !xH2 || !rho_d || !dust || !ct_new)
        return fail(c, LYD_ERR_ARG, "null argument");
    LYD_TRY(single_cloud(c, "lyd_find_rsl_lya"));
    cudaSetDevice(c->dev);
    if (!all_have(c, BIT_GEOM)) return fail(c, LYD_ERR_STATE, "geometry not set");
    if (!all_have(c, 1u << CF_PD)) return fail(c, LYD_ERR_STATE, "pd not set (lyd_rhd_lya_prepare or an upload)");
    const size_t nc = c->ncell;
    LYD_TRY(ensure_stage(c, 11 * nc + 1));
    double *d = c->stage;
    const double *src[8] = {u_r, u_Z, P, rho, gamma_ad, T, xHII, xH2};
    for (int q = 0; q < 8; q++) LYD_TRY(h2d(c, d + q * nc, src[q], nc));
    LYD_TRY(h2d(c, d + 8 * nc, rho_d, 3 * nc));
    RslArgs a;
    memset(&a, 0, sizeof(a));
    a.r_if = c->r_if; a.Z_if = c->Z_if;
    a.u_r = d; a.u_Z = d + nc; a.P = d + 2 * nc; a.rho = d + 3 * nc; a.gamma = d + 4 * nc; a.T = d + 5 * nc;
    a.xHII = d + 6 * nc; a.xH2 = d + 7 * nc; a.rho_d = d + 8 * nc; a.pd = c->cellf[CF_PD];
    for (int q = 0; q < 3; q++) a.kabs[q] = dust->kappa_abs[q];
    a.eps_rsl = eps_rsl; a.X_over_mH = X_over_mH; a.nr = c->nr[0]; a.ncell = nc;
    a.out = reinterpret_cast<unsigned long long *>(d + 11 * nc);
    launch_rsl(a, c->st);
    LYD_CU(c, cudaGetLastError());
    double m = 0.0;
    LYD_CU(c, cudaMemcpyAsync(&m, a.out, 8, cudaMemcpyDeviceToHost, c->st));
    LYD_CU(c, cudaStreamSynchronize(c->st));
    // clamps and the limits on the change from the previous value (:697-711)
    double v = m < ct_min ? ct_min : m;
    v = v < kC ? v : kC;
    if (v < ct_old) v = v > 0.75 * ct_old ? v : 0.75 * ct_old;
    if (v > ct_old) v = v < 4.0 * ct_old ? v : 4.0 * ct_old;
    *ct_new = v;
    return check_err(c);
}

int lyd_pd_lya(lyd_ctx *c, size_t n, const double *nHII, const double *ne, const double *nHI, const double *nHeI,
               const double *nH2, const double *T, double z, double *out) {
    if (!c || !out || !nHII || !ne || !nHI || !nHeI || !nH2 || !T) return LYD_ERR_ARG;
    if (n == 0) return LYD_OK;
    cudaSetDevice(c->dev);
    double *d = nullptr;
    LYD_TRY(dalloc(c, (void **)&d, n * 7 * 8));
    const double *src[6] = {nHII, ne, nHI, nHeI, nH2, T};
    int r = LYD_OK;
    for (int q = 0; q < 6 && r == LYD_OK; q++) r = h2d(c, d + q * n, src[q], n);
    if (r == LYD_OK) {
        launch_pd(n, d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n, z, d + 6 * n, c->st);
        cudaError_t e = cudaMemcpyAsync(out, d + 6 * n, n * 8, cudaMemcpyDeviceToHost, c->st);
        if (e != cudaSuccess) r = fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
        e = cudaStreamSynchronize(c->st);
        if (e != cudaSuccess && r == LYD_OK) r = fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaFree(d);
    return r;
}

int lyd_cfl_dt(lyd_ctx *c, double ct, const double *u_r, const double *u_Z, double cfl, double *dt_out) {
    if (!c || !u_r || !u_Z || !dt_out) return LYD_ERR_ARG;
    LYD_TRY(single_cloud(c, "lyd_cfl_dt"));
    cudaSetDevice(c->dev);
    if (!all_have(c, BIT_GEOM)) return fail(c, LYD_ERR_STATE, "geometry not set");
    double *d = nullptr;
    LYD_TRY(dalloc(c, (void **)&d, c->ncell * 2 * 8));
    int r = h2d(c, d, u_r, c->ncell);
    if (r == LYD_OK) r = h2d(c, d + c->ncell, u_Z, c->ncell);
    double m = 0.0;
    if (r == LYD_OK) {
        launch_cfl(c->r_if, c->Z_if, d, d + c->ncell, c->nr[0], c->nz[0], ct, c->small, c->st);
        cudaError_t e = cudaMemcpyAsync(&m, c->small, 8, cudaMemcpyDeviceToHost, c->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
        if (e != cudaSuccess) r = fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaFree(d);
    if (r == LYD_OK) *dt_out = cfl * m;
    return r;
}

int lyd_edge_spectra_cloud(lyd_ctx *c, int32_t q, double *raw, double *norm, int32_t *ridx, int32_t *zidx) {
    if (!c || !raw || !norm) return LYD_ERR_ARG;
    LYD_TRY(bad_cloud(c, q));
    cudaSetDevice(c->dev);
    if (!c->freq_set) return fail(c, LYD_ERR_STATE, "frequency grid not set");
    const int nr = c->nr[q], nz = c->nz[q];
    int ne = lyd_edge_count(nr, nz);
    if (ne <= 0) return fail(c, LYD_ERR_ARG, "grid too small for the edge ring");
    size_t n = (size_t)ne * c->nnu;
    double *d = nullptr;
    LYD_TRY(dalloc(c, (void **)&d, 2 * n * 8));
    launch_edge(c->sprec, at(Jc(c, 0), c->desc[q].o3, c->ssz), c->dnu, c->nnu, nr, nz, c->jscale, d, d + n, c->st);
    int r = LYD_OK;
    cudaError_t e = cudaMemcpyAsync(raw, d, n * 8, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(norm, d + n, n * 8, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) r = fail(c, LYD_ERR_CUDA, cudaGetErrorString(e));
    cudaFree(d);
    if (r != LYD_OK) return r;
    int k = 0;
    for (int j = 1; j <= nz - 2; j++, k++) { if (ridx) ridx[k] = nr - 2; if (zidx) zidx[k] = j; }
    for (int i = 1; i <= nr - 3; i++, k++) { if (ridx) ridx[k] = i; if (zidx) zidx[k] = nz - 2; }
    for (int i = 1; i <= nr - 3; i++, k++) { if (ridx) ridx[k] = i; if (zidx) zidx[k] = 1; }
    return check_err(c);
}

int lyd_edge_spectra(lyd_ctx *c, double *raw, double *norm, int32_t *ridx, int32_t *zidx) {
    if (!c || !raw || !norm) return LYD_ERR_ARG;
    LYD_TRY(single_cloud(c, "lyd_edge_spectra"));
    return lyd_edge_spectra_cloud(c, 0, raw, norm, ridx, zidx);
}

int lyd_voigt_tables(double *out, int32_t n, double xmax) {
    if (!out || n < 2 || !(xmax > 0.0)) return LYD_ERR_ARG;
    build_voigt_lut(out, n, xmax);
    return LYD_OK;
}

// ---- adjoint of the static-driver loop ---------------------------------------------------------
//
// Two-level checkpointing: the forward sweep stores the state at the start of every segment of
// `checkpoint_every` steps (and each step's active window); the reverse sweep walks the
// segments backwards, recomputes a segment's states from its checkpoint, then runs the
// adjoint steps of that segment from its last step to its first.

// C(s + r, s): the most steps s snapshots reverse with no step advanced more than r times
// (Griewank, "Achieving logarithmic growth of temporal and spatial complexity in reverse
// automatic differentiation", 1992), as a double (exact far beyond the step counts used here).
static double binomial_reach(int s, int r) {
    double b = 1.0;
    for (int q = 1; q <= s; q++) b = b * (double)(r + q) / (double)q;
    return b;
}

int lyd_adjoint_run(lyd_ctx *c, const lyd_adjoint_cfg *cfg, lyd_adjoint_out *out) {
    if (!c || !cfg || !out) return LYD_ERR_ARG;
    cudaSetDevice(c->dev);
    const lyd_step_params *p = &cfg->step;
    if (c->ncl != 1) return fail(c, LYD_ERR_STATE, "the adjoint runs on a single-cloud context");
    if (c->prec != LYD_PREC_FP64) return fail(c, LYD_ERR_STATE, "the adjoint runs in LYD_PREC_FP64");
    if (c->aF) return fail(c, LYD_ERR_STATE, "the adjoint needs alpha_F derived from alpha and H_voigt");
    LYD_TRY(check_bcs(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top));
    if (!(p->c_tilde > 0.0) || !(p->dt > 0.0) || p->n_steps < 1) return fail(c, LYD_ERR_ARG, "bad step parameters");
    LYD_TRY(need_inputs(c, true, true));
    const int N = p->n_steps;
    const size_t n3 = c->n3, nc = c->ncell, S = 3 * n3;
    // checkpoint_every 1, or 0 when every step's state and advection tape fit in free device
    // memory: the forward sweep keeps them all and the reverse sweep recomputes nothing.
    // Otherwise a checkpoint every K steps (0: 100) and one recomputation of each segment.
    // When there is room, every step's frequency factors are kept too (3 more doubles per
    // cell-bin), and the frequency-step adjoint reads them instead of recomputing them.
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) { cudaGetLastError(); fr = 0; }
    const size_t avail = fr + c->adj_ws_bytes, margin = 16 * S * 8 + ((size_t)2 << 30);
    // checkpoint_every < 0: the binomial schedule with `snapshots` state snapshots (0: the fewest
    // for which no step is advanced more than twice in the reverse sweep)
    const bool binom = cfg->checkpoint_every < 0;
    bool store_all = cfg->checkpoint_every == 1;
    if (cfg->checkpoint_every == 0) store_all = (size_t)N * (S + 4 * n3) * 8 + margin <= avail;
    const bool keep_ff = store_all && (size_t)N * (S + 7 * n3) * 8 + margin <= avail;
    int snaps = 0;
    if (binom) {
        if (cfg->snapshots < 0) return fail(c, LYD_ERR_ARG, "snapshots must be >= 0");
        snaps = cfg->snapshots > 0 ? cfg->snapshots : 1;
        if (cfg->snapshots == 0)
            while (binomial_reach(snaps + 1, 2) < (double)N) snaps++;
        if (snaps > N) snaps = N;
    }
    const int K = binom ? 1
                        : store_all ? 1
                                    : (cfg->checkpoint_every > 0 ? (cfg->checkpoint_every < N ? cfg->checkpoint_every : N)
                                                                 : (N < 100 ? N : 100));
    const int nseg = binom ? snaps + 1 : (N + K - 1) / K;
    const int nr = c->nr[0], nz = c->nz[0], nnu = c->nnu;
    params_all(c, p->c_tilde, p->dt, p->c_tilde * p->dt);
    for (CloudDesc &d : c->desc) d.z_center = p->z_center;
    bcs_all(c, c->cfg.bc_r_left, p->bc_r_right, p->bc_z_bot, p->bc_z_top);
    LYD_TRY(sync_desc(c));
    if (N > c->hist_cap) {
        LYD_CU(c, cudaStreamSynchronize(c->st));
        cudaFree(c->hist);
        c->hist = nullptr;
        c->hist_cap = 0;
        LYD_TRY(dalloc(c, (void **)&c->hist, (size_t)N * 7 * 8));
        c->hist_cap = N;
        drop_graph(c);
    }
    // One workspace, kept in the context between calls. It holds: the checkpoints (every
    // step's state when all are kept); per step of one segment the state (recomputation only);
    // the advected state of the step being recomputed; the advection tapes (of every step when
    // all are kept, else of one segment, recorded while it is recomputed); the adjoints; and
    // the gradient accumulators (zeroed here).
    const size_t ntape = store_all ? (size_t)N : (size_t)K;
    // With phase timing off, the recomputation runs on a second stream beside the reverse
    // sweep, into a second buffer of states and tapes (when it fits): with uniform segments
    // segment g-1 is recomputed while segment g is reversed; in the binomial schedule every
    // advance and record runs ahead of the reversals, one step's record per buffer.
    bool overlap = !store_all && (binom || nseg >= 2) && !c->timing;
    constexpr int NB = 24;
    size_t offs[NB], total = 0;
    for (;;) {
        const size_t ov = overlap ? 1 : 0;
        const size_t sizes[NB] = {(size_t)nseg * S * 8, store_all ? 0 : (size_t)K * S * 8, S * 8, ntape * 4 * n3 * 8,
                                  S * 8, S * 8, S * 8, S * 8, n3 * 8, n3 * 8, nc * 8, nc * 8, nc * 8, 5 * nc * 8,
                                  c->nrf * 8, c->nzf * 8, S * 8, (size_t)nnu * 8,
                                  2 * (size_t)nnu * (nr + nz + 2 * nr) * 8, (size_t)N * 2 * sizeof(int) + 16, 16,
                                  keep_ff ? (size_t)N * 3 * n3 * 8 : 0, ov * K * S * 8, ov * K * 4 * n3 * 8};
        total = 0;
        for (int q = 0; q < NB; q++) {
            offs[q] = total;
            total += (sizes[q] + 255) / 256 * 256;
        }
        if (!overlap || total + margin <= avail) break;
        overlap = false;
    }
    if (total > c->adj_ws_bytes) {
        LYD_CU(c, cudaStreamSynchronize(c->st));
        cudaFree(c->adj_ws);
        c->adj_ws = nullptr;
        c->adj_ws_bytes = 0;
        if (cudaMalloc(&c->adj_ws, total) != cudaSuccess) {
            cudaGetLastError();
            c->adj_ws = nullptr;
            return fail(c, LYD_ERR_NOMEM, "adjoint workspace: out of device memory (lower checkpoint_every)");
        }
        c->adj_ws_bytes = total;
    }
    auto W_ = [&](int q) { return reinterpret_cast<double *>(static_cast<char *>(c->adj_ws) + offs[q]); };
    double *ck = W_(0), *seg = W_(1), *segA = W_(2), *segT = W_(3);
    double *lam = W_(4), *lamA = W_(5), *lamN = W_(6), *pre = W_(7), *gaF = W_(8), *gHv = W_(9);
    double *g_alpha = W_(10), *g_alpha_c = W_(11), *g_T = W_(12), *g_u = W_(13);
    double *g_ur = W_(14), *g_uZ = W_(15), *fin = W_(16), *wsp = W_(17), *edge = W_(18);
    int *win = reinterpret_cast<int *>(W_(19));
    int *finwin = reinterpret_cast<int *>(W_(20));
    double *ffs = keep_ff ? W_(21) : nullptr;
    double *segB[2] = {seg, overlap ? W_(22) : nullptr}, *segTB[2] = {segT, overlap ? W_(23) : nullptr};
    // lambda and the accumulators start at zero (buffers 4 and 8..15 are contiguous in order)
    LYD_CU(c, cudaMemsetAsync(lam, 0, S * 8, c->st));
    LYD_CU(c, cudaMemsetAsync(gaF, 0, offs[16] - offs[8], c->st));
    auto copy_state = [&](double *dst, int set, cudaStream_t s = nullptr) -> int {
        for (int q = 0; q < 3; q++)
            LYD_CU(c, cudaMemcpyAsync(dst + q * n3, c->set[set][q], n3 * 8, cudaMemcpyDeviceToDevice, s ? s : c->st));
        return LYD_OK;
    };
    auto load_state = [&](const double *src, int set, cudaStream_t s = nullptr) -> int {
        for (int q = 0; q < 3; q++)
            LYD_CU(c, cudaMemcpyAsync(c->set[set][q], src + q * n3, n3 * 8, cudaMemcpyDeviceToDevice, s ? s : c->st));
        return LYD_OK;
    };
    // phase timing (lyd_set_timing): events around the forward sweep and every reverse phase
    const bool tm = c->timing;
    double acc[5] = {0, 0, 0, 0, 0};
    auto tick = [&](int e) { if (tm) cudaEventRecord(c->ev[e], c->st); };
    auto tock = [&](int e0, int e1, int slot) {
        if (!tm) return;
        cudaEventSynchronize(c->ev[e1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev[e0], c->ev[e1]);
        acc[slot] += ms;
    };
    // ---- forward sweep ----
    tick(0);
    LYD_CU(c, cudaMemsetAsync(c->step_ctr, 0, 2 * sizeof(int), c->st));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_R], 0, nc * 8, c->st));
    LYD_CU(c, cudaMemsetAsync(c->cellf[CF_DRU_Z], 0, nc * 8, c->st));
    if (!c->active_valid) LYD_TRY(run_find_active(c));
    // win[2n..2n+1] is step n's window: step 0's is copied here, each step's reduction writes
    // the next one's beside the context's own (no copy between the steps' kernels)
    LYD_CU(c, cudaMemcpyAsync(win, c->kwin, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    if (store_all) {
        // every state lives in the checkpoint storage: step n reads slot n and writes slot n + 1
        // (the last step writes the context's state)
        LYD_TRY(copy_state(ck, c->cur));
        for (int n = 0; n < N; n++) {
            double *out = n + 1 < N ? ck + (size_t)(n + 1) * S : nullptr;
            LYD_TRY(enqueue_step<double>(c, false, segT + (size_t)n * 4 * n3, ck + (size_t)n * S, out,
                                         ffs ? ffs + (size_t)n * 3 * n3 : nullptr, true,
                                         n + 1 < N ? win + 2 * (n + 1) : nullptr));
        }
    } else {
        for (int n = 0; n < N; n++) {
            if (binom ? n == 0 : n % K == 0) LYD_TRY(copy_state(ck + (size_t)(n / K) * S, c->cur));
            LYD_TRY(enqueue_step<double>(c, false, nullptr, nullptr, nullptr, nullptr, true,
                                         n + 1 < N ? win + 2 * (n + 1) : nullptr));
        }
    }
    LYD_TRY(copy_state(fin, c->cur));
    LYD_CU(c, cudaMemcpyAsync(finwin, c->kwin, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    tick(1);
    tock(0, 1, 0);
    std::vector<int> hwin((size_t)2 * N);
    std::vector<double> rec(7);
    LYD_CU(c, cudaMemcpyAsync(hwin.data(), win, hwin.size() * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    LYD_CU(c, cudaMemcpyAsync(rec.data(), c->hist + (size_t)(N - 1) * 7, 7 * 8, cudaMemcpyDeviceToHost, c->st));
    LYD_TRY(check_err(c));
    // objective: w_MF M_F(last step) + sum_k w_k S_k, S = edge-ring mean of the final J
    const int ne = lyd_edge_count(nr, nz);
    std::vector<double> spec(nnu, 0.0);
    if (ne > 0) {
        std::vector<double> raw((size_t)ne * nnu);
        launch_edge(c->sprec, Jc(c, 0), c->dnu, nnu, nr, nz, c->jscale, edge, edge + (size_t)ne * nnu, c->st);
        LYD_CU(c, cudaMemcpyAsync(raw.data(), edge, raw.size() * 8, cudaMemcpyDeviceToHost, c->st));
        LYD_CU(c, cudaStreamSynchronize(c->st));
        for (int e = 0; e < ne; e++)
            for (int k = 0; k < nnu; k++) spec[k] += raw[(size_t)e * nnu + k] / ne;
    }
    double obj = cfg->w_MF * rec[0];
    if (cfg->w_spec)
        for (int k = 0; k < nnu; k++) obj += cfg->w_spec[k] * spec[k];
    if (out->objective) *out->objective = obj;
    if (out->M_F) *out->M_F = rec[0];
    if (out->spectrum)
        for (int k = 0; k < nnu; k++) out->spectrum[k] = spec[k];
    // L of the normalisation: the record holds L_tot (x2 with a reflecting bottom)
    const double Lsim = (p->bc_z_bot == LYD_BC_REFLECT) ? 0.5 * rec[3] : rec[3];
    const double mf_w = (Lsim > 0.0) ? cfg->w_MF * kC / Lsim : 0.0;
    // ---- reverse sweep ----
    if (cfg->w_spec && ne > 0) {
        LYD_CU(c, cudaMemcpyAsync(wsp, cfg->w_spec, nnu * 8, cudaMemcpyHostToDevice, c->st));
        launch_seed_spectrum(lam, wsp, nnu, nr, nz, c->st);
    }
    const int B = 1 - c->cur;
    // One step forward from the state in the context's current set (or from `sn`, which then
    // receives a copy of it), in the forward sweep's window of step n: the advection into x_A,
    // with its tape when `tape` is given, then (with `freq`) emission + frequency step x_A -> the
    // current set. On stream `s` (the context's stream when null).
    auto forward_step = [&](int n, double *sn, double *tape, bool freq, cudaStream_t s = nullptr) -> int {
        if (!s) s = c->st;
        double *xA = segA;
        AdvArgs<double> aa;
        fill_adv<double>(c, aa, c->cur, B);
        if (sn) {
            LYD_TRY(copy_state(sn, c->cur, s));
            aa.J = sn; aa.Hr = sn + n3; aa.HZ = sn + 2 * n3;
            aa.tmaps = nullptr;     // the maps cover the context's buffer sets, not the workspace
        }
        aa.Jo = xA; aa.Hro = xA + n3; aa.HZo = xA + 2 * n3;
        aa.kwin = win + 2 * n;
        aa.tape = tape;
        aa.tape_stride = (long long)n3;
        launch_advect(LYD_PREC_FP64, c->cfg.flux_method, &aa, c->ntiles, 2, s);
        if (freq) {
            FreqArgs<double> fq;
            fill_freq<double>(c, fq, xA, xA + n3, xA + 2 * n3, xA, c->set[c->cur][0], c->set[c->cur][1],
                              c->set[c->cur][2]);
            fq.do_emission = 1; fq.do_freq = 1; fq.update_ff = 1;
            fq.parts = 0;
            launch_freq(LYD_PREC_FP64, &fq, nnu, c->nitems, s);
        }
        LYD_CU(c, cudaGetLastError());
        return LYD_OK;
    };
    // The adjoint of step n from its input state sn and advection tape: lambda_{n+1} -> lambda_n.
    auto reverse_step = [&](int n, const double *sn, const double *tape) -> int {
        tick(2);
        tick(3);
        // frequency step adjoint: lambda_{n+1} -> lambda of x_A
        FreqAdjArgs fa;
        memset(&fa, 0, sizeof(fa));
        fa.J = sn; fa.Hr = sn + n3; fa.HZ = sn + 2 * n3;
        fa.tape = tape; fa.tape_stride = (long long)n3;
        fa.kmin = hwin[2 * n]; fa.kmax = hwin[2 * n + 1];
        if (ffs) {
            fa.Fkp = ffs + (size_t)n * 3 * n3;
            fa.Fk = fa.Fkp + n3;
            fa.Fkm = fa.Fkp + 2 * n3;
        }
        fa.Hv = (const double *)c->Hv;
        fa.phi = c->phi ? (const double *)c->phi : nullptr;
        fa.phi_inv = c->phi_inv; fa.phi_kmin = c->phi_kmin; fa.phi_kmax = c->phi_kmax;
        fa.alpha = c->cellf[CF_ALPHA]; fa.alpha_c = c->cellf[CF_ALPHA_C];
        fa.alpha_cF = any_have(c, 1u << CF_ALPHA_CF) ? c->cellf[CF_ALPHA_CF] : nullptr;
        fa.pd = c->cellf[CF_PD]; fa.js = c->cellf[CF_JS]; fa.T = c->cellf[CF_T];
        fa.dur_dr = c->cellf[CF_DUR_DR]; fa.dur_dZ = c->cellf[CF_DUR_DZ]; fa.duZ_dr = c->cellf[CF_DUZ_DR];
        fa.duZ_dZ = c->cellf[CF_DUZ_DZ]; fa.ur_over_r = c->cellf[CF_UR_OVER_R];
        fa.nu = c->nu; fa.nuC = c->nuC; fa.dnu = c->dnu; fa.inv_dnu = c->inv_dnu; fa.inv_nuC = c->inv_nuC;
        fa.dV = c->dV; fa.cl = c->cl; fa.items = c->items;
        fa.alpha_floor = c->cfg.alpha_floor; fa.jeps = c->jeps_s; fa.heps2 = c->heps2_s; fa.j_scale = c->jscale;
        fa.recoil = c->cfg.recoil; fa.nnu = nnu; fa.ncell = (long long)nc;
        fa.gJ = lam; fa.gHr = lam + n3; fa.gHZ = lam + 2 * n3;
        fa.oJ = lamA; fa.oHr = lamA + n3; fa.oHZ = lamA + 2 * n3;
        fa.g_alpha = g_alpha; fa.g_alpha_c = g_alpha_c; fa.g_T = g_T; fa.g_u = g_u; fa.g_Hv = gHv;
        fa.mf_seed = (n == N - 1) && mf_w != 0.0;
        fa.mf_w = mf_w;
        launch_freq_adj(fa, c->nitems, c->st);
        tick(4);
        // advection adjoint: lambda of x_A -> lambda_n
        AdjAdvArgs ad;
        memset(&ad, 0, sizeof(ad));
        ad.J = sn; ad.Hr = sn + n3; ad.HZ = sn + 2 * n3;
        ad.tape = tape; ad.n3 = (long long)n3;
        ad.gJ = lamA; ad.gHr = lamA + n3; ad.gHZ = lamA + 2 * n3;
        ad.lJ = lamN; ad.lHr = lamN + n3; ad.lHZ = lamN + 2 * n3;
        ad.pJ = pre; ad.pHr = pre + n3; ad.pHZ = pre + 2 * n3;
        ad.Hv = (const double *)c->Hv; ad.alpha = c->cellf[CF_ALPHA]; ad.alpha_cF = fa.alpha_cF;
        ad.A_r = c->A_r; ad.A_Z = c->A_Z; ad.inv_dV = c->inv_dV; ad.inv_r_cell = c->inv_r_cell;
        ad.rint = c->rint; ad.zint = c->zint; ad.u_r_star = c->u_r_star; ad.u_Z_star = c->u_Z_star;
        ad.dur_dr = fa.dur_dr; ad.dur_dZ = fa.dur_dZ; ad.duZ_dr = fa.duZ_dr; ad.duZ_dZ = fa.duZ_dZ;
        ad.ur_over_r = fa.ur_over_r;
        ad.g_aF = gaF; ad.g_u = g_u; ad.g_ur = g_ur; ad.g_uZ = g_uZ;
        ad.nnu = nnu; ad.nr = nr; ad.nz = nz; ad.kmin = hwin[2 * n]; ad.kmax = hwin[2 * n + 1];
        ad.bc_r_left = c->cfg.bc_r_left;
        ad.bc_r_right = p->bc_r_right; ad.bc_z_bot = p->bc_z_bot; ad.bc_z_top = p->bc_z_top;
        ad.ctdt = p->c_tilde * p->dt; ad.jeps = c->jeps_s; ad.heps2 = c->heps2_s;
        ad.flux = c->cfg.flux_method == LYD_FLUX_HLL ? 1 : 0;
        launch_adv_adj(ad, c->st);
        tick(5);
        tock(2, 3, 2);
        tock(3, 4, 3);
        tock(4, 5, 4);
        LYD_CU(c, cudaGetLastError());
        double *t = lam;
        lam = lamN;
        lamN = t;
        return LYD_OK;
    };
    // the recomputation stream starts once the forward sweep and the seeds are done
    if (overlap && !c->st_rec) {
        LYD_CU(c, cudaStreamCreateWithFlags(&c->st_rec, cudaStreamNonBlocking));
        for (cudaEvent_t &e : c->adj_ev) LYD_CU(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaEvent_t *ev_rec = c->adj_ev, *ev_rev = c->adj_ev + 2;
    StreamDrain drain{c};
    if (overlap) {
        drain.armed = true;
        LYD_CU(c, cudaEventRecord(c->adj_ev[4], c->st));
        LYD_CU(c, cudaStreamWaitEvent(c->st_rec, c->adj_ev[4], 0));
    }
    // the stream of the forward work of the reverse sweep (advances, snapshots, records)
    cudaStream_t fs = overlap ? c->st_rec : c->st;
    if (!binom && overlap) {
        // segment g's states and tapes go to buffer g & 1, recomputed on the recomputation stream:
        // reversal g waits for recomputation g, and recomputation g - 2 (into the same buffer)
        // for reversal g, so recomputation g - 1 runs beside reversal g
        auto recompute = [&](int g) -> int {
            const int n0 = g * K, n1 = (n0 + K < N) ? n0 + K : N;
            double *sb = segB[g & 1], *tb = segTB[g & 1];
            LYD_TRY(load_state(ck + (size_t)g * S, c->cur, c->st_rec));
            for (int n = n0; n < n1; n++)
                LYD_TRY(forward_step(n, sb + (size_t)(n - n0) * S, tb + (size_t)(n - n0) * 4 * n3, n + 1 < n1,
                                     c->st_rec));
            LYD_CU(c, cudaEventRecord(ev_rec[g & 1], c->st_rec));
            return LYD_OK;
        };
        LYD_TRY(recompute(nseg - 1));
        LYD_TRY(recompute(nseg - 2));
        for (int g = nseg - 1; g >= 0; g--) {
            const int n0 = g * K, n1 = (n0 + K < N) ? n0 + K : N;
            LYD_CU(c, cudaStreamWaitEvent(c->st, ev_rec[g & 1], 0));
            for (int n = n1 - 1; n >= n0; n--)
                LYD_TRY(reverse_step(n, segB[g & 1] + (size_t)(n - n0) * S, segTB[g & 1] + (size_t)(n - n0) * 4 * n3));
            if (g >= 2) {
                LYD_CU(c, cudaEventRecord(ev_rev[g & 1], c->st));
                LYD_CU(c, cudaStreamWaitEvent(c->st_rec, ev_rev[g & 1], 0));
                LYD_TRY(recompute(g - 2));
            }
        }
    } else if (!binom) {
        for (int g = nseg - 1; g >= 0; g--) {
            const int n0 = g * K, n1 = (n0 + K < N) ? n0 + K : N;
            if (!store_all) {
                tick(0);
                LYD_TRY(load_state(ck + (size_t)g * S, c->cur));
                // recompute the segment, recording every step's input state and advection tape
                for (int n = n0; n < n1; n++)
                    LYD_TRY(forward_step(n, seg + (size_t)(n - n0) * S, segT + (size_t)(n - n0) * 4 * n3, n + 1 < n1));
                tick(1);
                tock(0, 1, 1);
            }
            for (int n = n1 - 1; n >= n0; n--) {
                const double *sn = store_all ? ck + (size_t)n * S : seg + (size_t)(n - n0) * S;
                const double *tape = segT + (size_t)(store_all ? n : n - n0) * 4 * n3;
                LYD_TRY(reverse_step(n, sn, tape));
            }
        }
    } else {
        // Binomial checkpointing (Griewank's Revolve schedule): reverse steps [i0, i1) with the
        // state s_i0 in snapshot `slot` and `nfree` more snapshots, s = nfree + 1 in all. With r
        // the least repetition number for which C(s + r, s) >= i1 - i0, the next snapshot goes
        // t steps ahead, t the least with i1 - i0 - t <= C(s - 1 + r, s - 1): the steps right
        // of it are reversed with one snapshot fewer and up to r advances, those left of it
        // (advanced once to place it) with the same snapshots and r - 1, so no step is advanced
        // more than r times. Each step is recorded (its input state and tape) right before its
        // reverse.
        // Advances, snapshot copies and records go to `fs`. Overlapped, step n records into
        // buffer n & 1 once reversal n + 2 (its last reader) is done, and reversal n waits for
        // that record: the advances and records of the next steps run beside the reversals.
        auto advance = [&](int slot, int i0, int n_to) -> int {
            tick(0);
            LYD_TRY(load_state(ck + (size_t)slot * S, c->cur, fs));
            for (int n = i0; n < n_to; n++) LYD_TRY(forward_step(n, nullptr, nullptr, true, fs));
            tick(1);
            tock(0, 1, 1);
            return LYD_OK;
        };
        auto record_and_reverse = [&](int n) -> int {
            double *sb = segB[overlap ? (n & 1) : 0], *tb = segTB[overlap ? (n & 1) : 0];
            tick(0);
            if (overlap) LYD_CU(c, cudaStreamWaitEvent(fs, ev_rev[n & 1], 0));
            LYD_TRY(forward_step(n, sb, tb, false, fs));
            if (overlap) {
                LYD_CU(c, cudaEventRecord(ev_rec[n & 1], fs));
                LYD_CU(c, cudaStreamWaitEvent(c->st, ev_rec[n & 1], 0));
            }
            tick(1);
            tock(0, 1, 1);
            LYD_TRY(reverse_step(n, sb, tb));
            if (overlap) LYD_CU(c, cudaEventRecord(ev_rev[n & 1], c->st));
            return LYD_OK;
        };
        std::function<int(int, int, int, int)> rev = [&](int i0, int i1, int slot, int nfree) -> int {
            const int l = i1 - i0;
            if (l == 1) {
                LYD_TRY(advance(slot, i0, i0));
                return record_and_reverse(i0);
            }
            if (nfree == 0) {
                for (int n = i1 - 1; n >= i0; n--) {
                    LYD_TRY(advance(slot, i0, n));
                    LYD_TRY(record_and_reverse(n));
                }
                return LYD_OK;
            }
            int r = 1;
            while (binomial_reach(nfree + 1, r) < (double)l) r++;
            int t = l - (int)std::min((double)(l - 1), binomial_reach(nfree, r));
            if (t < 1) t = 1;
            LYD_TRY(advance(slot, i0, i0 + t));
            LYD_TRY(copy_state(ck + (size_t)(slot + 1) * S, c->cur, fs));
            LYD_TRY(rev(i0 + t, i1, slot + 1, nfree - 1));
            return rev(i0, i0 + t, slot, nfree);
        };
        LYD_TRY(rev(0, N, 0, snaps));
    }
    drain.armed = false;
    // alpha_F = alpha H_voigt ; H_voigt(T) when it was computed on the device
    launch_af_params(gaF, c->cellf[CF_ALPHA], (const double *)c->Hv, nnu, (long long)nc, g_alpha, gHv, c->st);
    if (c->hv_from_T && c->lut)
        launch_hvoigt_adj(gHv, c->cellf[CF_T], c->nu, c->nuC, nnu, (long long)nc, c->lut, kLutN, kLutXmax, g_T, c->st);
    LYD_CU(c, cudaGetLastError());
    auto down = [&](double *host, const double *dev, size_t n) -> int {
        if (host) LYD_CU(c, cudaMemcpyAsync(host, dev, n * 8, cudaMemcpyDeviceToHost, c->st));
        return LYD_OK;
    };
    LYD_TRY(down(out->grad_alpha, g_alpha, nc));
    LYD_TRY(down(out->grad_alpha_c, g_alpha_c, nc));
    LYD_TRY(down(out->grad_T, g_T, nc));
    LYD_TRY(down(out->grad_Hv, gHv, n3));
    LYD_TRY(down(out->grad_u_r_star, g_ur, c->nrf));
    LYD_TRY(down(out->grad_u_Z_star, g_uZ, c->nzf));
    for (int q = 0; q < 5; q++) LYD_TRY(down(out->grad_du[q], g_u + (size_t)q * nc, nc));
    // lambda of the initial state, back in the caller's units (the state is held as value / j_scale)
    LYD_TRY(down(out->grad_J0, lam, n3));
    LYD_TRY(down(out->grad_H_r0, lam + n3, n3));
    LYD_TRY(down(out->grad_H_Z0, lam + 2 * n3, n3));
    if (tm)
        for (int q = 0; q < 5; q++) c->adj_ms[q] = acc[q];
    // the context ends in the forward sweep's final state
    LYD_TRY(load_state(fin, c->cur));
    LYD_CU(c, cudaMemcpyAsync(c->kwin, finwin, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    c->old_alias = true;
    c->active_valid = true;
    return check_err(c);
}

int lyd_get_adjoint_timing(lyd_ctx *c, double ms[5]) {
    if (!c || !ms) return LYD_ERR_ARG;
    for (int q = 0; q < 5; q++) ms[q] = c->adj_ms[q];
    return LYD_OK;
}
