// abi.cpp -- the C ABI of libldsc_b200 (include/ldsc_b200.h): contexts,
// resident panels, and the l2 run that replaces compute_ldscore_global
// (reference src/l2/compute.rs:1009-2447) plus its per-chromosome fan-out
// (src/l2/mod.rs:439-575).
//
// One l2 run on the device:
//   1. host plan: per-record left window limits (plan.cpp) and band tiles;
//   2. decode: per-record integer moments, and the operand panel of the
//      chosen form (INT8 genotype/mask rows, standardised f64 rows, or
//      CountSketch f32 rows);
//   3. finalise: MAF, standardisation constants, pq-scaled annotation, and
//      l2 seeded with the diagonal term;
//   4. band Gram with the r^2 epilogue accumulating l2 in f64;
//   5. copy l2 / MAF back.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ldsc_b200.h"
#include "engine.h"
#include "plan.h"
#include "regress.h"

using namespace ldsc;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    // Context workspace is allocated stream-ordered on the context's stream
    // (from the device's memory pool): growing or freeing it then does not
    // wait for other contexts' work, as cudaFree would.
    cudaStream_t* owner = nullptr;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        release();
        if (bytes == 0) bytes = 16;
        cudaError_t e = owner ? cudaMallocAsync(&p, bytes, *owner) : cudaMalloc(&p, bytes);
        if (e == cudaSuccess) {
            cap = bytes;
        } else {
            p = nullptr;
            cudaGetLastError();
        }
        return e;
    }
    void release() {
        if (p) {
            if (owner)
                cudaFreeAsync(p, *owner);
            else
                cudaFree(p);
        }
        p = nullptr;
        cap = 0;
    }
    template <typename T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Instantiated CUDA graphs of fixed launch sequences, keyed by everything
// their kernels' parameters depend on (sizes and buffer addresses).
struct GraphCache {
    struct Entry {
        std::vector<uint64_t> key;
        cudaGraphExec_t exec = nullptr;
        uint64_t tick = 0;
    };
    std::vector<Entry> e;
    uint64_t tick = 0;
    void clear() {
        for (auto& x : e)
            if (x.exec) cudaGraphExecDestroy(x.exec);
        e.clear();
    }
};

// Bucket-major CountSketch layout of a panel: the individuals' order, the
// segment tables and the panel rows rewritten in that order.
struct SketchCache {
    DevBuf perm, seg, segt, pp;
    uint64_t n = 0, key = 0, pitch_words = 0;
    uint32_t d = 0;
    bool valid = false;
    bool matches(uint64_t n_, uint32_t d_, uint64_t key_) const { return valid && n == n_ && d == d_ && key == key_; }
    void release() {
        perm.release();
        seg.release();
        segt.release();
        pp.release();
        valid = false;
    }
};

}  // namespace

struct ldsc_ctx {
    int device = 0;
    uint32_t flags = 0;
    int sms = 148;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t copy = nullptr;  // host-to-device BED stream of ldsc_l2_from_bed
    cudaStream_t side = nullptr;  // low-priority stream of the decode that overlaps the Gram
    std::vector<cudaEvent_t> ovl_ev;  // per decoded record chunk
    cudaEvent_t ovl_go = nullptr;
    std::mutex mu;
    std::string last_error;
    uint64_t kernels = 0;
    // workspace (grow-only)
    DevBuf ops, xf64, xsk, recrows, keep, left, tiles, annot, aeff, l2, maf, pq, err;
    DevBuf st_n, st_s, st_q, st_q3, st_q4, st_mean, st_inv, st_qinv, st_kappa, packed, tsum, dbg;
    // private CountSketch layout (explicit bucket/sign arrays, or a panel
    // whose shared layout is in use under another key)
    SketchCache sk;
    uint64_t sk_panel = 0;
    GraphCache graphs;            // regression pipelines
    uint64_t graph_launches = 0;  // replays of cached graphs
    DevBuf rtiles, cptr_r, cidx_r, cptr_l, cidx_l;  // K > 1 contraction: r2u tiles and CSR tile lists
    DevBuf prow, pcol;                              // K = 1: per-tile row / column sums
    DevBuf rg_jobs, rg_states, rg_outs, rg_part, rg_tdel, rg_y, rg_y2, rg_n, rg_ld, rg_wld, rg_sel, rg_pairs, rg_res;
    DevBuf ts_seps, ts_n1, ts_cnt, ts_dv, ts_outs;  // --two-step
    // partitioned h2
    DevBuf p_l2, p_w, p_y, p_n, p_m, p_rjobs, p_seps, p_n1, p_cnt, p_jobs, p_st, p_xtot, p_part, p_gram, p_tot,
        p_sol, p_res;
    // the host plan of the last l2 call, kept so the next one reuses its pages
    LeftLimits plan_left;
    std::vector<Tile> plan_tiles;
    std::vector<int32_t> plan_ptr_r, plan_idx_r, plan_ptr_l, plan_idx_l;  // CSR tile lists
    // whole-file entry: staged file rows, the pitched panel, per-chunk events
    DevBuf bed_stage, bed_rows;
    std::vector<cudaEvent_t> feed_ev;
    cudaEvent_t feed_t0 = nullptr, feed_t1 = nullptr, feed_go = nullptr, up_ev = nullptr;

    std::vector<DevBuf*> workspace() {
        return {&ops, &xf64, &xsk, &recrows, &keep, &left,
                      &tiles, &annot, &aeff, &l2, &maf,
                      &pq, &err, &st_n, &st_s, &st_q, &st_q3,
                      &st_q4, &st_mean, &st_inv, &st_qinv, &st_kappa,
                      &packed, &tsum, &dbg,
                      &rtiles, &cptr_r, &cidx_r, &cptr_l, &cidx_l, &prow, &pcol,
                      &rg_jobs, &rg_states, &rg_outs, &rg_part, &rg_tdel,
                      &rg_y, &rg_y2, &rg_n, &rg_ld, &rg_wld, &rg_sel,
                      &rg_pairs, &rg_res, &bed_stage, &bed_rows, &ts_seps, &ts_n1, &ts_cnt, &ts_dv, &ts_outs,
                      &p_l2, &p_w, &p_y, &p_n, &p_m, &p_rjobs, &p_seps, &p_n1, &p_cnt, &p_jobs,
                      &p_st, &p_xtot, &p_part, &p_gram, &p_tot, &p_sol, &p_res};
    }
};

struct ldsc_panel {
    ldsc_ctx* ctx = nullptr;
    uint8_t* rows = nullptr;
    uint64_t n_snp = 0, n_indiv = 0, bpr = 0, pitch = 0;
    uint64_t id = 0;  // unique per panel, keys the contexts' private sketch layouts
    // shared CountSketch layout, usable by every context on the device;
    // rebuilt only while no run is using it
    mutable std::mutex mu;
    mutable SketchCache sk;
    mutable int sk_users = 0;
};

static std::atomic<uint64_t> g_panel_ids{1};

static int fail(ldsc_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

static int cuda_fail(ldsc_ctx* ctx, cudaError_t e, const char* what) {
    const int code = e == cudaErrorMemoryAllocation ? LDSC_E_NOMEM : LDSC_E_CUDA;
    cudaGetLastError();  // clear sticky-free errors
    return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

extern "C" {

int ldsc_abi_version(void) { return LDSC_B200_ABI_VERSION; }

int ldsc_ctx_create(int device, uint32_t flags, ldsc_ctx** out) {
    if (!out || (flags & ~LDSC_CTX_FUSED_OPERANDS)) return LDSC_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return LDSC_E_CUDA;
    }
    if (device < 0 || device >= n) return LDSC_E_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return LDSC_E_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return LDSC_E_CUDA;
    if (prop.major != 10) return LDSC_E_UNSUPPORTED;  // sm_100a kernels only
    {
        // every kernel of the library is loaded on this device before the
        // context's first launch (a lazy load in the middle of a run can stall
        // the work of other contexts on the device)
        static std::mutex preload_mu;
        static std::vector<int> preloaded;
        std::lock_guard<std::mutex> g(preload_mu);
        if (std::find(preloaded.begin(), preloaded.end(), device) == preloaded.end()) {
            for (cudaError_t (*f)() : {preload_gram_tc, preload_gram_simt, preload_decode, preload_sketch,
                                       preload_contract, preload_synth, preload_regress, preload_partitioned})
                if (f() != cudaSuccess) {
                    cudaGetLastError();
                    return LDSC_E_CUDA;
                }
            preloaded.push_back(device);
        }
    }
    ldsc_ctx* c = new ldsc_ctx();
    c->device = device;
    c->flags = flags;
    c->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) {
        if (c->own) cudaStreamDestroy(c->own);
        delete c;
        return LDSC_E_CUDA;
    }
    c->stream = c->own;
    for (DevBuf* b : c->workspace()) b->owner = &c->stream;
    for (DevBuf* b : {&c->sk.perm, &c->sk.seg, &c->sk.segt, &c->sk.pp}) b->owner = &c->stream;
    // keep freed workspace in the pool for the next call instead of returning it
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep_all = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
    }
    cudaGetLastError();
    *out = c;
    return LDSC_OK;
}

int ldsc_ctx_destroy(ldsc_ctx* ctx) {
    if (!ctx) return LDSC_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    std::vector<DevBuf*> bufs = ctx->workspace();
    cudaStreamSynchronize(ctx->copy);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    for (DevBuf* b : bufs) b->release();
    ctx->sk.release();
    ctx->graphs.clear();
    cudaStreamSynchronize(ctx->stream);
    for (cudaEvent_t e : ctx->feed_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->ovl_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : {ctx->feed_t0, ctx->feed_t1, ctx->feed_go, ctx->up_ev, ctx->ovl_go})
        if (e) cudaEventDestroy(e);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->copy) cudaStreamDestroy(ctx->copy);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return LDSC_OK;
}

int ldsc_ctx_set_stream(ldsc_ctx* ctx, void* s) {
    if (!ctx) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->stream = s ? reinterpret_cast<cudaStream_t>(s) : ctx->own;
    return LDSC_OK;
}

int ldsc_last_error(const ldsc_ctx* ctx, char* buf, size_t len) {
    if (!buf || len == 0) return LDSC_E_INVALID;
    const std::string& s = ctx ? ctx->last_error : std::string("null context");
    std::snprintf(buf, len, "%s", s.c_str());
    return LDSC_OK;
}

uint64_t ldsc_ctx_kernel_count(const ldsc_ctx* ctx) { return ctx ? ctx->kernels : 0; }

uint64_t ldsc_ctx_graph_launches(const ldsc_ctx* ctx) { return ctx ? ctx->graph_launches : 0; }

int ldsc_ctx_trim(ldsc_ctx* ctx) {
    if (!ctx) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->copy);
    ctx->graphs.clear();  // their kernels hold the buffers' addresses
    for (DevBuf* b : ctx->workspace()) b->release();
    ctx->sk.release();
    ctx->sk_panel = 0;
    return LDSC_OK;
}

int ldsc_panel_shape(const ldsc_panel* p, uint64_t* n_indiv, uint64_t* n_snp) {
    if (!p) return LDSC_E_INVALID;
    if (n_indiv) *n_indiv = p->n_indiv;
    if (n_snp) *n_snp = p->n_snp;
    return LDSC_OK;
}

int ldsc_bed_validate(const uint8_t* bed, uint64_t len, uint64_t n_indiv, uint64_t n_snp, char* err,
                      size_t errlen) {
    auto set = [&](const std::string& m) {
        if (err && errlen) std::snprintf(err, errlen, "%s", m.c_str());
        return LDSC_E_BED;
    };
    if (len < 3) return set("BED too short (" + std::to_string(len) + "B)");
    if (!bed) return set("BED buffer is null");
    if (bed[0] != 0x6c || bed[1] != 0x1b) return set("BED has invalid magic bytes");
    if (bed[2] != 0x01) return set("BED is not SNP-major (mode=1 required)");
    const unsigned __int128 expected = (unsigned __int128)((n_indiv + 3) / 4) * n_snp + 3;
    if (expected != len)
        return set("BED has invalid length (expected " + std::to_string((uint64_t)expected) + ", got " +
                   std::to_string(len) + ")");
    return LDSC_OK;
}

int ldsc_panel_upload(ldsc_ctx* ctx, const uint8_t* body, uint64_t body_bytes, uint64_t n_indiv,
                      uint64_t n_snp, ldsc_panel** out) {
    if (!ctx || !out) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = nullptr;
    if (n_indiv == 0) return fail(ctx, LDSC_E_INVALID, "n_indiv must be > 0");
    const uint64_t bpr = (n_indiv + 3) / 4;
    if (body_bytes != bpr * n_snp)
        return fail(ctx, LDSC_E_BED, "BED has invalid length (expected " + std::to_string(bpr * n_snp + 3) +
                                         ", got " + std::to_string(body_bytes + 3) + ")");
    if (n_snp > 0 && !body) return fail(ctx, LDSC_E_INVALID, "null BED body");
    CK(cudaSetDevice(ctx->device));
    ldsc_panel* p = new ldsc_panel();
    p->ctx = ctx;
    p->n_snp = n_snp;
    p->n_indiv = n_indiv;
    p->bpr = bpr;
    p->pitch = round_up(bpr, 16);
    p->id = g_panel_ids.fetch_add(1);
    const size_t bytes = (size_t)p->pitch * (n_snp ? n_snp : 1);
    cudaError_t e = cudaMalloc(&p->rows, bytes);
    if (e != cudaSuccess) {
        delete p;
        return cuda_fail(ctx, e, "cudaMalloc(panel)");
    }
    e = cudaMemsetAsync(p->rows, 0, bytes, ctx->stream);
    if (e == cudaSuccess && n_snp)
        e = cudaMemcpy2DAsync(p->rows, p->pitch, body, bpr, bpr, n_snp, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(p->rows);
        delete p;
        return cuda_fail(ctx, e, "panel upload");
    }
    *out = p;
    return LDSC_OK;
}

int ldsc_panel_synth(ldsc_ctx* ctx, const ldsc_synth_spec* spec, ldsc_panel** out) {
    if (!ctx || !spec || !out) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = nullptr;
    if (spec->n_indiv == 0 || spec->founders == 0)
        return fail(ctx, LDSC_E_INVALID, "synthetic panel needs n_indiv > 0 and founders > 0");
    CK(cudaSetDevice(ctx->device));
    ldsc_panel* p = new ldsc_panel();
    p->ctx = ctx;
    p->n_snp = spec->n_snp;
    p->n_indiv = spec->n_indiv;
    p->bpr = (spec->n_indiv + 3) / 4;
    p->pitch = round_up(p->bpr, 16);
    p->id = g_panel_ids.fetch_add(1);
    const size_t bytes = (size_t)p->pitch * (spec->n_snp ? spec->n_snp : 1);
    uint8_t* table = nullptr;
    cudaError_t e = cudaMalloc(&p->rows, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&table, (size_t)spec->founders * (spec->n_snp ? spec->n_snp : 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(p->rows, 0, bytes, ctx->stream);
    if (e == cudaSuccess)
        e = launch_synth(p->rows, p->pitch, spec->n_indiv, spec->n_snp, spec->founders, spec->switch_p,
                         spec->miss, spec->seed, table, ctx->stream);
    ctx->kernels += 2;
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (table) cudaFree(table);
    if (e != cudaSuccess) {
        if (p->rows) cudaFree(p->rows);
        delete p;
        return cuda_fail(ctx, e, "synthetic panel");
    }
    *out = p;
    return LDSC_OK;
}

int ldsc_panel_download(ldsc_ctx* ctx, const ldsc_panel* p, uint64_t b, uint64_t end, uint8_t* out) {
    if (!ctx || !p || !out || b > end || end > p->n_snp) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    CK(cudaSetDevice(ctx->device));
    if (end == b) return LDSC_OK;
    CK(cudaMemcpy2DAsync(out, p->bpr, p->rows + b * p->pitch, p->pitch, p->bpr, end - b,
                         cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return LDSC_OK;
}

int ldsc_panel_destroy(ldsc_panel* p) {
    if (!p) return LDSC_OK;
    if (p->ctx) cudaSetDevice(p->ctx->device);
    if (p->rows) cudaFree(p->rows);
    p->sk.release();
    delete p;
    return LDSC_OK;
}

int ldsc_countsketch_hash(uint64_t n, uint32_t d, uint64_t seed, uint32_t* bucket, float* sign) {
    if ((n && (!bucket || !sign)) || d == 0) return LDSC_E_INVALID;
    countsketch_hash(n, d, seed, bucket, sign);
    return LDSC_OK;
}

int ldsc_l2_left_limits(const ldsc_l2_args* a, int64_t* left_out) {
    if (!a || (a->n_snp && !left_out)) return LDSC_E_INVALID;
    LeftLimits L;
    std::string err;
    if (!left_limits((int64_t)a->n_snp, a->chr, a->cm, a->bp, a->window_mode, a->window_size, a->window_snps,
                     a->chunk_size, a->snp_level_masking != 0, a->global_pass != 0, &L, &err))
        return LDSC_E_INVALID;
    if (a->n_snp) std::memcpy(left_out, L.left.data(), sizeof(int64_t) * a->n_snp);
    return LDSC_OK;
}

int ldsc_l2_workspace_bytes(const ldsc_l2_args* a, uint64_t n_indiv, uint64_t* bytes) {
    if (!a || !bytes) return LDSC_E_INVALID;
    const uint64_t m = a->n_snp;
    LeftLimits L;
    std::string err;
    if (!left_limits((int64_t)m, a->chr, a->cm, a->bp, a->window_mode, a->window_size, a->window_snps, a->chunk_size,
                     a->snp_level_masking != 0, a->global_pass != 0, &L, &err))
        return LDSC_E_INVALID;
    const uint64_t n_used = a->keep_iids ? a->n_keep : n_indiv;
    const uint64_t K = a->annot ? a->n_annot : 1;
    const uint32_t d = a->sketch_d;
    const bool exact_i8 = !d && a->precision == LDSC_PRECISION_INT8;
    const int ta = (exact_i8 || d) ? 64 : 128, tb = 128;
    const uint64_t ntiles = band_tiles(L.left, ta, tb).size();
    uint64_t b = m * (12 + 32 + 16 * K) + 8 * m + 8 * (ntiles + 1) + 64;  // stats, l2/aeff, left, tiles
    if (d && a->sketch_maf_aware) b += 16 * m;
    // f64 r2u tiles (K > 1) or per-tile row / column sums (K = 1), CSR tile lists
    const uint64_t nt_room = ntiles + ntiles / 8;  // the run's headroom on tile-count buffers
    b += (K > 1 ? (uint64_t)8 * ta * tb * nt_room : (uint64_t)8 * (ta + tb) * nt_room) + 8 * nt_room +
         4 * (m / 64 + m / 128 + 4);
    if (a->annot && !a->annot_on_device) b += 8 * m * K;
    if (a->bed_idx) b += 8 * m;
    if (a->keep_iids) b += 8 * a->n_keep;
    // INT8 operand rows (the default two-pass form; an upper bound for the fused one)
    if (exact_i8) b += 2 * m * round_up(n_used, 128);
    else if (d) b += 8 * m * round_up(d, 32);
    else b += 8 * m * round_up(n_used, 128);
    *bytes = b;
    return LDSC_OK;
}

int ldsc_l2_pair_count(const ldsc_l2_args* a, uint64_t* n_pairs) {
    if (!a || !n_pairs) return LDSC_E_INVALID;
    LeftLimits L;
    std::string err;
    if (!left_limits((int64_t)a->n_snp, a->chr, a->cm, a->bp, a->window_mode, a->window_size, a->window_snps,
                     a->chunk_size, a->snp_level_masking != 0, a->global_pass != 0, &L, &err))
        return LDSC_E_INVALID;
    *n_pairs = L.n_pairs;
    return LDSC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// the l2 run
// ---------------------------------------------------------------------------

namespace {

struct Events {
    cudaEvent_t ev[8] = {};
    int n = 0;
    cudaStream_t s;
    explicit Events(cudaStream_t st) : s(st) {}
    ~Events() {
        for (int i = 0; i < n; i++) cudaEventDestroy(ev[i]);
    }
    int mark() { return mark_on(s); }
    int mark_on(cudaStream_t on) {
        cudaEventCreate(&ev[n]);
        cudaEventRecord(ev[n], on);
        return n++;
    }
    double ms(int a, int b) const {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[a], ev[b]);
        return (double)t;
    }
};

// Bucket-major order for a sketch, uploaded, and the panel rewritten in that
// order into cache c.
int sketch_prepare(ldsc_ctx* ctx, const ldsc_panel* panel, uint64_t n_used, uint32_t d, const uint32_t* bucket,
                   const float* sign, const int64_t* keep, uint64_t key, SketchCache& c) {
    cudaStream_t s = ctx->stream;
    SketchOrder o = sketch_order(n_used, d, bucket, sign, keep);
    const uint64_t words = (n_used + 15) / 16;
    const uint64_t pitch_words = round_up(words, 4);
    c.valid = false;
    CK(c.perm.ensure(4 * (size_t)n_used));
    CK(c.seg.ensure(4 * o.seg_off.size()));
    CK(c.pp.ensure((size_t)4 * pitch_words * (panel->n_snp ? panel->n_snp : 1)));
    CK(cudaMemcpyAsync(c.perm.p, o.perm.data(), 4 * (size_t)n_used, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(c.seg.p, o.seg_off.data(), 4 * o.seg_off.size(), cudaMemcpyHostToDevice, s));
    PanelView pv{panel->rows, panel->n_snp, panel->n_indiv, panel->bpr, panel->pitch};
    CK(launch_sketch_permute(pv, c.perm.as<int32_t>(), n_used, c.pp.as<uint32_t>(), pitch_words, s));
    CK(c.segt.ensure(4 * (size_t)sketch_segt_count(n_used, d)));
    CK(launch_sketch_segt(c.seg.as<int32_t>(), n_used, d, c.segt.as<int32_t>(), s));
    ctx->kernels += 2;
    // host vectors go out of scope, and other streams may read the layout next
    CK(cudaStreamSynchronize(s));
    c.n = n_used;
    c.d = d;
    c.key = key;
    c.pitch_words = pitch_words;
    c.valid = true;
    return LDSC_OK;
}

// Streams a BED body from host memory into the pitched panel: the chunks'
// copies are queued on the context's copy stream (all at once, or the first
// one ahead of the host plan and the rest after it), and issue(c) makes the
// compute stream wait for chunk c and re-pitch it, so decoding chunk c
// overlaps the copies of the chunks after it.
struct RowFeed {
    ldsc_ctx* ctx = nullptr;
    const uint8_t* host = nullptr;  // file body (after the 3 magic bytes)
    uint64_t bpr = 0, pitch = 0, rows = 0, per = 0;
    int nchunks = 0, issued = 0, queued = 0;
    uint8_t* dst = nullptr;

    bool started = false;

    uint64_t row_end(int c) const { return std::min<uint64_t>(rows, (uint64_t)(c + 1) * per); }
    // buffers and events; the panel's rows pointer is valid after this
    int prepare() {
        ldsc_ctx* c = ctx;
        per = std::max<uint64_t>(1, (64ull << 20) / bpr);
        nchunks = (int)((rows + per - 1) / per);
        while ((int)c->feed_ev.size() < nchunks) {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            c->feed_ev.push_back(e);
        }
        if (!c->feed_t0) CK(cudaEventCreate(&c->feed_t0));
        if (!c->feed_t1) CK(cudaEventCreate(&c->feed_t1));
        if (!c->feed_go) CK(cudaEventCreateWithFlags(&c->feed_go, cudaEventDisableTiming));
        if (!c->up_ev) CK(cudaEventCreateWithFlags(&c->up_ev, cudaEventDisableTiming));
        CK(c->bed_stage.ensure(bpr * rows));
        CK(c->bed_rows.ensure(pitch * rows));
        dst = c->bed_rows.as<uint8_t>();
        return LDSC_OK;
    }
    // queue the copies of chunks [queued, k_end) (after the small uploads
    // already on the copy stream, so those are not held behind the file);
    // start() queues all of them
    int start_until(cudaStream_t s, int k_end) {
        ldsc_ctx* c = ctx;
        if (!started) {
            started = true;
            // the staging buffer may still be read by earlier work on the compute stream
            CK(cudaEventRecord(c->feed_go, s));
            CK(cudaStreamWaitEvent(c->copy, c->feed_go, 0));
            CK(cudaEventRecord(c->feed_t0, c->copy));
        }
        for (; queued < std::min(k_end, nchunks); queued++) {
            const int k = queued;
            const uint64_t r0 = (uint64_t)k * per, r1 = row_end(k);
            CK(cudaMemcpyAsync(c->bed_stage.as<uint8_t>() + r0 * bpr, host + r0 * bpr, (r1 - r0) * bpr,
                               cudaMemcpyHostToDevice, c->copy));
            CK(cudaEventRecord(c->feed_ev[k], c->copy));
            if (k == nchunks - 1) CK(cudaEventRecord(c->feed_t1, c->copy));
        }
        return LDSC_OK;
    }
    int start(cudaStream_t s) { return start_until(s, nchunks); }
    int issue_until(int k_end, cudaStream_t s) {  // chunks [issued, k_end)
        ldsc_ctx* c = ctx;
        if (queued < nchunks) {  // every waited-on chunk's copy (and event) is queued first
            int rc = start(s);
            if (rc != LDSC_OK) return rc;
        }
        for (; issued < std::min(k_end, nchunks); issued++) {
            CK(cudaStreamWaitEvent(s, c->feed_ev[issued], 0));
            CK(launch_repitch(c->bed_stage.as<uint8_t>(), bpr, dst, pitch, (uint64_t)issued * per, row_end(issued),
                              s));
            c->kernels++;
        }
        return LDSC_OK;
    }
    int issue_all(cudaStream_t s) { return issue_until(nchunks, s); }
    double upload_secs() const {
        float t = 0.f;
        if (!started) return 0.0;
        if (cudaEventSynchronize(ctx->feed_t1) != cudaSuccess ||
            cudaEventElapsedTime(&t, ctx->feed_t0, ctx->feed_t1) != cudaSuccess) {
            cudaGetLastError();
            return 0.0;
        }
        return t / 1e3;
    }
};

// The decode-overlap side stream (lowest priority, so the Gram's CTAs are
// placed first when both wait for an SM) and n per-chunk events, created on
// first use.
int ensure_overlap(ldsc_ctx* ctx, int n) {
    if (!ctx->side) {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CK(cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, least));
    }
    if (!ctx->ovl_go) CK(cudaEventCreateWithFlags(&ctx->ovl_go, cudaEventDisableTiming));
    while ((int)ctx->ovl_ev.size() < n) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->ovl_ev.push_back(e);
    }
    return LDSC_OK;
}

// Record chunks of the overlapped decode (each a multiple of the 128-record
// right block), and the smallest run that overlaps.  On B200 at 50,000
// individuals x 100,000 records, 4 and 8 equal chunks both cut a pass from
// 15.9 to 15.4 ms; 16 chunks, or a decode confined to fewer blocks, slow the
// Gram beside it more than they save.  A first chunk of 1/8 of the records
// (the rest in three equal chunks) shortens the decode no Gram tile can
// overlap: 15.23 / 15.46 -> 15.01 / 15.04 ms per pass over two runs each
// (1/16: 15.04 / 15.08, 1/32: 15.45).
constexpr int64_t OVERLAP_CHUNKS = 4;
constexpr int64_t OVERLAP_FIRST_DIV = 8;
constexpr int64_t OVERLAP_MIN_RECORDS = 16384;

int run_l2(ldsc_ctx* ctx, const ldsc_panel* panel, const ldsc_l2_args* a, double* l2_out, double* maf_out,
           ldsc_perf* perf, double upload_secs, RowFeed* feed = nullptr) {
    const auto t_wall0 = std::chrono::steady_clock::now();
    const int64_t m = (int64_t)a->n_snp;
    const uint64_t n_file = panel->n_indiv;
    const uint64_t n_used = a->keep_iids ? a->n_keep : n_file;
    const int32_t K = a->annot ? (int32_t)a->n_annot : 1;
    ldsc_perf pf;
    std::memset(&pf, 0, sizeof(pf));
    pf.m = (uint64_t)m;
    pf.n_indiv = n_used;
    pf.sketch_secs = -1.0;
    pf.bed_read_secs = upload_secs;

    // ---- argument validation (the reference's anyhow::ensure! sites) ----
    if (a->chunk_size < 1)
        return fail(ctx, LDSC_E_INVALID, "compute_ldscore_global: chunk_size must be >= 1, got 0");
    if (a->annot && a->n_annot == 0) return fail(ctx, LDSC_E_INVALID, "annotation matrix has zero columns");
    if (a->keep_iids) {
        if (a->n_keep == 0) return fail(ctx, LDSC_E_INVALID, "--keep: no individuals retained");
        for (uint64_t i = 0; i < a->n_keep; i++)
            if (a->keep_iids[i] < 0 || (uint64_t)a->keep_iids[i] >= n_file)
                return fail(ctx, LDSC_E_INVALID, "index " + std::to_string(a->keep_iids[i]) +
                                                     " out of range (max " + std::to_string(n_file) + ")");
    }
    const uint32_t d = a->sketch_d;
    if (d && !(d >= 3 && (uint64_t)d < n_used))
        return fail(ctx, LDSC_E_INVALID, "--sketch " + std::to_string(d) +
                                             " is out of bounds (must be 3 <= d < n_indiv=" +
                                             std::to_string(n_used) + ")");
    if (d > 12288) return fail(ctx, LDSC_E_UNSUPPORTED, "--sketch d > 12288 is not supported on the GPU");
    if (d && !sketch_supported(n_used, d))
        return fail(ctx, LDSC_E_UNSUPPORTED, "--sketch: too many individuals for the sketch kernel's shared memory");
    if (a->precision != LDSC_PRECISION_FP64 && a->precision != LDSC_PRECISION_INT8)
        return fail(ctx, LDSC_E_INVALID, "unknown precision");
    if (a->window_mode < 0 || a->window_mode > 2) return fail(ctx, LDSC_E_INVALID, "invalid window mode");
    if (m > 0 && (!a->chr || (a->window_mode == 0 && !a->cm) || (a->window_mode == 1 && !a->bp)))
        return fail(ctx, LDSC_E_INVALID, "missing chr / cm / bp arrays for the window mode");
    if (!d && a->precision == LDSC_PRECISION_INT8 && n_used > 1000000)
        return fail(ctx, LDSC_E_UNSUPPORTED, "INT8 form supports up to 1,000,000 individuals");
    if (m > 0 && a->bed_idx) {
        for (int64_t i = 0; i < m; i++)
            if (a->bed_idx[i] >= panel->n_snp)
                return fail(ctx, LDSC_E_INVALID, "SNP index " + std::to_string(a->bed_idx[i]) +
                                                     " out of range (max " + std::to_string(panel->n_snp) + ")");
    } else if (a->row_begin > panel->n_snp || (uint64_t)m > panel->n_snp - a->row_begin) {
        return fail(ctx, LDSC_E_INVALID, "more SNP records than panel rows");
    }
    if (a->annot && a->annot_ld && a->annot_ld < (uint64_t)m)
        return fail(ctx, LDSC_E_INVALID, "annot_ld is smaller than the number of SNP records");
    // records that are consecutive panel rows run as a row range (no record
    // list on the device; the INT8 Gram can read the packed rows in place)
    ldsc_l2_args as_range;
    if (m > 0 && a->bed_idx) {
        bool consecutive = true;
        for (int64_t i = 1; i < m && consecutive; i++) consecutive = a->bed_idx[i] == a->bed_idx[0] + (uint64_t)i;
        if (consecutive) {
            as_range = *a;
            as_range.row_begin = a->bed_idx[0];
            as_range.bed_idx = nullptr;
            a = &as_range;
        }
    }
    if (m == 0) {
        if (perf) *perf = pf;
        return LDSC_OK;
    }

    const bool exact_i8 = !d && a->precision == LDSC_PRECISION_INT8;
    // with LDSC_CTX_FUSED_OPERANDS the INT8 Gram reads the packed rows in
    // place when the records are the panel rows in order and every individual
    // is used
    const bool fused_i8 = exact_i8 && !a->bed_idx && !a->keep_iids && (ctx->flags & LDSC_CTX_FUSED_OPERANDS);
    const int ta = (exact_i8 || d) ? 64 : 128, tb = 128;  // tcgen05 tiles: 64 x 128 records
    pf.gram_kind = d ? 2u : (exact_i8 ? 1u : 0u);

    cudaStream_t s = ctx->stream;
    CK(cudaSetDevice(ctx->device));
    const uint64_t kernels0 = ctx->kernels;

    // ---- device buffers ----
    const uint64_t nmom = (uint64_t)m;
    CK(ctx->st_n.ensure(4 * nmom));
    CK(ctx->st_s.ensure(4 * nmom));
    CK(ctx->st_q.ensure(4 * nmom));
    CK(ctx->maf.ensure(8 * nmom));
    CK(ctx->st_mean.ensure(8 * nmom));
    CK(ctx->st_inv.ensure(8 * nmom));
    CK(ctx->st_qinv.ensure(8 * nmom));
    CK(ctx->l2.ensure(8 * nmom * K));
    CK(ctx->aeff.ensure(8 * nmom * K));
    CK(ctx->err.ensure(16));
    const bool maf_aware = d && a->sketch_maf_aware;
    if (maf_aware) {
        CK(ctx->st_q3.ensure(4 * nmom));
        CK(ctx->st_q4.ensure(4 * nmom));
        CK(ctx->st_kappa.ensure(8 * nmom));
    }
    if (a->annot && !a->annot_on_device) CK(ctx->annot.ensure(8 * nmom * K));
    if (a->bed_idx) CK(ctx->recrows.ensure(8 * nmom));
    if (a->keep_iids) CK(ctx->keep.ensure(8 * a->n_keep));

    // Host-to-device uploads.  With a streamed file they go through the copy
    // stream, ahead of the file's chunks: a copy issued on the compute stream
    // leaves that stream's next operations queued on the copy engine, behind
    // the whole file.  join_up() makes the compute stream wait for them.
    cudaStream_t up = feed ? ctx->copy : s;
    auto join_up = [&]() -> int {
        if (up == s) return LDSC_OK;
        CK(cudaEventRecord(ctx->up_ev, up));
        CK(cudaStreamWaitEvent(s, ctx->up_ev, 0));
        return LDSC_OK;
    };
    if (feed) {  // the buffers below may still be read by earlier work on the compute stream
        CK(cudaEventRecord(ctx->up_ev, s));
        CK(cudaStreamWaitEvent(up, ctx->up_ev, 0));
    }
    if (a->annot && !a->annot_on_device) {
        const uint64_t ald = a->annot_ld ? a->annot_ld : nmom;
        CK(cudaMemcpy2DAsync(ctx->annot.p, 8 * nmom, a->annot, 8 * ald, 8 * nmom, K, cudaMemcpyHostToDevice, up));
    }
    // annotations on the device: column c of record r at annot_dev[r + c * annot_ld_dev]
    const double* annot_dev = !a->annot ? nullptr : (a->annot_on_device ? a->annot : ctx->annot.as<double>());
    const uint64_t annot_ld_dev = !a->annot ? 0 : (a->annot_on_device && a->annot_ld ? a->annot_ld : nmom);
    if (a->bed_idx) CK(cudaMemcpyAsync(ctx->recrows.p, a->bed_idx, 8 * nmom, cudaMemcpyHostToDevice, up));
    if (a->keep_iids) CK(cudaMemcpyAsync(ctx->keep.p, a->keep_iids, 8 * a->n_keep, cudaMemcpyHostToDevice, up));
    CK(cudaMemsetAsync(ctx->err.p, 0, 16, s));

    PanelView pv{panel->rows, panel->n_snp, panel->n_indiv, panel->bpr, panel->pitch};
    if (!a->bed_idx) {
        pv.rows += a->row_begin * panel->pitch;
        pv.n_snp -= a->row_begin;
    }
    IndivSel sel{a->keep_iids ? ctx->keep.as<int64_t>() : nullptr, n_used};
    const uint64_t* rr = a->bed_idx ? ctx->recrows.as<uint64_t>() : nullptr;
    RecStats st{};
    st.n = ctx->st_n.as<int32_t>();
    st.s = ctx->st_s.as<int32_t>();
    st.q = ctx->st_q.as<int32_t>();
    st.q3 = maf_aware ? ctx->st_q3.as<int32_t>() : nullptr;
    st.q4 = maf_aware ? ctx->st_q4.as<int32_t>() : nullptr;
    st.maf = ctx->maf.as<double>();
    st.mean = ctx->st_mean.as<double>();
    st.inv_std = ctx->st_inv.as<double>();
    st.qinv = ctx->st_qinv.as<double>();
    st.kappa = maf_aware ? ctx->st_kappa.as<double>() : nullptr;
    st.pq = nullptr;

    // decode in feed chunks when records map to rows in order; else wait for the whole panel
    bool rows_in_order = true;
    if (a->bed_idx)
        for (int64_t i = 1; i < m && rows_in_order; i++) rows_in_order = a->bed_idx[i] >= a->bed_idx[i - 1];
    const bool chunked = feed && !d && rows_in_order;
    {
        int rc = join_up();
        if (rc != LDSC_OK) return rc;
    }
    if (feed && !chunked) {
        int rc = feed->issue_all(s);
        if (rc != LDSC_OK) return rc;
    }

    // the sketch layout: the panel's shared one, or this context's own when the
    // shared one is in use under another key
    const SketchCache* skc = nullptr;
    struct SketchUse {
        const ldsc_panel* p = nullptr;
        ~SketchUse() {
            if (p) {
                std::lock_guard<std::mutex> g(p->mu);
                p->sk_users--;
            }
        }
    } sk_use;
    if (d) {
        uint64_t key = 1469598103934665603ull;
        if (a->keep_iids)
            for (uint64_t i = 0; i < a->n_keep; i++) key = (key ^ (uint64_t)a->keep_iids[i]) * 1099511628211ull;
        std::vector<uint32_t> bucket;
        std::vector<float> sign;
        auto hash = [&]() {
            bucket.resize(n_used);
            sign.resize(n_used);
            countsketch_hash(n_used, d, 42, bucket.data(), sign.data());  // the reference's seed-42 stream
        };
        {
            std::lock_guard<std::mutex> g(panel->mu);
            if (!panel->sk.matches(n_used, d, key) && panel->sk_users == 0) {
                const auto tl0 = std::chrono::steady_clock::now();
                hash();
                int rc = sketch_prepare(ctx, panel, n_used, d, bucket.data(), sign.data(), a->keep_iids, key, panel->sk);
                if (rc != LDSC_OK) return rc;
                pf.layout_secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl0).count();
            }
            if (panel->sk.matches(n_used, d, key)) {
                panel->sk_users++;
                sk_use.p = panel;
                skc = &panel->sk;
            }
        }
        if (!skc) {
            if (!(ctx->sk_panel == panel->id && ctx->sk.matches(n_used, d, key))) {
                const auto tl0 = std::chrono::steady_clock::now();
                if (bucket.empty()) hash();
                ctx->sk_panel = 0;
                int rc = sketch_prepare(ctx, panel, n_used, d, bucket.data(), sign.data(), a->keep_iids, key, ctx->sk);
                if (rc != LDSC_OK) return rc;
                ctx->sk_panel = panel->id;
                pf.layout_secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - tl0).count();
            }
            skc = &ctx->sk;
        }
        CK(ctx->xsk.ensure((size_t)4 * 2 * nmom * round_up(d, 32)));
    }

    // ---- host plan: left limits, band tiles, contraction lists ----
    LeftLimits& L = ctx->plan_left;
    std::vector<Tile>& tiles = ctx->plan_tiles;
    const int32_t n_right = (int32_t)((m + tb - 1) / tb), n_left = (int32_t)((m + ta - 1) / ta);
    auto plan = [&]() -> int {
        std::string perr;
        if (!left_limits(m, a->chr, a->cm, a->bp, a->window_mode, a->window_size, a->window_snps, a->chunk_size,
                         a->snp_level_masking != 0, a->global_pass != 0, &L, &perr))
            return fail(ctx, LDSC_E_INVALID, perr);
        if (L.any_full && !a->yes_really)
            std::printf("WARNING: LD window spans the entire chromosome. Use --yes-really to silence this warning.\n");
        pf.n_pairs = L.n_pairs;
        band_tiles(L.left, ta, tb, &tiles);
        pf.n_tiles = tiles.size();
        CK(ctx->left.ensure(sizeof(int64_t) * nmom));
        // buffers sized by the tile count get an eighth more when they grow: a
        // later call over a few more tiles then reuses them instead of
        // allocating (a pool growth while other work runs stalls it)
        const size_t nt_room = tiles.size() + tiles.size() / 8;
        CK(ctx->tiles.ensure(sizeof(Tile) * (nt_room + 1)));
        CK(cudaMemcpyAsync(ctx->left.p, L.left.data(), 8 * nmom, cudaMemcpyHostToDevice, up));
        if (!tiles.empty())
            CK(cudaMemcpyAsync(ctx->tiles.p, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, up));
        // CSR lists of tiles per right block and per left block: the K > 1
        // contraction passes and the K = 1 reduction of per-tile sums.  The
        // host lists live in the context until the next call (the copies
        // read them asynchronously).
        if (!tiles.empty()) {
            std::vector<int32_t>&ptr_r = ctx->plan_ptr_r, &ptr_l = ctx->plan_ptr_l, &idx_r = ctx->plan_idx_r,
                                  &idx_l = ctx->plan_idx_l;
            ptr_r.assign(n_right + 1, 0);
            ptr_l.assign(n_left + 1, 0);
            idx_r.resize(tiles.size());
            idx_l.resize(tiles.size());
            for (const Tile& t : tiles) {
                ptr_r[t.b_blk + 1]++;
                ptr_l[t.a_blk + 1]++;
            }
            for (int32_t i = 0; i < n_right; i++) ptr_r[i + 1] += ptr_r[i];
            for (int32_t i = 0; i < n_left; i++) ptr_l[i + 1] += ptr_l[i];
            std::vector<int32_t> fr(ptr_r.begin(), ptr_r.end() - 1), fl(ptr_l.begin(), ptr_l.end() - 1);
            for (int32_t t = 0; t < (int32_t)tiles.size(); t++) {
                idx_r[fr[tiles[t].b_blk]++] = t;
                idx_l[fl[tiles[t].a_blk]++] = t;
            }
            if (K > 1) {
                CK(ctx->rtiles.ensure(sizeof(double) * (size_t)ta * tb * nt_room));
            } else {
                CK(ctx->prow.ensure(sizeof(double) * (size_t)ta * nt_room));
                CK(ctx->pcol.ensure(sizeof(double) * (size_t)tb * nt_room));
            }
            CK(ctx->cptr_r.ensure(4 * ptr_r.size()));
            CK(ctx->cidx_r.ensure(4 * nt_room));
            CK(ctx->cptr_l.ensure(4 * ptr_l.size()));
            CK(ctx->cidx_l.ensure(4 * nt_room));
            CK(cudaMemcpyAsync(ctx->cptr_r.p, ptr_r.data(), 4 * ptr_r.size(), cudaMemcpyHostToDevice, up));
            CK(cudaMemcpyAsync(ctx->cidx_r.p, idx_r.data(), 4 * idx_r.size(), cudaMemcpyHostToDevice, up));
            CK(cudaMemcpyAsync(ctx->cptr_l.p, ptr_l.data(), 4 * ptr_l.size(), cudaMemcpyHostToDevice, up));
            CK(cudaMemcpyAsync(ctx->cidx_l.p, idx_l.data(), 4 * idx_l.size(), cudaMemcpyHostToDevice, up));
        }
        return join_up();
    };

    // ---- epilogue constants ----
    EpilogueArgs ep{};
    ep.n = st.n;
    ep.s = st.s;
    ep.qinv = st.qinv;
    ep.kappa = st.kappa;
    ep.aeff = ctx->aeff.as<double>();
    ep.l2 = ctx->l2.as<double>();
    ep.m = m;
    ep.K = K;
    const double N = (double)n_used;
    const double denom = n_used > 2 ? N - 2.0 : N;
    ep.r2u_a = 1.0 + 1.0 / denom;
    ep.r2u_b = -1.0 / denom;
    ep.n_inv_sq_r2u_a = (1.0 / N) * (1.0 / N) * ep.r2u_a;
    ep.n_inv_sq = (1.0 / N) * (1.0 / N);
    ep.sketch_d = (double)d;
    ep.err = ctx->err.as<unsigned int>();

    // Whole-file INT8 runs with one annotation column overlap the band Gram
    // with the upload too: after chunk k is decoded and finalised, the tiles
    // whose records all lie in chunks [0, k] run while later chunks copy.
    const bool stream_gram = chunked && exact_i8 && K == 1;
    // Resident panels (two-pass INT8 form, one annotation column) overlap the
    // decode of record chunk k + 1, on the side stream, with the band Gram of
    // the tiles whose records all lie in chunks [0, k]: the decode is
    // HBM-bound, the Gram tensor-bound, and decode blocks (40 registers x 256
    // threads, no shared memory) fit on an SM beside a Gram CTA.
    const bool overlap = !feed && exact_i8 && !fused_i8 && K == 1 && m >= OVERLAP_MIN_RECORDS;
    // chunk k = records [ov_b[k], ov_b[k + 1]); the first chunk is
    // 1/OVERLAP_FIRST_DIV of the records (its decode runs before any Gram tile
    // can), the rest are equal
    std::vector<int64_t> ov_b;
    if (overlap) {
        const int64_t first = std::min<int64_t>(
            m, (int64_t)round_up((uint64_t)((m + OVERLAP_FIRST_DIV - 1) / OVERLAP_FIRST_DIV), 128));
        ov_b.push_back(0);
        ov_b.push_back(first);
        const int64_t rest = m - first, nrest = OVERLAP_CHUNKS - 1;
        const int64_t per = rest > 0 ? (int64_t)round_up((uint64_t)((rest + nrest - 1) / nrest), 128) : 0;
        for (int64_t r = first; r < m;) {
            r = std::min<int64_t>(m, r + per);
            ov_b.push_back(r);
        }
    }
    const int ov_n = overlap ? (int)ov_b.size() - 1 : 0;
    if (stream_gram) {
        // the first chunk's copy runs while the host plans; the plan's uploads
        // queue behind that chunk only
        int rc = feed->start_until(s, 1);
        if (rc != LDSC_OK) return rc;
        rc = plan();
        if (rc != LDSC_OK) return rc;
        ep.left = ctx->left.as<int64_t>();
        ep.rtiles = nullptr;
        ep.prow = tiles.empty() ? nullptr : ctx->prow.as<double>();
        ep.pcol = tiles.empty() ? nullptr : ctx->pcol.as<double>();
    }
    if (chunked) {
        int rc = feed->start(s);
        if (rc != LDSC_OK) return rc;
    }

    Events ev(s);
    const int e0 = ev.mark();

    // ---- decode ----
    const uint64_t ld_i8 = round_up(n_used, 128);
    const uint64_t ld_sk = round_up(d ? d : 1, 32);  // 128-byte operand rows for TMA
    int e_sk = -1, e_side = -1;
    const bool staged_i8 = exact_i8 && !fused_i8;
    if (staged_i8) CK(ctx->ops.ensure((size_t)2 * nmom * ld_i8));
    if (chunked) {
        // records [r0, r1) whose rows arrived with chunks [0, k]
        int64_t r0 = 0;
        size_t t0 = 0;
        for (int k = 0; k < feed->nchunks; k++) {
            const uint64_t rend = feed->row_end(k);
            int64_t r1 = r0;
            if (a->bed_idx)
                r1 = std::lower_bound(a->bed_idx + r0, a->bed_idx + m, rend) - a->bed_idx;
            else
                r1 = std::max<int64_t>(r0, std::min<int64_t>(m, (int64_t)rend - (int64_t)a->row_begin));
            int rc = feed->issue_until(k + 1, s);
            if (rc != LDSC_OK) return rc;
            if (r1 > r0) {
                PanelView pc = pv;
                if (!rr) pc.rows = pv.rows + (uint64_t)r0 * pv.pitch;
                RecStats sc = st;
                sc.n += r0;
                sc.s += r0;
                sc.q += r0;
                uint8_t* oc = staged_i8 ? ctx->ops.as<uint8_t>() + (size_t)2 * r0 * ld_i8 : nullptr;
                CK(launch_decode_i8(pc, rr ? rr + r0 : nullptr, r1 - r0, sel, oc, staged_i8 ? ld_i8 : 0, sc, 0, s));
                ctx->kernels++;
                if (stream_gram) {
                    sc.maf += r0;
                    sc.mean += r0;
                    sc.inv_std += r0;
                    sc.qinv += r0;
                    CK(launch_finalize_stats(r1 - r0, n_used, sc, annot_dev ? annot_dev + r0 : nullptr, 1,
                                             a->has_pq_exp, a->pq_exp, ctx->aeff.as<double>() + r0,
                                             ctx->l2.as<double>() + r0, s, annot_ld_dev));
                    ctx->kernels++;
                    // tiles are ordered by right block; take those whose right block is complete
                    size_t t1 = t0;
                    while (t1 < tiles.size() && (r1 == m || (int64_t)(tiles[t1].b_blk + 1) * tb <= r1)) t1++;
                    if (t1 > t0) {
                        // this launch's tiles write their sums at their own tile indices
                        EpilogueArgs ec = ep;
                        ec.prow += t0 * ta;
                        ec.pcol += t0 * tb;
                        if (fused_i8)
                            CK(launch_gram_i8_packed(pv.rows, pv.pitch, n_used, m, ctx->tiles.as<Tile>() + t0,
                                                     (int64_t)(t1 - t0), ec, nullptr, ctx->sms, s));
                        else
                            CK(launch_gram_i8(ctx->ops.as<uint8_t>(), ld_i8, m, ctx->tiles.as<Tile>() + t0,
                                              (int64_t)(t1 - t0), ec, nullptr, ctx->sms, s));
                        ctx->kernels++;
                    }
                    t0 = t1;
                }
            }
            r0 = r1;
        }
        ctx->kernels--;  // counted once below
    } else if (overlap) {
        // decode and finalise chunk by chunk on the side stream, after the
        // compute stream's work so far (uploads, the error-word reset)
        int rc = ensure_overlap(ctx, ov_n);
        if (rc != LDSC_OK) return rc;
        CK(cudaEventRecord(ctx->ovl_go, s));
        CK(cudaStreamWaitEvent(ctx->side, ctx->ovl_go, 0));
        for (int k = 0; k < ov_n; k++) {
            const int64_t r0 = ov_b[k], r1 = ov_b[k + 1];
            PanelView pc = pv;
            if (!rr) pc.rows = pv.rows + (uint64_t)r0 * pv.pitch;
            RecStats sc = st;
            sc.n += r0;
            sc.s += r0;
            sc.q += r0;
            sc.maf += r0;
            sc.mean += r0;
            sc.inv_std += r0;
            sc.qinv += r0;
            CK(launch_decode_i8(pc, rr ? rr + r0 : nullptr, r1 - r0, sel, ctx->ops.as<uint8_t>() + (size_t)2 * r0 * ld_i8,
                                ld_i8, sc, 0, ctx->side));
            CK(launch_finalize_stats(r1 - r0, n_used, sc, annot_dev ? annot_dev + r0 : nullptr, 1, a->has_pq_exp,
                                     a->pq_exp, ctx->aeff.as<double>() + r0, ctx->l2.as<double>() + r0, ctx->side,
                                     annot_ld_dev));
            CK(cudaEventRecord(ctx->ovl_ev[k], ctx->side));
            ctx->kernels += 2;
        }
        e_side = ev.mark_on(ctx->side);
        ctx->kernels--;  // counted once below
    } else if (staged_i8) {
        CK(launch_decode_i8(pv, rr, m, sel, ctx->ops.as<uint8_t>(), ld_i8, st, 0, s));
    } else if (d) {
        // fused: moments + CountSketch rows in one pass over the permuted panel
        CK(launch_sketch_seg(skc->pp.as<uint32_t>() + (rr ? 0 : a->row_begin * skc->pitch_words), skc->pitch_words,
                             rr, m, n_used, skc->segt.as<int32_t>(), d, st, maf_aware ? 1 : 0, 1,
                             ctx->xsk.as<float>(), ld_sk, s));
        e_sk = ev.mark();
    } else {
        CK(launch_decode_i8(pv, rr, m, sel, nullptr, 0, st, 0, s));
    }
    ctx->kernels++;
    if (!stream_gram && !overlap) {
        CK(launch_finalize_stats(m, n_used, st, annot_dev, K, a->has_pq_exp, a->pq_exp, ctx->aeff.as<double>(),
                                 ctx->l2.as<double>(), s, annot_ld_dev));
        ctx->kernels++;
    }
    const uint64_t ld_f64 = round_up(n_used, 128);
    if (!d && !exact_i8) {
        CK(ctx->xf64.ensure((size_t)8 * nmom * ld_f64));
        CK(launch_decode_f64(pv, rr, m, sel, st, ctx->xf64.as<double>(), ld_f64, s));
        ctx->kernels++;
    }
    const int e1 = ev.mark();

    if (!stream_gram) {
        // ---- host plan (runs while the decode kernels execute) ----
        int rc = plan();
        if (rc != LDSC_OK) return rc;
        ep.left = ctx->left.as<int64_t>();
        ep.rtiles = (K > 1 && !tiles.empty()) ? ctx->rtiles.as<double>() : nullptr;
        ep.prow = (K == 1 && !tiles.empty()) ? ctx->prow.as<double>() : nullptr;
        ep.pcol = (K == 1 && !tiles.empty()) ? ctx->pcol.as<double>() : nullptr;
    }
    // ---- band Gram + epilogue ----
    if (overlap) CK(cudaStreamWaitEvent(s, ctx->ovl_ev[0], 0));  // the Gram's time starts at its first tiles
    const int e2 = ev.mark();
    int e_c = -1;
    if (!tiles.empty() && overlap) {
        // tiles are ordered by right block; chunk k's launch takes those whose
        // right block is complete once chunks [0, k] are decoded
        size_t t0 = 0;
        for (int k = 0; k < ov_n; k++) {
            const int64_t r1 = ov_b[k + 1];
            size_t t1 = t0;
            while (t1 < tiles.size() && (r1 == m || (int64_t)(tiles[t1].b_blk + 1) * tb <= r1)) t1++;
            if (t1 == t0) continue;
            CK(cudaStreamWaitEvent(s, ctx->ovl_ev[k], 0));
            EpilogueArgs ec = ep;  // this launch's tiles write their sums at their own tile indices
            ec.prow += t0 * ta;
            ec.pcol += t0 * tb;
            CK(launch_gram_i8(ctx->ops.as<uint8_t>(), ld_i8, m, ctx->tiles.as<Tile>() + t0, (int64_t)(t1 - t0), ec,
                              nullptr, ctx->sms, s));
            ctx->kernels++;
            t0 = t1;
        }
    }
    // every record's statistics are final before the reduction reads them
    if (overlap) CK(cudaStreamWaitEvent(s, ctx->ovl_ev[ov_n - 1], 0));
    if (!tiles.empty() && !stream_gram && !overlap) {
        if (d) {
            CK(launch_gram_tf32(ctx->xsk.as<float>(), ld_sk, m, ctx->tiles.as<Tile>(), (int64_t)tiles.size(), ep,
                                maf_aware ? 1 : 0, nullptr, ctx->sms, s));
        } else if (fused_i8) {
            CK(launch_gram_i8_packed(pv.rows, pv.pitch, n_used, m, ctx->tiles.as<Tile>(), (int64_t)tiles.size(), ep,
                                     nullptr, ctx->sms, s));
        } else if (exact_i8) {
            CK(launch_gram_i8(ctx->ops.as<uint8_t>(), ld_i8, m, ctx->tiles.as<Tile>(), (int64_t)tiles.size(), ep,
                              nullptr, ctx->sms, s));
        } else {
            CK(launch_gram_f64(ctx->xf64.as<double>(), ld_f64, ld_f64, ctx->tiles.as<Tile>(), (int64_t)tiles.size(),
                               ep, ctx->sms, s));
        }
        ctx->kernels++;
        e_c = ev.mark();
        if (K > 1) {
            CK(launch_contract(ctx->rtiles.as<double>(), ta, tb, ctx->tiles.as<Tile>(), ctx->cptr_r.as<int32_t>(),
                               ctx->cidx_r.as<int32_t>(), n_right, true, ep, s));
            CK(launch_contract(ctx->rtiles.as<double>(), ta, tb, ctx->tiles.as<Tile>(), ctx->cptr_l.as<int32_t>(),
                               ctx->cidx_l.as<int32_t>(), n_left, false, ep, s));
            ctx->kernels += 2;
        }
    }
    if (K == 1 && !tiles.empty()) {
        // the per-tile sums into l2, in a fixed order
        CK(launch_l2_reduce(m, ta, tb, ctx->cptr_r.as<int32_t>(), ctx->cidx_r.as<int32_t>(), ctx->cptr_l.as<int32_t>(),
                            ctx->cidx_l.as<int32_t>(), ctx->prow.as<double>(), ctx->pcol.as<double>(),
                            ctx->l2.as<double>(), s));
        ctx->kernels++;
    }
    const int e3 = ev.mark();
    const cudaMemcpyKind okind = a->out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(l2_out, ctx->l2.p, 8 * nmom * K, okind, s));
    if (maf_out) CK(cudaMemcpyAsync(maf_out, ctx->maf.p, 8 * nmom, okind, s));
    unsigned int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(herr, ctx->err.p, 16, cudaMemcpyDeviceToHost, s));
    const int e4 = ev.mark();
    CK(cudaStreamSynchronize(s));
    if (herr[0] != 0)
        return fail(ctx, LDSC_E_TIMEOUT, "a device wait in the Gram kernel exceeded its bound (error word " +
                                             std::to_string(herr[0]) + ")");
    pf.norm_secs = ev.ms(d ? e_sk : e0, overlap ? e_side : e1) / 1e3;
    if (d) pf.sketch_secs = ev.ms(e0, e_sk) / 1e3;
    pf.ab_dot_secs = ev.ms(e2, e3) / 1e3;
    if (e_c >= 0 && K > 1) pf.contract_secs = ev.ms(e_c, e3) / 1e3;
    pf.device_ms = ev.ms(e0, e4);
    pf.kernel_launches = (uint32_t)(ctx->kernels - kernels0);
    if (perf) *perf = pf;
    if (a->on_progress) {
        ldsc_progress pr;
        pr.chunks_done = L.chunks;
        pr.chunks_total = L.chunks;
        pr.snps_done = (uint64_t)m;
        pr.snps_total = (uint64_t)m;
        pr.chunk_wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_wall0).count();
        a->on_progress(&pr, a->progress_user);
    }
    return LDSC_OK;
}

}  // namespace

extern "C" {

int ldsc_snp_stats(ldsc_ctx* ctx, const ldsc_panel* panel, const ldsc_l2_args* a, double* maf_out,
                   uint8_t* het_miss_ok_out) {
    if (!ctx || !panel || !a) return LDSC_E_INVALID;
    const int64_t m = (int64_t)a->n_snp;
    if (m > 0 && (!maf_out || !het_miss_ok_out)) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    const uint64_t n_file = panel->n_indiv;
    const uint64_t n_used = a->keep_iids ? a->n_keep : n_file;
    if (a->keep_iids) {
        if (a->n_keep == 0) return fail(ctx, LDSC_E_INVALID, "--keep: no individuals retained");
        for (uint64_t i = 0; i < a->n_keep; i++)
            if (a->keep_iids[i] < 0 || (uint64_t)a->keep_iids[i] >= n_file)
                return fail(ctx, LDSC_E_INVALID, "index " + std::to_string(a->keep_iids[i]) +
                                                     " out of range (max " + std::to_string(n_file) + ")");
    }
    if (a->bed_idx) {
        for (int64_t i = 0; i < m; i++)
            if (a->bed_idx[i] >= panel->n_snp)
                return fail(ctx, LDSC_E_INVALID, "SNP index " + std::to_string(a->bed_idx[i]) +
                                                     " out of range (max " + std::to_string(panel->n_snp) + ")");
    } else if (a->row_begin > panel->n_snp || (uint64_t)m > panel->n_snp - a->row_begin) {
        return fail(ctx, LDSC_E_INVALID, "more SNP records than panel rows");
    }
    if (m == 0) return LDSC_OK;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    CK(ctx->st_n.ensure(4 * (size_t)m));
    CK(ctx->st_s.ensure(4 * (size_t)m));
    CK(ctx->st_q.ensure(4 * (size_t)m));
    if (a->bed_idx) {
        CK(ctx->recrows.ensure(8 * (size_t)m));
        CK(cudaMemcpyAsync(ctx->recrows.p, a->bed_idx, 8 * (size_t)m, cudaMemcpyHostToDevice, s));
    }
    if (a->keep_iids) {
        CK(ctx->keep.ensure(8 * a->n_keep));
        CK(cudaMemcpyAsync(ctx->keep.p, a->keep_iids, 8 * a->n_keep, cudaMemcpyHostToDevice, s));
    }
    PanelView pv{panel->rows, panel->n_snp, panel->n_indiv, panel->bpr, panel->pitch};
    if (!a->bed_idx) {
        pv.rows += a->row_begin * panel->pitch;
        pv.n_snp -= a->row_begin;
    }
    IndivSel sel{a->keep_iids ? ctx->keep.as<int64_t>() : nullptr, n_used};
    RecStats st{};
    st.n = ctx->st_n.as<int32_t>();
    st.s = ctx->st_s.as<int32_t>();
    st.q = ctx->st_q.as<int32_t>();
    CK(launch_decode_i8(pv, a->bed_idx ? ctx->recrows.as<uint64_t>() : nullptr, m, sel, nullptr, 0, st, 0, s));
    ctx->kernels++;
    std::vector<int32_t> hn((size_t)m), hs((size_t)m), hq((size_t)m);
    CK(cudaMemcpyAsync(hn.data(), st.n, 4 * (size_t)m, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hs.data(), st.s, 4 * (size_t)m, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hq.data(), st.q, 4 * (size_t)m, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // compute_snp_stats (src/l2/snp_stats.rs:150-163): freq = sum / (2 count),
    // MAF = min(freq, 1 - freq); keep when het + missing < n.  With s = #1 + 2 #2
    // and q = #1 + 4 #2, het = #1 = 2 s - q.
    for (int64_t i = 0; i < m; i++) {
        const int64_t n = hn[i], sm = hs[i], q = hq[i];
        const double freq = n > 0 ? (double)sm / (2.0 * (double)n) : 0.0;
        maf_out[i] = freq < 1.0 - freq ? freq : 1.0 - freq;
        const int64_t het = 2 * sm - q, missing = (int64_t)n_used - n;
        het_miss_ok_out[i] = (uint8_t)(het + missing < (int64_t)n_used);
    }
    return LDSC_OK;
}

int ldsc_l2_run(ldsc_ctx* ctx, const ldsc_panel* panel, const ldsc_l2_args* args, double* l2_out,
                double* maf_out, ldsc_perf* perf) {
    if (!ctx || !panel || !args) return LDSC_E_INVALID;
    if (args->n_snp && !l2_out) return fail(ctx, LDSC_E_INVALID, "null l2_out");
    std::lock_guard<std::mutex> g(ctx->mu);
    return run_l2(ctx, panel, args, l2_out, maf_out, perf, 0.0);
}

int ldsc_l2_from_bed(ldsc_ctx* ctx, const uint8_t* bed_file, uint64_t len, uint64_t n_indiv,
                     const ldsc_l2_args* args, double* l2_out, double* maf_out, ldsc_perf* perf) {
    if (!ctx || !args) return LDSC_E_INVALID;
    // the panel's SNP count is implied by the file length
    if (n_indiv == 0) return fail(ctx, LDSC_E_INVALID, "compute_l2_from_bed: FAM has zero individuals");
    const uint64_t bpr = (n_indiv + 3) / 4;
    const uint64_t n_rows = len >= 3 ? (len - 3) / bpr : 0;
    char msg[256];
    uint64_t need_rows = args->n_snp;
    if (args->bed_idx)
        for (uint64_t i = 0; i < args->n_snp; i++) need_rows = args->bed_idx[i] + 1 > need_rows ? args->bed_idx[i] + 1 : need_rows;
    const uint64_t rows = args->bed_idx ? n_rows : args->n_snp;
    int rc = ldsc_bed_validate(bed_file, len, n_indiv, rows, msg, sizeof msg);
    if (rc != LDSC_OK) return fail(ctx, rc, msg);
    if (need_rows > rows) return fail(ctx, LDSC_E_INVALID, "SNP records point past the BED rows");
    std::lock_guard<std::mutex> g(ctx->mu);
    CK(cudaSetDevice(ctx->device));
    // the panel lives in context-owned memory for the duration of the call
    ldsc_panel p;
    p.ctx = ctx;
    p.n_snp = rows;
    p.n_indiv = n_indiv;
    p.bpr = bpr;
    p.pitch = round_up(bpr, 16);
    p.id = g_panel_ids.fetch_add(1);
    RowFeed feed;
    feed.ctx = ctx;
    feed.host = bed_file + 3;
    feed.bpr = bpr;
    feed.pitch = p.pitch;
    feed.rows = rows;
    if (rows > 0) {
        rc = feed.prepare();
        if (rc != LDSC_OK) return rc;
        p.rows = feed.dst;
    } else {
        CK(ctx->bed_rows.ensure(16));
        p.rows = ctx->bed_rows.as<uint8_t>();
    }
    rc = run_l2(ctx, &p, args, l2_out, maf_out, perf, 0.0, rows > 0 ? &feed : nullptr);
    p.sk.release();  // the call's panel layout does not outlive the call
    if (feed.started) {
        // a run that failed part-way returns before the feed is drained: finish it here
        int rc2 = feed.issue_all(ctx->stream);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (rc == LDSC_OK && rc2 != LDSC_OK) rc = rc2;
        if (rc == LDSC_OK && e != cudaSuccess) rc = cuda_fail(ctx, e, "BED upload");
        if (rc == LDSC_OK && perf) perf->bed_read_secs = feed.upload_secs();
    }
    return rc;
}

int ldsc_sketch_project(ldsc_ctx* ctx, const ldsc_panel* panel, uint64_t b, uint64_t e, const int64_t* keep,
                        uint64_t n_keep, const uint32_t* bucket, const float* sign, uint32_t d, float* out) {
    if (!ctx || !panel || !bucket || !sign || !out || b > e || e > panel->n_snp || d == 0) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (d > 12288) return fail(ctx, LDSC_E_UNSUPPORTED, "d > 12288");
    const int64_t m = (int64_t)(e - b);
    if (m == 0) return LDSC_OK;
    const uint64_t n_used = keep ? n_keep : panel->n_indiv;
    if (n_used == 0) return fail(ctx, LDSC_E_INVALID, "no individuals");
    if (!sketch_supported(n_used, d))
        return fail(ctx, LDSC_E_UNSUPPORTED, "too many individuals for the sketch kernel's shared memory");
    for (uint64_t i = 0; i < n_used; i++) {
        if (bucket[i] >= d) return fail(ctx, LDSC_E_INVALID, "bucket index >= d");
        if (keep && (keep[i] < 0 || (uint64_t)keep[i] >= panel->n_indiv))
            return fail(ctx, LDSC_E_INVALID, "keep index out of range");
    }
    cudaStream_t s = ctx->stream;
    CK(cudaSetDevice(ctx->device));
    ctx->sk_panel = 0;  // explicit bucket/sign arrays: the layout is not reused by l2 runs
    int rc = sketch_prepare(ctx, panel, n_used, d, bucket, sign, keep, 0, ctx->sk);
    if (rc != LDSC_OK) return rc;
    std::vector<uint64_t> rows((size_t)m);
    for (int64_t i = 0; i < m; i++) rows[i] = b + (uint64_t)i;
    CK(ctx->recrows.ensure(8 * (size_t)m));
    CK(ctx->st_n.ensure(4 * (size_t)m));
    CK(ctx->st_s.ensure(4 * (size_t)m));
    CK(ctx->st_q.ensure(4 * (size_t)m));
    CK(ctx->xsk.ensure(4 * (size_t)m * d));
    CK(cudaMemcpyAsync(ctx->recrows.p, rows.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, s));
    RecStats st{};
    st.n = ctx->st_n.as<int32_t>();
    st.s = ctx->st_s.as<int32_t>();
    st.q = ctx->st_q.as<int32_t>();
    CK(launch_sketch_seg(ctx->sk.pp.as<uint32_t>(), ctx->sk.pitch_words, ctx->recrows.as<uint64_t>(), m, n_used,
                         ctx->sk.segt.as<int32_t>(), d, st, 0, 0, ctx->xsk.as<float>(), d, s));
    ctx->kernels += 1;
    CK(cudaMemcpyAsync(out, ctx->xsk.p, 4 * (size_t)m * d, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return LDSC_OK;
}

int ldsc_debug_gram_i8_tile(ldsc_ctx* ctx, const ldsc_panel* panel, uint64_t k0, uint64_t j0, int32_t* out) {
    if (!ctx || !panel || !out) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (k0 % 64 || j0 % 128 || k0 >= panel->n_snp || j0 >= panel->n_snp)
        return fail(ctx, LDSC_E_INVALID, "tile origin must be k0 % 64 == 0, j0 % 128 == 0, inside the panel");
    const int64_t m = (int64_t)panel->n_snp;
    const uint64_t n = panel->n_indiv;
    const uint64_t ld = round_up(n, 128);
    cudaStream_t s = ctx->stream;
    CK(cudaSetDevice(ctx->device));
    const bool fused = (ctx->flags & LDSC_CTX_FUSED_OPERANDS) != 0;
    if (!fused) CK(ctx->ops.ensure((size_t)2 * m * ld));
    CK(ctx->st_n.ensure(4 * (size_t)m));
    CK(ctx->st_s.ensure(4 * (size_t)m));
    CK(ctx->st_q.ensure(4 * (size_t)m));
    CK(ctx->maf.ensure(8 * (size_t)m));
    CK(ctx->st_mean.ensure(8 * (size_t)m));
    CK(ctx->st_inv.ensure(8 * (size_t)m));
    CK(ctx->st_qinv.ensure(8 * (size_t)m));
    CK(ctx->left.ensure(8 * (size_t)m));
    CK(ctx->aeff.ensure(8 * (size_t)m));
    CK(ctx->l2.ensure(8 * (size_t)m));
    CK(ctx->tiles.ensure(sizeof(Tile)));
    CK(ctx->err.ensure(16));
    CK(ctx->dbg.ensure(4 * 128 * 256));
    PanelView pv{panel->rows, panel->n_snp, panel->n_indiv, panel->bpr, panel->pitch};
    IndivSel sel{nullptr, n};
    RecStats st{};
    st.n = ctx->st_n.as<int32_t>();
    st.s = ctx->st_s.as<int32_t>();
    st.q = ctx->st_q.as<int32_t>();
    st.maf = ctx->maf.as<double>();
    st.mean = ctx->st_mean.as<double>();
    st.inv_std = ctx->st_inv.as<double>();
    st.qinv = ctx->st_qinv.as<double>();
    CK(launch_decode_i8(pv, nullptr, m, sel, fused ? nullptr : ctx->ops.as<uint8_t>(), fused ? 0 : ld, st, 0, s));
    CK(launch_finalize_stats(m, n, st, nullptr, 1, 0, 0.0, ctx->aeff.as<double>(), ctx->l2.as<double>(), s));
    CK(cudaMemsetAsync(ctx->left.p, 0, 8 * (size_t)m, s));
    CK(cudaMemsetAsync(ctx->err.p, 0, 16, s));
    Tile t{(uint32_t)(k0 / 64), (uint32_t)(j0 / 128)};
    CK(cudaMemcpyAsync(ctx->tiles.p, &t, sizeof(Tile), cudaMemcpyHostToDevice, s));
    EpilogueArgs ep{};
    ep.left = ctx->left.as<int64_t>();
    ep.n = st.n;
    ep.s = st.s;
    ep.qinv = st.qinv;
    ep.aeff = ctx->aeff.as<double>();
    ep.l2 = ctx->l2.as<double>();
    ep.m = m;
    ep.K = 1;
    ep.r2u_a = 1.0;
    ep.r2u_b = 0.0;
    ep.err = ctx->err.as<unsigned int>();
    if (fused)
        CK(launch_gram_i8_packed(panel->rows, panel->pitch, n, m, ctx->tiles.as<Tile>(), 1, ep,
                                 ctx->dbg.as<int32_t>(), ctx->sms, s));
    else
        CK(launch_gram_i8(ctx->ops.as<uint8_t>(), ld, m, ctx->tiles.as<Tile>(), 1, ep, ctx->dbg.as<int32_t>(),
                          ctx->sms, s));
    ctx->kernels += 3;
    unsigned int herr[4];
    CK(cudaMemcpyAsync(out, ctx->dbg.p, 4 * 128 * 256, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(herr, ctx->err.p, 16, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (herr[0]) return fail(ctx, LDSC_E_TIMEOUT, "Gram kernel wait timed out");
    return LDSC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// regressions
// ---------------------------------------------------------------------------

namespace {

// Launches body(s) through a cached graph: captured and instantiated on the
// first call with this key, replayed afterwards.
template <typename F>
cudaError_t graph_launch(ldsc_ctx* ctx, const std::vector<uint64_t>& key, cudaStream_t s, F&& body) {
    GraphCache& gc = ctx->graphs;
    for (auto& x : gc.e)
        if (x.key == key) {
            x.tick = ++gc.tick;
            ctx->graph_launches++;
            return cudaGraphLaunch(x.exec, s);
        }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const cudaError_t eb = body(s);
    e = cudaStreamEndCapture(s, &g);
    if (eb != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return eb != cudaSuccess ? eb : e;
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return e;
    if (gc.e.size() >= 16) {
        size_t old = 0;
        for (size_t i = 1; i < gc.e.size(); i++)
            if (gc.e[i].tick < gc.e[old].tick) old = i;
        cudaGraphExecDestroy(gc.e[old].exec);
        gc.e.erase(gc.e.begin() + (long)old);
    }
    gc.e.push_back(GraphCache::Entry{key, ex, ++gc.tick});
    ctx->graph_launches++;
    return cudaGraphLaunch(ex, s);
}

static uint64_t dbits(double v) {
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
}

// Device copies (or views) of the inputs shared by every job of a batch.
int reg_inputs(ldsc_ctx* ctx, int device_pointers, uint64_t n, const double* ld, const double* wld,
               const double** d_ld, const double** d_wld) {
    if (device_pointers) {
        *d_ld = ld;
        *d_wld = wld;
        return LDSC_OK;
    }
    cudaStream_t s = ctx->stream;
    CK(ctx->rg_ld.ensure(8 * n));
    CK(ctx->rg_wld.ensure(8 * n));
    CK(cudaMemcpyAsync(ctx->rg_ld.p, ld, 8 * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->rg_wld.p, wld, 8 * n, cudaMemcpyHostToDevice, s));
    *d_ld = ctx->rg_ld.as<double>();
    *d_wld = ctx->rg_wld.as<double>();
    return LDSC_OK;
}

const double* dev_array(ldsc_ctx* ctx, DevBuf& buf, const double* src, size_t count, int device_pointers,
                        cudaError_t* err) {
    *err = cudaSuccess;
    if (!src) return nullptr;
    if (device_pointers) return src;
    *err = buf.ensure(8 * count);
    if (*err != cudaSuccess) return nullptr;
    *err = cudaMemcpyAsync(buf.p, src, 8 * count, cudaMemcpyHostToDevice, ctx->stream);
    return buf.as<double>();
}

}  // namespace

extern "C" int ldsc_h2_batch(ldsc_ctx* ctx, const ldsc_h2_args* a, ldsc_h2_result* res) {
    if (!ctx || !a || !res) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    const uint64_t n = a->n_snp;
    const int T = (int)a->n_traits;
    if (T == 0) return LDSC_OK;
    if (n == 0 || !a->chi2 || !a->ref_l2 || !a->w_l2 || (!a->n_per_snp && !a->n_scalar))
        return fail(ctx, LDSC_E_INVALID, "ldsc_h2_batch: missing inputs");
    // n_blocks = min(n_obs, --n-blocks) as the callers do (src/regressions.rs:697, 2389)
    const int nb = (int)std::min<uint64_t>(a->n_blocks, n);
    if (nb < 2) return fail(ctx, LDSC_E_INVALID, "n_blocks must be >= 2");
    if (!(a->m_snps > 0)) return fail(ctx, LDSC_E_INVALID, "M must be > 0");
    const bool two = a->two_step != 0;
    if (two && a->fixed_intercept)
        return fail(ctx, LDSC_E_INVALID, "twostep is not compatible with constrained intercept");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const double *d_ld, *d_wld;
    int rc = reg_inputs(ctx, a->device_pointers, n, a->ref_l2, a->w_l2, &d_ld, &d_wld);
    if (rc != LDSC_OK) return rc;
    cudaError_t e;
    const double* d_y = dev_array(ctx, ctx->rg_y, a->chi2, (size_t)T * n, a->device_pointers, &e);
    CK(e);
    const double* d_n = dev_array(ctx, ctx->rg_n, a->n_per_snp, (size_t)T * n, a->device_pointers, &e);
    CK(e);
    std::vector<RegJob> jobs(T);
    for (int t = 0; t < T; t++) {
        RegJob& jb = jobs[t];
        std::memset(&jb, 0, sizeof(jb));
        jb.ya = d_y + (size_t)t * n;
        jb.ymode = REG_Y_DIRECT;
        jb.kind = REG_HSQ;
        jb.n1 = d_n ? d_n + (size_t)t * n : nullptr;
        jb.n1s = a->n_scalar && !d_n ? (a->device_pointers ? 0.0 : a->n_scalar[t]) : 0.0;
        jb.fixed = a->fixed_intercept;
        jb.fixed_int = a->intercept;
        jb.hsq1 = jb.hsq2 = -1;
        jb.int_from = -1;
    }
    if (a->device_pointers && !d_n) {
        // scalar sample sizes live on the device: fetch them (T doubles)
        std::vector<double> ns(T);
        CK(cudaMemcpyAsync(ns.data(), a->n_scalar, 8 * (size_t)T, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (int t = 0; t < T; t++) jobs[t].n1s = ns[t];
    }
    // --two-step (src/h2.rs:319-393): jobs [0, T) fit both parameters on the
    // SNPs with chi2 below the cutoff, jobs [T, 2T) refit the slope on all SNPs
    // with that intercept held, over the same jackknife blocks
    const int J = two ? 2 * T : T;
    const int nch = (int)((n + 4095) / 4096);
    if (two) {
        CK(ctx->ts_seps.ensure(sizeof(int32_t) * (size_t)T * (nb + 1)));
        CK(ctx->ts_n1.ensure(sizeof(int32_t) * (size_t)T));
        CK(ctx->ts_cnt.ensure(sizeof(int32_t) * (size_t)T * nch));
        CK(ctx->ts_dv.ensure(sizeof(double) * 2 * (size_t)J * nb));
        CK(ctx->ts_outs.ensure(sizeof(RegOut) * (size_t)J));
        jobs.resize(J);
        for (int t = 0; t < T; t++) {
            RegJob& s1 = jobs[t];
            s1.seps = ctx->ts_seps.as<int32_t>() + (size_t)t * (nb + 1);
            s1.use_mask = 1;
            s1.mask_max = a->two_step_cutoff;
            s1.ld_from_x = 1;
            RegJob& s2 = jobs[T + t];
            s2 = jobs[t];
            s2.use_mask = 0;
            s2.ld_from_x = 0;
            s2.fixed = 1;
            s2.int_from = t;
        }
    }
    CK(ctx->rg_jobs.ensure(sizeof(RegJob) * J));
    CK(ctx->rg_states.ensure(sizeof(RegState) * J));
    CK(ctx->rg_outs.ensure(sizeof(RegOut) * T));
    CK(ctx->rg_part.ensure(sizeof(double) * 5 * (size_t)J * nb));
    CK(ctx->rg_sel.ensure(sizeof(double) * 2 * T));
    CK(cudaMemcpyAsync(ctx->rg_jobs.p, jobs.data(), sizeof(RegJob) * J, cudaMemcpyHostToDevice, s));
    // the whole pipeline (8 regression kernels + the median; 2 x 8 + 3 for
    // --two-step) replays as one graph
    const std::vector<uint64_t> gkey{1, (uint64_t)T, n, (uint64_t)nb, dbits(a->m_snps), (uint64_t)a->want_lambda_gc,
                                     (uint64_t)d_ld, (uint64_t)d_wld, (uint64_t)ctx->rg_jobs.p,
                                     (uint64_t)ctx->rg_states.p, (uint64_t)ctx->rg_outs.p, (uint64_t)ctx->rg_part.p,
                                     (uint64_t)ctx->rg_sel.p, (uint64_t)two, (uint64_t)ctx->ts_seps.p,
                                     (uint64_t)ctx->ts_dv.p, (uint64_t)ctx->ts_outs.p};
    CK(graph_launch(ctx, gkey, s, [&](cudaStream_t gs) -> cudaError_t {
        RegJob* dj = ctx->rg_jobs.as<RegJob>();
        RegState* dst = ctx->rg_states.as<RegState>();
        cudaError_t e2;
        if (!two) {
            e2 = launch_regressions(dj, dst, ctx->rg_outs.as<RegOut>(), nullptr, ctx->rg_part.as<double>(), nullptr,
                                    d_ld, d_wld, n, nb, a->m_snps, T, gs);
        } else {
            RegOut* o12 = ctx->ts_outs.as<RegOut>();
            double* dv = ctx->ts_dv.as<double>();
            e2 = launch_twostep_seps(dj, n, nb, ctx->ts_seps.as<int32_t>(), ctx->ts_n1.as<int32_t>(),
                                     ctx->ts_cnt.as<int32_t>(), T, gs);
            if (e2 == cudaSuccess)
                e2 = launch_regressions(dj, dst, o12, nullptr, ctx->rg_part.as<double>(), nullptr, d_ld, d_wld, n,
                                        nb, a->m_snps, T, gs, dv);
            if (e2 == cudaSuccess)
                e2 = launch_regressions(dj + T, dst + T, o12 + T, o12, ctx->rg_part.as<double>() + (size_t)5 * T * nb,
                                        nullptr, d_ld, d_wld, n, nb, a->m_snps, T, gs, dv + (size_t)2 * T * nb);
            if (e2 == cudaSuccess)
                e2 = launch_twostep_combine(o12, o12 + T, dst + T, dv, dv + (size_t)2 * T * nb, nb, a->m_snps,
                                            ctx->rg_outs.as<RegOut>(), T, gs);
        }
        if (e2 != cudaSuccess || !a->want_lambda_gc) return e2;
        // median (src/h2.rs:394-414): middle order statistic, mean of the two for even n
        // (rank n/2 in sel[0, T), rank n/2 - 1 in sel[T, 2T) for even n)
        return launch_select_mid(ctx->rg_jobs.as<RegJob>(), n, n % 2 ? n / 2 : n / 2 - 1, n / 2,
                                 ctx->rg_sel.as<double>() + T, ctx->rg_sel.as<double>(), T, gs);
    }));
    ctx->kernels += (two ? 19 : 8) + (a->want_lambda_gc ? 1 : 0);
    std::vector<RegOut> outs(T);
    std::vector<double> sel(2 * T, NAN);
    std::vector<int32_t> n1(two ? T : 0);
    CK(cudaMemcpyAsync(outs.data(), ctx->rg_outs.p, sizeof(RegOut) * T, cudaMemcpyDeviceToHost, s));
    if (a->want_lambda_gc) CK(cudaMemcpyAsync(sel.data(), ctx->rg_sel.p, 8 * 2 * (size_t)T, cudaMemcpyDeviceToHost, s));
    if (two) CK(cudaMemcpyAsync(n1.data(), ctx->ts_n1.p, 4 * (size_t)T, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int t = 0; t < (two ? T : 0); t++)  // jackknife_fast on the step-1 SNPs (src/h2.rs:121-123)
        if (n1[t] < nb) return fail(ctx, LDSC_E_INVALID, "More blocks than data points.");
    for (int t = 0; t < T; t++) {
        const RegOut& o = outs[t];
        ldsc_h2_result& r = res[t];
        r.h2 = o.tot;
        r.h2_se = o.tot_se;
        r.intercept = o.intercept;
        r.intercept_se = o.intercept_se;
        r.mean_chi2 = o.mean_y;
        r.coef = o.est[0] / o.nbar;
        r.coef_se = o.se[0] / o.nbar;
        r.lambda_gc = NAN;
        if (a->want_lambda_gc) {
            const double med = n % 2 == 0 ? (sel[t] + sel[T + t]) / 2.0 : sel[t];
            r.lambda_gc = med / 0.4549;
        }
        if (!a->fixed_intercept && r.mean_chi2 > 1.0) {
            r.ratio = (r.intercept - 1.0) / (r.mean_chi2 - 1.0);
            r.ratio_se = r.intercept_se / (r.mean_chi2 - 1.0);
        } else {
            r.ratio = NAN;
            r.ratio_se = NAN;
        }
    }
    return LDSC_OK;
}

extern "C" int ldsc_h2_partitioned(ldsc_ctx* ctx, const ldsc_h2p_args* a, ldsc_h2p_result* res) {
    if (!ctx || !a || !res) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    const uint64_t n = a->n_snp;
    const int T = (int)a->n_traits, K = (int)a->n_annot;
    if (T == 0) return LDSC_OK;
    if (n == 0 || K == 0 || !a->chi2 || !a->ref_l2 || !a->w_l2 || !a->m_vec || !a->chisq_max ||
        (!a->n_per_snp && !a->n_scalar))
        return fail(ctx, LDSC_E_INVALID, "ldsc_h2_partitioned: missing inputs");
    if (n > (uint64_t)INT32_MAX) return fail(ctx, LDSC_E_INVALID, "ldsc_h2_partitioned: more than 2^31-1 SNPs");
    const bool fixed = a->fixed_intercept != 0;
    const int P = part_params(K, fixed), Q = P + 1;
    if (P > 160)
        return fail(ctx, LDSC_E_INVALID, "ldsc_h2_partitioned: too many annotations (P = K + 1 must be <= 160)");
    const uint64_t ld = a->ref_ld ? a->ref_ld : n;
    if (ld < n) return fail(ctx, LDSC_E_INVALID, "ldsc_h2_partitioned: ref_ld < n_snp");
    if (a->n_blocks < 2) return fail(ctx, LDSC_E_INVALID, "n_blocks must be >= 2");
    double m_tot = 0.0;
    for (int k = 0; k < K; k++) m_tot += a->m_vec[k];
    if (!(m_tot > 0)) return fail(ctx, LDSC_E_INVALID, "sum of M must be > 0");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    cudaError_t e;
    // inputs on the device
    const double* d_l2 = a->ref_l2;
    uint64_t d_ld = ld;
    if (!a->device_pointers) {
        CK(ctx->p_l2.ensure(8 * n * (uint64_t)K));
        CK(cudaMemcpy2DAsync(ctx->p_l2.p, 8 * n, a->ref_l2, 8 * ld, 8 * n, (size_t)K, cudaMemcpyHostToDevice, s));
        d_l2 = ctx->p_l2.as<double>();
        d_ld = n;
    }
    const double* d_w = dev_array(ctx, ctx->p_w, a->w_l2, n, a->device_pointers, &e);
    CK(e);
    const double* d_y = dev_array(ctx, ctx->p_y, a->chi2, (size_t)T * n, a->device_pointers, &e);
    CK(e);
    const double* d_n = dev_array(ctx, ctx->p_n, a->n_per_snp, (size_t)T * n, a->device_pointers, &e);
    CK(e);
    std::vector<double> ns(T, 0.0);
    if (!d_n) {
        if (a->device_pointers) {
            CK(cudaMemcpyAsync(ns.data(), a->n_scalar, 8 * (size_t)T, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        } else {
            for (int t = 0; t < T; t++) ns[t] = a->n_scalar[t];
        }
    }
    CK(ctx->p_m.ensure(8 * (size_t)K));
    CK(cudaMemcpyAsync(ctx->p_m.p, a->m_vec, 8 * (size_t)K, cudaMemcpyHostToDevice, s));
    // kept SNPs (chi2 < chisq_max) and the jackknife block starts over them
    // (get_separators on the filtered SNPs, src/h2.rs:31-41)
    const int nb = (int)a->n_blocks;
    const int nch = (int)((n + 4095) / 4096);
    std::vector<RegJob> rj(T);
    for (int t = 0; t < T; t++) {
        std::memset(&rj[t], 0, sizeof(RegJob));
        rj[t].ya = d_y + (size_t)t * n;
        rj[t].ymode = REG_Y_DIRECT;
        rj[t].use_mask = 1;
        rj[t].mask_max = a->chisq_max[t];
        rj[t].int_from = -1;
    }
    CK(ctx->p_rjobs.ensure(sizeof(RegJob) * T));
    CK(ctx->p_seps.ensure(sizeof(int32_t) * 2 * (size_t)T * (nb + 1)));
    CK(ctx->p_n1.ensure(sizeof(int32_t) * T));
    CK(ctx->p_cnt.ensure(sizeof(int32_t) * (size_t)T * nch));
    CK(cudaMemcpyAsync(ctx->p_rjobs.p, rj.data(), sizeof(RegJob) * T, cudaMemcpyHostToDevice, s));
    RegJob* drj = ctx->p_rjobs.as<RegJob>();
    int32_t* seps = ctx->p_seps.as<int32_t>();
    CK(launch_twostep_seps(drj, n, nb, seps, ctx->p_n1.as<int32_t>(), ctx->p_cnt.as<int32_t>(), T, s));
    ctx->kernels += 2;
    std::vector<int32_t> n1(T);
    CK(cudaMemcpyAsync(n1.data(), ctx->p_n1.p, 4 * (size_t)T, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int t = 0; t < T; t++)
        if (n1[t] < 2) return fail(ctx, LDSC_E_INVALID, "fewer than 2 SNPs below the chi2 cut");
    // traits with at least nb kept SNPs run together; a trait with fewer runs
    // alone with nb = its SNP count (src/regressions.rs:1151)
    std::vector<std::vector<int>> groups(1);
    for (int t = 0; t < T; t++) {
        if (n1[t] >= nb)
            groups[0].push_back(t);
        else
            groups.push_back({t});
    }
    std::vector<PartJob> pj(T);
    std::vector<int> gnb(groups.size()), gofs(groups.size());
    size_t res_len = 0;
    for (size_t gi = 0, o = 0; gi < groups.size(); gi++) {
        gnb[gi] = gi == 0 ? nb : n1[groups[gi][0]];
        gofs[gi] = (int)o;
        for (int t : groups[gi]) {
            PartJob& jb = pj[o++];
            jb.chi2 = d_y + (size_t)t * n;
            jb.nv = d_n ? d_n + (size_t)t * n : nullptr;
            jb.ns = ns[t];
            // group 0 uses the block starts above; others get their own below
            jb.seps = gi == 0 ? seps + (size_t)t * (nb + 1) : nullptr;
            jb.mask_max = a->chisq_max[t];
            jb.n_obs = (double)n1[t];
            jb.fixed = fixed;
            jb.fixed_int = fixed ? a->intercept : 0.0;
            res_len += part_result_len(gnb[gi], K, P);
        }
    }
    // block starts of the small traits (fewer than nb + 1 each), after the
    // T x (nb + 1) of the first pass
    size_t off = (size_t)T * (nb + 1);
    for (size_t gi = 1; gi < groups.size(); gi++) {
        const int t = groups[gi][0];
        int32_t* sp = seps + off;
        CK(launch_twostep_seps(drj + t, n, gnb[gi], sp, ctx->p_n1.as<int32_t>() + t, ctx->p_cnt.as<int32_t>(), 1, s));
        ctx->kernels += 2;
        pj[gofs[gi]].seps = sp;
        off += (size_t)gnb[gi] + 1;
    }
    size_t max_gj = 0;
    for (auto& gr : groups) max_gj = std::max(max_gj, gr.size());
    // traits per launch, so the block Grams stay within a fixed budget
    const size_t chunk = (size_t)part_trait_chunk((int)std::max<size_t>(max_gj, 1), nb, Q);
    max_gj = std::min(max_gj, chunk);
    CK(ctx->p_jobs.ensure(sizeof(PartJob) * T));
    CK(ctx->p_st.ensure(sizeof(PartState) * T));
    CK(ctx->p_xtot.ensure(8 * n));
    CK(ctx->p_part.ensure(8 * 3 * max_gj * (size_t)nb));
    CK(ctx->p_gram.ensure(8 * max_gj * (size_t)nb * Q * Q));
    CK(ctx->p_tot.ensure(8 * max_gj * (size_t)Q * Q));
    CK(ctx->p_sol.ensure(8 * max_gj * (size_t)(nb + 1) * P));
    CK(ctx->p_res.ensure(8 * res_len));
    CK(cudaMemcpyAsync(ctx->p_jobs.p, pj.data(), sizeof(PartJob) * T, cudaMemcpyHostToDevice, s));
    std::vector<double> hres(res_len);
    size_t ro = 0;
    bool first = true;
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const int gb = gnb[gi];
        for (size_t c0 = 0; c0 < groups[gi].size(); c0 += chunk) {
            const int nj = (int)std::min(chunk, groups[gi].size() - c0);
            const size_t jo = (size_t)gofs[gi] + c0;
            CK(launch_partitioned(ctx->p_jobs.as<PartJob>() + jo, ctx->p_st.as<PartState>() + jo, d_l2, d_ld, K,
                                  fixed, d_w, n, gb, m_tot, ctx->p_m.as<double>(), ctx->p_xtot.as<double>(), first,
                                  ctx->p_part.as<double>(), ctx->p_gram.as<double>(), ctx->p_tot.as<double>(),
                                  ctx->p_sol.as<double>(), ctx->p_res.as<double>() + ro, nj, s));
            ctx->kernels += first ? 7 : 6;
            first = false;
            ro += (size_t)nj * part_result_len(gb, K, P);
        }
    }
    CK(cudaMemcpyAsync(hres.data(), ctx->p_res.p, 8 * res_len, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ro = 0;
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const int gb = gnb[gi];
        for (int t : groups[gi]) {
            const double* R = hres.data() + ro;
            ro += part_result_len(gb, K, P);
            const double* est = R;
            const double* cov = est + P;
            const double* dv = cov + (size_t)P * P;
            const double* h2a = dv + (size_t)gb * P;
            const double* sc = h2a + K;
            if (a->est) std::memcpy(a->est + (size_t)t * P, est, 8 * (size_t)P);
            if (a->cov) std::memcpy(a->cov + (size_t)t * P * P, cov, 8 * (size_t)P * P);
            if (a->delete_values) {
                double* o = a->delete_values + (size_t)t * nb * P;
                std::memcpy(o, dv, 8 * (size_t)gb * P);
                for (size_t x = (size_t)gb * P; x < (size_t)nb * P; x++) o[x] = NAN;
            }
            if (a->h2_annot) std::memcpy(a->h2_annot + (size_t)t * K, h2a, 8 * (size_t)K);
            ldsc_h2p_result& r = res[t];
            r.h2_total = sc[0];
            r.h2_total_se = sc[1];
            r.intercept = sc[2];
            r.intercept_se = sc[3];
            r.n_mean = sc[4];
            r.mean_chi2 = sc[5];
            r.n_obs = (uint64_t)sc[6];
            r.n_blocks = (uint32_t)gb;
        }
    }
    return LDSC_OK;
}

extern "C" int ldsc_rg_batch(ldsc_ctx* ctx, const ldsc_rg_args* a, ldsc_rg_result* res) {
    if (!ctx || !a || !res) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    const uint64_t n = a->n_snp;
    const int P = (int)a->n_pairs;
    if (P == 0) return LDSC_OK;
    if (n == 0 || !a->z1 || !a->z2 || !a->n1 || !a->n2 || !a->ref_l2 || !a->w_l2)
        return fail(ctx, LDSC_E_INVALID, "ldsc_rg_batch: missing inputs");
    // n_blocks = min(n_obs, --n-blocks) as the callers do (src/regressions.rs:697, 2389)
    const int nb = (int)std::min<uint64_t>(a->n_blocks, n);
    if (nb < 2) return fail(ctx, LDSC_E_INVALID, "n_blocks must be >= 2");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const double *d_ld, *d_wld;
    int rc = reg_inputs(ctx, a->device_pointers, n, a->ref_l2, a->w_l2, &d_ld, &d_wld);
    if (rc != LDSC_OK) return rc;
    cudaError_t e;
    const double* d_z1 = dev_array(ctx, ctx->rg_y, a->z1, (size_t)P * n, a->device_pointers, &e);
    CK(e);
    const double* d_z2 = dev_array(ctx, ctx->rg_y2, a->z2, (size_t)P * n, a->device_pointers, &e);
    CK(e);
    std::vector<double> n1(P), n2(P);
    if (a->device_pointers) {
        CK(cudaMemcpyAsync(n1.data(), a->n1, 8 * (size_t)P, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(n2.data(), a->n2, 8 * (size_t)P, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    } else {
        for (int p = 0; p < P; p++) {
            n1[p] = a->n1[p];
            n2[p] = a->n2[p];
        }
    }
    // jobs 0..2P-1: h2 of z1^2 and z2^2; jobs 2P..3P-1: genetic covariance
    std::vector<RegJob> jobs(3 * P);
    std::vector<RgPairIdx> idx(P);
    for (int p = 0; p < P; p++) {
        for (int q = 0; q < 3; q++) {
            RegJob& jb = jobs[q == 2 ? 2 * P + p : 2 * p + q];
            std::memset(&jb, 0, sizeof(jb));
            jb.hsq1 = jb.hsq2 = -1;
            jb.int_from = -1;
        }
        RegJob& h1 = jobs[2 * p];
        h1.ya = d_z1 + (size_t)p * n;
        h1.ymode = REG_Y_SQUARE;
        h1.kind = REG_HSQ;
        h1.n1s = n1[p];
        RegJob& h2 = jobs[2 * p + 1];
        h2.ya = d_z2 + (size_t)p * n;
        h2.ymode = REG_Y_SQUARE;
        h2.kind = REG_HSQ;
        h2.n1s = n2[p];
        RegJob& gc = jobs[2 * P + p];
        gc.ya = d_z1 + (size_t)p * n;
        gc.yb = d_z2 + (size_t)p * n;
        gc.ymode = REG_Y_PRODUCT;
        gc.kind = REG_GENCOV;
        gc.n1s = n1[p];
        gc.n2s = n2[p];
        gc.hsq1 = 2 * p;
        gc.hsq2 = 2 * p + 1;
        idx[p] = RgPairIdx{2 * p, 2 * p + 1, 2 * P + p};
    }
    const int J = 3 * P;
    CK(ctx->rg_jobs.ensure(sizeof(RegJob) * J));
    CK(ctx->rg_states.ensure(sizeof(RegState) * J));
    CK(ctx->rg_outs.ensure(sizeof(RegOut) * J));
    CK(ctx->rg_part.ensure(sizeof(double) * 5 * (size_t)J * nb));
    CK(ctx->rg_tdel.ensure(sizeof(double) * (size_t)J * nb));
    CK(ctx->rg_pairs.ensure(sizeof(RgPairIdx) * P));
    CK(ctx->rg_res.ensure(sizeof(RgOut) * P));
    CK(cudaMemcpyAsync(ctx->rg_jobs.p, jobs.data(), sizeof(RegJob) * J, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->rg_pairs.p, idx.data(), sizeof(RgPairIdx) * P, cudaMemcpyHostToDevice, s));
    RegJob* dj = ctx->rg_jobs.as<RegJob>();
    RegState* dst = ctx->rg_states.as<RegState>();
    RegOut* dout = ctx->rg_outs.as<RegOut>();
    double* dtd = ctx->rg_tdel.as<double>();
    // stage 1: the h2 fits; stage 2: the covariance fits, whose weights use
    // them; then the ratio jackknife -- 17 kernels replayed as one graph
    const std::vector<uint64_t> gkey{2, (uint64_t)P, n, (uint64_t)nb, dbits(a->m_snps), (uint64_t)d_ld,
                                     (uint64_t)d_wld, (uint64_t)dj, (uint64_t)dst, (uint64_t)dout,
                                     (uint64_t)ctx->rg_part.p, (uint64_t)dtd, (uint64_t)ctx->rg_pairs.p,
                                     (uint64_t)ctx->rg_res.p};
    CK(graph_launch(ctx, gkey, s, [&](cudaStream_t gs) -> cudaError_t {
        cudaError_t e2 = launch_regressions(dj, dst, dout, nullptr, ctx->rg_part.as<double>(), dtd, d_ld, d_wld, n,
                                            nb, a->m_snps, 2 * P, gs, nullptr, REG_FORM_HSQ_SQUARE);
        if (e2 != cudaSuccess) return e2;
        e2 = launch_regressions(dj + 2 * P, dst + 2 * P, dout + 2 * P, dout,
                                ctx->rg_part.as<double>() + (size_t)2 * P * nb * 5, dtd + (size_t)2 * P * nb, d_ld,
                                d_wld, n, nb, a->m_snps, P, gs, nullptr, REG_FORM_GENCOV_PRODUCT);
        if (e2 != cudaSuccess) return e2;
        return launch_rg_finish(ctx->rg_pairs.as<RgPairIdx>(), dout, dtd, nb, ctx->rg_res.as<RgOut>(), P, gs);
    }));
    ctx->kernels += 17;
    std::vector<RgOut> outs(P);
    CK(cudaMemcpyAsync(outs.data(), ctx->rg_res.p, sizeof(RgOut) * P, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int p = 0; p < P; p++) {
        const RgOut& o = outs[p];
        ldsc_rg_result& r = res[p];
        r.rg = o.rg;
        r.rg_se = o.rg_se;
        r.gencov = o.gencov;
        r.gencov_se = o.gencov_se;
        r.gencov_intercept = o.gencov_intercept;
        r.gencov_intercept_se = o.gencov_intercept_se;
        r.h2_1 = o.h2_1;
        r.h2_1_se = o.h2_1_se;
        r.h2_2 = o.h2_2;
        r.h2_2_se = o.h2_2_se;
        r.mean_z1z2 = o.mean_z1z2;
        // p_z_norm: two-sided normal p-value (1 - chi2_1 cdf of z^2)
        if (std::isfinite(r.rg_se) && r.rg_se != 0.0) {
            r.z = r.rg / r.rg_se;
            r.p = std::isfinite(r.z) ? std::erfc(std::fabs(r.z) / std::sqrt(2.0)) : 0.0;
        } else {
            r.z = INFINITY;
            r.p = 0.0;
        }
    }
    return LDSC_OK;
}
