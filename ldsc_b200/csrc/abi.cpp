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
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ldsc_b200.h"
#include "engine.h"
#include "plan.h"

using namespace ldsc;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        if (bytes == 0) bytes = 16;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <typename T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct ldsc_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string last_error;
    uint64_t kernels = 0;
    // workspace (grow-only)
    DevBuf ops, xf64, xsk, recrows, keep, left, tiles, annot, aeff, aeff32, l2, maf, pq, err;
    DevBuf st_n, st_s, st_q, st_q3, st_q4, st_mean, st_inv, st_qinv, st_kappa, packed, tsum, dbg;
};

struct ldsc_panel {
    ldsc_ctx* ctx = nullptr;
    uint8_t* rows = nullptr;
    uint64_t n_snp = 0, n_indiv = 0, bpr = 0, pitch = 0;
};

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
    (void)flags;
    if (!out) return LDSC_E_INVALID;
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
    ldsc_ctx* c = new ldsc_ctx();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return LDSC_E_CUDA;
    }
    c->stream = c->own;
    *out = c;
    return LDSC_OK;
}

int ldsc_ctx_destroy(ldsc_ctx* ctx) {
    if (!ctx) return LDSC_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    DevBuf* bufs[] = {&ctx->ops, &ctx->xf64, &ctx->xsk, &ctx->recrows, &ctx->keep, &ctx->left,
                      &ctx->tiles, &ctx->annot, &ctx->aeff, &ctx->aeff32, &ctx->l2, &ctx->maf,
                      &ctx->pq, &ctx->err, &ctx->st_n, &ctx->st_s, &ctx->st_q, &ctx->st_q3,
                      &ctx->st_q4, &ctx->st_mean, &ctx->st_inv, &ctx->st_qinv, &ctx->st_kappa,
                      &ctx->packed, &ctx->tsum, &ctx->dbg};
    for (DevBuf* b : bufs) b->release();
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
    int mark() {
        cudaEventCreate(&ev[n]);
        cudaEventRecord(ev[n], s);
        return n++;
    }
    double ms(int a, int b) const {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[a], ev[b]);
        return (double)t;
    }
};

int run_l2(ldsc_ctx* ctx, const ldsc_panel* panel, const ldsc_l2_args* a, double* l2_out, double* maf_out,
           ldsc_perf* perf, double upload_secs) {
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
    if (a->precision != LDSC_PRECISION_FP64 && a->precision != LDSC_PRECISION_INT8)
        return fail(ctx, LDSC_E_INVALID, "unknown precision");
    if (!d && a->precision == LDSC_PRECISION_INT8 && n_used > 1000000)
        return fail(ctx, LDSC_E_UNSUPPORTED, "INT8 form supports up to 1,000,000 individuals");
    if (m > 0 && a->bed_idx) {
        for (int64_t i = 0; i < m; i++)
            if (a->bed_idx[i] >= panel->n_snp)
                return fail(ctx, LDSC_E_INVALID, "SNP index " + std::to_string(a->bed_idx[i]) +
                                                     " out of range (max " + std::to_string(panel->n_snp) + ")");
    } else if ((uint64_t)m > panel->n_snp) {
        return fail(ctx, LDSC_E_INVALID, "more SNP records than panel rows");
    }
    if (m == 0) {
        if (perf) *perf = pf;
        return LDSC_OK;
    }

    // ---- host plan ----
    LeftLimits L;
    std::string perr;
    if (!left_limits(m, a->chr, a->cm, a->bp, a->window_mode, a->window_size, a->window_snps, a->chunk_size,
                     a->snp_level_masking != 0, a->global_pass != 0, &L, &perr))
        return fail(ctx, LDSC_E_INVALID, perr);
    if (L.any_full && !a->yes_really)
        std::printf("WARNING: LD window spans the entire chromosome. Use --yes-really to silence this warning.\n");
    pf.n_pairs = L.n_pairs;
    const bool exact_i8 = !d && a->precision == LDSC_PRECISION_INT8;
    const int ta = exact_i8 ? 64 : 128, tb = 128;
    std::vector<Tile> tiles = band_tiles(L.left, ta, tb);
    pf.n_tiles = tiles.size();
    pf.gram_kind = d ? 2u : (exact_i8 ? 1u : 0u);

    cudaStream_t s = ctx->stream;
    CK(cudaSetDevice(ctx->device));
    const uint64_t kernels0 = ctx->kernels;

    // ---- device buffers ----
    const uint64_t nmom = (uint64_t)m;
    CK(ctx->left.ensure(sizeof(int64_t) * nmom));
    CK(ctx->tiles.ensure(sizeof(Tile) * (tiles.size() + 1)));
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
    if (K > 1) CK(ctx->aeff32.ensure(4 * nmom * K));
    if (a->annot) CK(ctx->annot.ensure(8 * nmom * K));
    if (a->bed_idx) CK(ctx->recrows.ensure(8 * nmom));
    if (a->keep_iids) CK(ctx->keep.ensure(8 * a->n_keep));

    CK(cudaMemcpyAsync(ctx->left.p, L.left.data(), 8 * nmom, cudaMemcpyHostToDevice, s));
    if (!tiles.empty())
        CK(cudaMemcpyAsync(ctx->tiles.p, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, s));
    if (a->annot) CK(cudaMemcpyAsync(ctx->annot.p, a->annot, 8 * nmom * K, cudaMemcpyHostToDevice, s));
    if (a->bed_idx) CK(cudaMemcpyAsync(ctx->recrows.p, a->bed_idx, 8 * nmom, cudaMemcpyHostToDevice, s));
    if (a->keep_iids) CK(cudaMemcpyAsync(ctx->keep.p, a->keep_iids, 8 * a->n_keep, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->err.p, 0, 16, s));

    PanelView pv{panel->rows, panel->n_snp, panel->n_indiv, panel->bpr, panel->pitch};
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

    Events ev(s);
    const int e0 = ev.mark();

    // ---- decode ----
    const uint64_t ld_i8 = round_up(n_used, 128);
    if (exact_i8) {
        CK(ctx->ops.ensure((size_t)2 * nmom * ld_i8));
        CK(launch_decode_i8(pv, rr, m, sel, ctx->ops.as<uint8_t>(), ld_i8, st, 0, s));
    } else {
        CK(launch_decode_i8(pv, rr, m, sel, nullptr, 0, st, maf_aware ? 1 : 0, s));
    }
    ctx->kernels++;
    CK(launch_finalize_stats(m, n_used, st, a->annot ? ctx->annot.as<double>() : nullptr, K, a->has_pq_exp,
                             a->pq_exp, ctx->aeff.as<double>(), K > 1 ? ctx->aeff32.as<float>() : nullptr,
                             ctx->l2.as<double>(), s));
    ctx->kernels++;
    const uint64_t ld_f64 = round_up(n_used, 128);
    if (!d && !exact_i8) {
        CK(ctx->xf64.ensure((size_t)8 * nmom * ld_f64));
        CK(launch_decode_f64(pv, rr, m, sel, st, ctx->xf64.as<double>(), ld_f64, s));
        ctx->kernels++;
    }
    const int e1 = ev.mark();
    int e_sk = -1;
    const uint64_t ld_sk = round_up(d ? d : 1, 8);
    if (d) {
        // CountSketch hash on the host, exactly the reference's stream (seed 42)
        std::vector<uint32_t> bucket(n_used);
        std::vector<float> sign(n_used);
        countsketch_hash(n_used, d, 42, bucket.data(), sign.data());
        const uint64_t npad = round_up(n_used, 16);
        std::vector<uint32_t> packed(npad, 0);
        std::vector<int32_t> tsum(d, 0);
        for (uint64_t i = 0; i < n_used; i++) {
            packed[i] = bucket[i] | (sign[i] < 0 ? 0x80000000u : 0u);
            tsum[bucket[i]] += sign[i] < 0 ? -1 : 1;
        }
        CK(ctx->packed.ensure(4 * npad));
        CK(ctx->tsum.ensure(4 * (size_t)d));
        CK(ctx->xsk.ensure((size_t)4 * nmom * ld_sk));
        CK(cudaMemcpyAsync(ctx->packed.p, packed.data(), 4 * npad, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(ctx->tsum.p, tsum.data(), 4 * (size_t)d, cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(ctx->xsk.p, 0, (size_t)4 * nmom * ld_sk, s));
        CK(launch_sketch_scatter(pv, rr, m, sel, ctx->packed.as<uint32_t>(), ctx->tsum.as<int32_t>(), d, st,
                                 ctx->xsk.as<float>(), ld_sk, s));
        ctx->kernels++;
        CK(cudaStreamSynchronize(s));  // host vectors go out of scope
        e_sk = ev.mark();
    }

    // ---- band Gram + epilogue ----
    EpilogueArgs ep{};
    ep.left = ctx->left.as<int64_t>();
    ep.n = st.n;
    ep.s = st.s;
    ep.qinv = st.qinv;
    ep.kappa = st.kappa;
    ep.aeff = ctx->aeff.as<double>();
    ep.aeff32 = K > 1 ? ctx->aeff32.as<float>() : nullptr;
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
    const int e2 = d ? e_sk : e1;
    if (!tiles.empty()) {
        if (d) {
            CK(launch_gram_f32(ctx->xsk.as<float>(), ld_sk, ld_sk, ctx->tiles.as<Tile>(), (int64_t)tiles.size(), ep,
                               maf_aware ? 1 : 0, ctx->sms, s));
        } else if (exact_i8) {
            CK(launch_gram_i8(ctx->ops.as<uint8_t>(), ld_i8, m, ctx->tiles.as<Tile>(), (int64_t)tiles.size(), ep,
                              nullptr, ctx->sms, s));
        } else {
            CK(launch_gram_f64(ctx->xf64.as<double>(), ld_f64, ld_f64, ctx->tiles.as<Tile>(), (int64_t)tiles.size(),
                               ep, ctx->sms, s));
        }
        ctx->kernels++;
    }
    const int e3 = ev.mark();
    CK(cudaMemcpyAsync(l2_out, ctx->l2.p, 8 * nmom * K, cudaMemcpyDeviceToHost, s));
    if (maf_out) CK(cudaMemcpyAsync(maf_out, ctx->maf.p, 8 * nmom, cudaMemcpyDeviceToHost, s));
    unsigned int herr[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(herr, ctx->err.p, 16, cudaMemcpyDeviceToHost, s));
    const int e4 = ev.mark();
    CK(cudaStreamSynchronize(s));
    if (herr[0] != 0)
        return fail(ctx, LDSC_E_TIMEOUT, "a device wait in the Gram kernel exceeded its bound (error word " +
                                             std::to_string(herr[0]) + ")");
    pf.norm_secs = ev.ms(e0, e1) / 1e3;
    if (d) pf.sketch_secs = ev.ms(e1, e_sk) / 1e3;
    pf.ab_dot_secs = ev.ms(e2, e3) / 1e3;
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
    const auto t0 = std::chrono::steady_clock::now();
    ldsc_panel* p = nullptr;
    rc = ldsc_panel_upload(ctx, bed_file + 3, len - 3, n_indiv, rows, &p);
    if (rc != LDSC_OK) return rc;
    const double up = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        rc = run_l2(ctx, p, args, l2_out, maf_out, perf, up);
    }
    ldsc_panel_destroy(p);
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
    cudaStream_t s = ctx->stream;
    CK(cudaSetDevice(ctx->device));
    std::vector<uint64_t> rows((size_t)m);
    for (int64_t i = 0; i < m; i++) rows[i] = b + (uint64_t)i;
    const uint64_t npad = round_up(n_used, 16);
    std::vector<uint32_t> packed(npad, 0);
    std::vector<int32_t> tsum(d, 0);
    for (uint64_t i = 0; i < n_used; i++) {
        if (bucket[i] >= d) return fail(ctx, LDSC_E_INVALID, "bucket index >= d");
        packed[i] = bucket[i] | (sign[i] < 0 ? 0x80000000u : 0u);
        tsum[bucket[i]] += sign[i] < 0 ? -1 : 1;
    }
    CK(ctx->recrows.ensure(8 * (size_t)m));
    CK(ctx->st_n.ensure(4 * (size_t)m));
    CK(ctx->st_s.ensure(4 * (size_t)m));
    CK(ctx->st_q.ensure(4 * (size_t)m));
    CK(ctx->maf.ensure(8 * (size_t)m));
    CK(ctx->st_mean.ensure(8 * (size_t)m));
    CK(ctx->st_inv.ensure(8 * (size_t)m));
    CK(ctx->st_qinv.ensure(8 * (size_t)m));
    CK(ctx->packed.ensure(4 * npad));
    CK(ctx->tsum.ensure(4 * (size_t)d));
    CK(ctx->xsk.ensure(4 * (size_t)m * d));
    if (keep) {
        CK(ctx->keep.ensure(8 * n_keep));
        CK(cudaMemcpyAsync(ctx->keep.p, keep, 8 * n_keep, cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemcpyAsync(ctx->recrows.p, rows.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->packed.p, packed.data(), 4 * npad, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->tsum.p, tsum.data(), 4 * (size_t)d, cudaMemcpyHostToDevice, s));
    PanelView pv{panel->rows, panel->n_snp, panel->n_indiv, panel->bpr, panel->pitch};
    IndivSel sel{keep ? ctx->keep.as<int64_t>() : nullptr, n_used};
    RecStats st{};
    st.n = ctx->st_n.as<int32_t>();
    st.s = ctx->st_s.as<int32_t>();
    st.q = ctx->st_q.as<int32_t>();
    st.maf = ctx->maf.as<double>();
    st.mean = ctx->st_mean.as<double>();
    st.inv_std = ctx->st_inv.as<double>();
    st.qinv = ctx->st_qinv.as<double>();
    const uint64_t* rr = ctx->recrows.as<uint64_t>();
    CK(launch_decode_i8(pv, rr, m, sel, nullptr, 0, st, 0, s));
    CK(launch_finalize_stats(m, n_used, st, nullptr, 0, 0, 0.0, nullptr, nullptr, nullptr, s));
    CK(launch_sketch_scatter(pv, rr, m, sel, ctx->packed.as<uint32_t>(), ctx->tsum.as<int32_t>(), d, st,
                             ctx->xsk.as<float>(), d, s));
    ctx->kernels += 3;
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
    CK(ctx->ops.ensure((size_t)2 * m * ld));
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
    CK(launch_decode_i8(pv, nullptr, m, sel, ctx->ops.as<uint8_t>(), ld, st, 0, s));
    CK(launch_finalize_stats(m, n, st, nullptr, 1, 0, 0.0, ctx->aeff.as<double>(), nullptr, ctx->l2.as<double>(), s));
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
