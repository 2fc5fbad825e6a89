// noalloc.cu -- the INT8-exact l2 pass without any device allocation.
//
// Some callers cannot call cudaMalloc: a host that owns all device memory
// through its own arena (a JVM / Rust / serving runtime with a fixed memory
// budget, where an allocation behind its back breaks its accounting), and
// latency-critical request loops where an allocation or free would
// synchronise the device.  ldsc_l2_int8_noalloc() serves them: the caller
// passes device buffers for the inputs and outputs, and the kernels' scratch
// (INT8 genotype/mask operands, per-SNP statistics, the tile list, the error
// word) lives in one file-scope device array of fixed size,
// LDSC_NOALLOC_SCRATCH_BYTES.  Every GPU that loads this library holds that
// array until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents: calls that overlap on the GPU (different streams, or host threads
// without ordering) race on it.  Each call clears what must start at zero (the
// error word) and overwrites everything else it reads.  The call runs on the
// current device: the caller's buffers and stream must belong to it.  The
// first call on a device looks up the array's device address
// (cudaGetSymbolAddress, once per device, with that device current) and keeps
// it for the life of the process; make that first call before any stream
// capture begins.  A device reset (cudaDeviceReset) ends the context that
// address belongs to, so after one the library must be unloaded and loaded
// again before this entry point is used.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ldsc_b200.h"
#include "engine.h"
#include "plan.h"

namespace {

static __device__ __align__(256) unsigned char g_scratch[LDSC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};
std::string g_last_error;

uint64_t up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// Device address of g_scratch on the current device (looked up once per device).
int scratch_base(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(LDSC_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return set_error(LDSC_E_UNSUPPORTED, "device index too large");
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return set_error(LDSC_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return LDSC_OK;
}

}  // namespace

extern "C" int ldsc_noalloc_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return LDSC_E_INVALID;
    std::lock_guard<std::mutex> g(g_mu);
    std::snprintf(buf, len, "%s", g_last_error.c_str());
    return LDSC_OK;
}

extern "C" int ldsc_l2_int8_noalloc(const uint8_t* d_rows, uint64_t pitch, uint64_t n_indiv, uint64_t n_snp,
                                    const int64_t* left, double* d_l2, double* d_maf, void* stream) {
    using namespace ldsc;
    std::lock_guard<std::mutex> g(g_mu);
    if (n_snp == 0) return LDSC_OK;
    if (!d_rows || !left || !d_l2 || !d_maf) return set_error(LDSC_E_INVALID, "null argument");
    if (n_indiv == 0 || n_indiv > 1000000) return set_error(LDSC_E_INVALID, "n_indiv must be in 1..1,000,000");
    if (pitch < (n_indiv + 3) / 4 || pitch % 16 != 0 || (reinterpret_cast<uintptr_t>(d_rows) & 15) != 0)
        return set_error(LDSC_E_INVALID, "rows must be 16-byte aligned with a pitch >= ceil(n_indiv/4), multiple of 16");
    for (uint64_t j = 0; j < n_snp; j++)
        if (left[j] < 0 || (uint64_t)left[j] > j || (j > 0 && left[j] < left[j - 1]))
            return set_error(LDSC_E_INVALID, "left limits must satisfy 0 <= left[j] <= j, non-decreasing");

    // scratch layout
    const uint64_t m = n_snp;
    const uint64_t ld = up(n_indiv, 128);
    std::vector<int64_t> lv(left, left + m);
    const std::vector<Tile> tiles = band_tiles(lv, 64, 128);
    uint64_t off = 0;
    auto take = [&](uint64_t bytes) {
        const uint64_t o = off;
        off = up(off + bytes, 256);
        return o;
    };
    const uint64_t o_ops = take(2 * m * ld), o_n = take(4 * m), o_s = take(4 * m), o_q = take(4 * m),
                   o_mean = take(8 * m), o_inv = take(8 * m), o_qinv = take(8 * m), o_aeff = take(8 * m),
                   o_left = take(8 * m), o_tiles = take(sizeof(Tile) * (tiles.size() + 1)), o_err = take(16);
    if (off > (uint64_t)LDSC_NOALLOC_SCRATCH_BYTES)
        return set_error(LDSC_E_INVALID, "ldsc_l2_int8_noalloc: n_snp=" + std::to_string(m) + ", n_indiv=" +
                                             std::to_string(n_indiv) + " needs " + std::to_string(off) +
                                             " bytes of scratch; the static scratch holds " +
                                             std::to_string((uint64_t)LDSC_NOALLOC_SCRATCH_BYTES));
    unsigned char* base = nullptr;
    int rc = scratch_base(&base);
    if (rc != LDSC_OK) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    auto ck = [&](cudaError_t e, const char* what) -> int {
        if (e == cudaSuccess) return (int)LDSC_OK;
        return set_error(LDSC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    if ((rc = ck(cudaMemcpyAsync(base + o_left, lv.data(), 8 * m, cudaMemcpyHostToDevice, s), "copy left"))) return rc;
    if (!tiles.empty() &&
        (rc = ck(cudaMemcpyAsync(base + o_tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, s),
                 "copy tiles")))
        return rc;
    if ((rc = ck(cudaMemsetAsync(base + o_err, 0, 16, s), "clear error word"))) return rc;

    PanelView pv{d_rows, m, n_indiv, (n_indiv + 3) / 4, pitch};
    IndivSel sel{nullptr, n_indiv};
    RecStats st{};
    st.n = reinterpret_cast<int32_t*>(base + o_n);
    st.s = reinterpret_cast<int32_t*>(base + o_s);
    st.q = reinterpret_cast<int32_t*>(base + o_q);
    st.maf = d_maf;
    st.mean = reinterpret_cast<double*>(base + o_mean);
    st.inv_std = reinterpret_cast<double*>(base + o_inv);
    st.qinv = reinterpret_cast<double*>(base + o_qinv);
    uint8_t* ops = base + o_ops;
    if ((rc = ck(launch_decode_i8(pv, nullptr, (int64_t)m, sel, ops, ld, st, 0, s), "decode"))) return rc;
    if ((rc = ck(launch_finalize_stats((int64_t)m, n_indiv, st, nullptr, 1, 0, 0.0,
                                       reinterpret_cast<double*>(base + o_aeff), d_l2, s),
                 "finalize")))
        return rc;
    EpilogueArgs ep{};
    ep.left = reinterpret_cast<int64_t*>(base + o_left);
    ep.n = st.n;
    ep.s = st.s;
    ep.qinv = st.qinv;
    ep.aeff = reinterpret_cast<double*>(base + o_aeff);
    ep.l2 = d_l2;
    ep.m = (int64_t)m;
    ep.K = 1;
    const double N = (double)n_indiv;
    const double denom = n_indiv > 2 ? N - 2.0 : N;
    ep.r2u_a = 1.0 + 1.0 / denom;
    ep.r2u_b = -1.0 / denom;
    ep.err = reinterpret_cast<unsigned int*>(base + o_err);
    if (!tiles.empty() &&
        (rc = ck(launch_gram_i8(ops, ld, (int64_t)m, reinterpret_cast<Tile*>(base + o_tiles), (int64_t)tiles.size(),
                                ep, nullptr, sms, s),
                 "gram")))
        return rc;
    unsigned int herr = 0;
    if ((rc = ck(cudaMemcpyAsync(&herr, base + o_err, 4, cudaMemcpyDeviceToHost, s), "read error word"))) return rc;
    if ((rc = ck(cudaStreamSynchronize(s), "synchronize"))) return rc;
    if (herr) return set_error(LDSC_E_TIMEOUT, "a device wait in the Gram kernel exceeded its bound");
    return LDSC_OK;
}
