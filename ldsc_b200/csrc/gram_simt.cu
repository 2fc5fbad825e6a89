// gram_simt.cu -- band Gram on CUDA cores for the two non-integer forms:
//   * FP64 plain form: standardised f64 columns, val = x_k . x_j, and the
//     reference's fused unbiased-r^2 transform val^2 * r2u_a / N^2 + r2u_b
//     (src/l2/compute.rs:1067-1077, 2229-2235);
//   * FP32 CountSketch form: sketched, renormalised f32 rows, val = s_k . s_j,
//     then the quadratic bias inversion (+ MAF-aware shift) in f64
//     (src/l2/compute.rs:947-998).
// Tiles are 128 x 128 records, 256 threads, 8 x 8 outputs per thread.
// K-slices of 16 are copied into shared memory by cp.async, three in flight,
// row-major with an odd row stride (17 elements) so the 16 lanes that read
// one operand column hit distinct banks; rows past the record count are
// zero-filled by the copy.  The epilogue masks pairs
// outside the band and accumulates l2 in f64.
#include <cuda_runtime.h>

#include "engine.h"
#include "epilogue.cuh"

namespace ldsc {

namespace {

constexpr int TA = 128, TB = 128, BK = 16, NT = 256;
constexpr int SK = BK + 1;   // staged row stride (elements)
constexpr int NSTAGE = 3;    // K-slices in flight

// Element-sized asynchronous copy global -> shared; with valid == false the
// destination is zero-filled and nothing is read.
template <typename T>
__device__ __forceinline__ void cp_elem(T* dst, const T* src, bool valid) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int MODE>
__device__ __forceinline__ double correct(double v, int64_t k, int64_t j, const EpilogueArgs& ep) {
    if (MODE == 0) {
        return v * v * ep.n_inv_sq_r2u_a + ep.r2u_b;
    } else {
        const double kap = MODE == 2 ? __ldg(ep.kappa + k) + __ldg(ep.kappa + j) : 0.0;
        const double tilde = v * v * ep.n_inv_sq;
        const double dm3 = ep.sketch_d - 3.0 - 2.0 * kap;
        const double disc = dm3 * dm3 + 8.0 * (ep.sketch_d * tilde - 1.0);
        const double r2 = disc >= 0.0 ? (-dm3 + sqrt(disc)) * 0.25 : 0.0;
        return r2 * ep.r2u_a + ep.r2u_b;
    }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(NT, 1)
    k_gram_simt(const T* __restrict__ x, uint64_t ld, uint64_t kdim, const Tile* __restrict__ tiles,
                int64_t n_tiles, EpilogueArgs ep) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);  // [NSTAGE][TA][SK]
    T* Bs = As + NSTAGE * TA * SK;           // [NSTAGE][TB][SK]
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int64_t m = ep.m;
    const uint64_t nk = kdim / BK;

    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        const int64_t k0 = (int64_t)tl.a_blk * TA, j0 = (int64_t)tl.b_blk * TB;
        T acc[8][8];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int l = 0; l < 8; l++) acc[i][l] = T(0);

        // K-slice `it` into stage it % NSTAGE: TA x BK and TB x BK elements,
        // 8 + 8 per thread, consecutive threads along a row's K elements
        auto issue = [&](uint64_t it) {
            if (it < nk) {
                const int st = (int)(it % NSTAGE);
                const uint64_t kk = it * BK;
#pragma unroll
                for (int q = 0; q < TA * BK / NT; q++) {
                    const int e = tid + NT * q, r = e / BK, c = e % BK;
                    const bool va = k0 + r < m, vb = j0 + r < m;
                    cp_elem(As + (st * TA + r) * SK + c, va ? x + (uint64_t)(k0 + r) * ld + kk + c : x, va);
                    cp_elem(Bs + (st * TB + r) * SK + c, vb ? x + (uint64_t)(j0 + r) * ld + kk + c : x, vb);
                }
            }
            cp_commit();
        };
#pragma unroll
        for (int s0 = 0; s0 < NSTAGE - 1; s0++) issue(s0);
        for (uint64_t it = 0; it < nk; it++) {
            cp_wait<NSTAGE - 2>();
            __syncthreads();              // slice `it` landed; slice it - 1 is no longer read
            issue(it + NSTAGE - 1);       // into the stage slice it - 1 used
            const int st = (int)(it % NSTAGE);
            const T* as = As + st * TA * SK;
            const T* bs = Bs + st * TB * SK;
#pragma unroll
            for (int s = 0; s < BK; s++) {
                T a[8], b[8];
#pragma unroll
                for (int i = 0; i < 8; i++) a[i] = as[(ty + 16 * i) * SK + s];
#pragma unroll
                for (int l = 0; l < 8; l++) b[l] = bs[(tx + 16 * l) * SK + s];
#pragma unroll
                for (int i = 0; i < 8; i++)
#pragma unroll
                    for (int l = 0; l < 8; l++) acc[i][l] = fma(a[i], b[l], acc[i][l]);
            }
        }
        cp_wait<0>();
        __syncthreads();  // the epilogue reuses the staging memory

        // ---- epilogue: r^2 correction, band mask, l2 accumulation ----
        if (ep.K == 1) {
            double rsum[8], csum[8];
#pragma unroll
            for (int i = 0; i < 8; i++) rsum[i] = csum[i] = 0.0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int64_t k = k0 + ty + 16 * i;
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    const int64_t j = j0 + tx + 16 * l;
                    if (pair_in_band(k, j, m, ep.left)) {
                        const double r2u = correct<MODE>((double)acc[i][l], k, j, ep);
                        rsum[i] += r2u * __ldg(ep.aeff + j);
                        csum[l] += r2u * __ldg(ep.aeff + k);
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                double v = rsum[i];
                v += __shfl_xor_sync(0xFFFFFFFFu, v, 8);
                v += __shfl_xor_sync(0xFFFFFFFFu, v, 4);
                v += __shfl_xor_sync(0xFFFFFFFFu, v, 2);
                v += __shfl_xor_sync(0xFFFFFFFFu, v, 1);
                const int64_t k = k0 + ty + 16 * i;
                if (ep.prow) {
                    if (tx == 0) ep.prow[(size_t)t * TA + ty + 16 * i] = v;   // summed by launch_l2_reduce
                } else if (tx == 0 && k < m && v != 0.0) {
                    atomicAdd(ep.l2 + k, v);
                }
            }
            double* cpart = reinterpret_cast<double*>(smem_raw);  // [16][TB], fits the operand area
#pragma unroll
            for (int l = 0; l < 8; l++) cpart[ty * TB + tx + 16 * l] = csum[l];
            __syncthreads();
            if (tid < TB) {
                double v = 0.0;
#pragma unroll
                for (int r = 0; r < 16; r++) v += cpart[r * TB + tid];
                const int64_t j = j0 + tid;
                if (ep.pcol)
                    ep.pcol[(size_t)t * TB + tid] = v;
                else if (j < m && v != 0.0)
                    atomicAdd(ep.l2 + j, v);
            }
            __syncthreads();
        } else {
            // K > 1: the masked r2u tile goes to global memory in f64 (row k of
            // TB values) for the banded annotation contraction (contract.cu);
            // the 16 lanes of a row store 128 contiguous bytes
            double* dst = ep.rtiles + (size_t)t * TA * TB;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int64_t k = k0 + ty + 16 * i;
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    const int64_t j = j0 + tx + 16 * l;
                    double r = 0.0;
                    if (pair_in_band(k, j, m, ep.left)) r = correct<MODE>((double)acc[i][l], k, j, ep);
                    dst[(ty + 16 * i) * TB + tx + 16 * l] = r;
                }
            }
        }
    }
}

template <typename T, int MODE>
cudaError_t launch(const T* x, uint64_t ld, uint64_t kdim, const Tile* tiles, int64_t n_tiles,
                   const EpilogueArgs& ep, int sms, cudaStream_t stream) {
    if (n_tiles <= 0) return cudaSuccess;
    size_t op_bytes = sizeof(T) * NSTAGE * (TA + TB) * SK;
    size_t cpart_bytes = sizeof(double) * 16 * TB;
    size_t smem = op_bytes;
    if (cpart_bytes > smem) smem = cpart_bytes;
    cudaError_t e = cudaFuncSetAttribute(k_gram_simt<T, MODE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int64_t grid = n_tiles < (int64_t)sms * 2 ? n_tiles : (int64_t)sms * 2;
    k_gram_simt<T, MODE><<<(unsigned)grid, NT, smem, stream>>>(x, ld, kdim, tiles, n_tiles, ep);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_gram_f64(const double* x, uint64_t ld, uint64_t kdim, const Tile* tiles,
                            int64_t n_tiles, const EpilogueArgs& ep, int sms, cudaStream_t stream) {
    return launch<double, 0>(x, ld, kdim, tiles, n_tiles, ep, sms, stream);
}

cudaError_t launch_gram_f32(const float* x, uint64_t ld, uint64_t kdim, const Tile* tiles,
                            int64_t n_tiles, const EpilogueArgs& ep, int maf_aware, int sms,
                            cudaStream_t stream) {
    if (maf_aware) return launch<float, 2>(x, ld, kdim, tiles, n_tiles, ep, sms, stream);
    return launch<float, 1>(x, ld, kdim, tiles, n_tiles, ep, sms, stream);
}

cudaError_t preload_gram_simt() {
    cudaError_t e = preload_kernel(k_gram_simt<double, 0>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_simt<float, 1>);
    if (e == cudaSuccess) e = preload_kernel(k_gram_simt<float, 2>);
    return e;
}

}  // namespace ldsc
