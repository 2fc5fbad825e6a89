// gram_simt.cu -- band Gram on CUDA cores for the two non-integer forms:
//   * FP64 plain form: standardised f64 columns, val = x_k . x_j, and the
//     reference's fused unbiased-r^2 transform val^2 * r2u_a / N^2 + r2u_b
//     (src/l2/compute.rs:1067-1077, 2229-2235);
//   * FP32 CountSketch form: sketched, renormalised f32 rows, val = s_k . s_j,
//     then the quadratic bias inversion (+ MAF-aware shift) in f64
//     (src/l2/compute.rs:947-998).
// Tiles are 128 x 128 records, 256 threads, 8 x 8 outputs per thread, K-slices
// of 16 double-buffered through shared memory (rows padded by one element so
// the transposed staging stores do not share banks).  The epilogue masks pairs
// outside the band and accumulates l2 in f64.
#include <cuda_runtime.h>

#include "engine.h"
#include "epilogue.cuh"

namespace ldsc {

namespace {

constexpr int TA = 128, TB = 128, BK = 16, NT = 256;
constexpr int STA = TA + 1, STB = TB + 1;  // staged row strides
constexpr int RLD = TB + 1;  // padded row stride of the staged R tile

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

template <typename T>
struct Vec4;
template <>
struct Vec4<double> {
    static __device__ __forceinline__ void load(const double* p, double (&r)[4]) {
        const double2 a = *reinterpret_cast<const double2*>(p);
        const double2 b = *reinterpret_cast<const double2*>(p + 2);
        r[0] = a.x; r[1] = a.y; r[2] = b.x; r[3] = b.y;
    }
};
template <>
struct Vec4<float> {
    static __device__ __forceinline__ void load(const float* p, float (&r)[4]) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    }
};

template <typename T, int MODE>
__global__ void __launch_bounds__(NT, 1)
    k_gram_simt(const T* __restrict__ x, uint64_t ld, uint64_t kdim, const Tile* __restrict__ tiles,
                int64_t n_tiles, EpilogueArgs ep) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);  // [2][BK][STA]
    T* Bs = As + 2 * BK * STA;               // [2][BK][STB]
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int lrow = tid >> 1, lcol = (tid & 1) * (BK / 2);
    const int64_t m = ep.m;

    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        const int64_t k0 = (int64_t)tl.a_blk * TA, j0 = (int64_t)tl.b_blk * TB;
        const T* arow = (k0 + lrow < m) ? x + (uint64_t)(k0 + lrow) * ld : nullptr;
        const T* brow = (j0 + lrow < m) ? x + (uint64_t)(j0 + lrow) * ld : nullptr;
        T acc[8][8];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int l = 0; l < 8; l++) acc[i][l] = T(0);

        T ra[BK / 2], rb[BK / 2];
        auto gload = [&](uint64_t kk) {
#pragma unroll
            for (int h = 0; h < BK / 8; h++) {
                T* pa = ra + 4 * h;
                T* pb = rb + 4 * h;
                if (arow) Vec4<T>::load(arow + kk + lcol + 4 * h, *reinterpret_cast<T(*)[4]>(pa));
                else pa[0] = pa[1] = pa[2] = pa[3] = T(0);
                if (brow) Vec4<T>::load(brow + kk + lcol + 4 * h, *reinterpret_cast<T(*)[4]>(pb));
                else pb[0] = pb[1] = pb[2] = pb[3] = T(0);
            }
        };
        auto sstore = [&](int buf) {
#pragma unroll
            for (int q = 0; q < BK / 2; q++) {
                As[(buf * BK + lcol + q) * STA + lrow] = ra[q];
                Bs[(buf * BK + lcol + q) * STB + lrow] = rb[q];
            }
        };
        gload(0);
        sstore(0);
        __syncthreads();
        int buf = 0;
        for (uint64_t kk = 0; kk < kdim; kk += BK) {
            const bool more = kk + BK < kdim;
            if (more) gload(kk + BK);
#pragma unroll
            for (int s = 0; s < BK; s++) {
                T a[8], b[8];
#pragma unroll
                for (int i = 0; i < 8; i++) a[i] = As[(buf * BK + s) * STA + ty + 16 * i];
#pragma unroll
                for (int l = 0; l < 8; l++) b[l] = Bs[(buf * BK + s) * STB + tx + 16 * l];
#pragma unroll
                for (int i = 0; i < 8; i++)
#pragma unroll
                    for (int l = 0; l < 8; l++) acc[i][l] = fma(a[i], b[l], acc[i][l]);
            }
            if (more) sstore(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }

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
                if (tx == 0 && k < m && v != 0.0) atomicAdd(ep.l2 + k, v);
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
                if (j < m && v != 0.0) atomicAdd(ep.l2 + j, v);
            }
            __syncthreads();
        } else {
            float* Rs = reinterpret_cast<float*>(smem_raw);  // [TA][RLD]
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int64_t k = k0 + ty + 16 * i;
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    const int64_t j = j0 + tx + 16 * l;
                    float r = 0.f;
                    if (pair_in_band(k, j, m, ep.left))
                        r = (float)correct<MODE>((double)acc[i][l], k, j, ep);
                    Rs[(ty + 16 * i) * RLD + tx + 16 * l] = r;
                }
            }
            __syncthreads();
            // K > 1: the masked r2u tile goes to global memory for the banded
            // annotation contraction (contract.cu)
            float4* dst = reinterpret_cast<float4*>(ep.rtiles + (size_t)t * TA * TB);
            for (int q = tid; q < TA * TB / 4; q += NT) {
                const int e = q * 4, rr = e / TB, cc = e % TB;
                dst[q] = make_float4(Rs[rr * RLD + cc], Rs[rr * RLD + cc + 1], Rs[rr * RLD + cc + 2],
                                     Rs[rr * RLD + cc + 3]);
            }
            __syncthreads();
        }
    }
}

template <typename T, int MODE>
cudaError_t launch(const T* x, uint64_t ld, uint64_t kdim, const Tile* tiles, int64_t n_tiles,
                   const EpilogueArgs& ep, int sms, cudaStream_t stream) {
    if (n_tiles <= 0) return cudaSuccess;
    size_t op_bytes = sizeof(T) * 2 * BK * (STA + STB);
    size_t cpart_bytes = sizeof(double) * 16 * TB;
    size_t r_bytes = ep.K > 1 ? sizeof(float) * TA * RLD : 0;
    size_t smem = op_bytes;
    if (cpart_bytes > smem) smem = cpart_bytes;
    if (r_bytes > smem) smem = r_bytes;
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

}  // namespace ldsc
