// step_common.cuh -- pieces of the fused FP32 step (step_fp32.cu) that do not depend on
// its kernels: tile geometry, the C2 kernel as the reference's float table holds it,
// and launch helpers.
#pragma once

#include "fft_core.cuh"
#include "pfc_internal.h"
#include "tile_io.cuh"

namespace pfc {

constexpr int COL_TILE = 4096;  // complex elements per column-kernel tile (32 KB in FP32)

// Column-kernel tile: L rows x C packed columns, C a power of two in [1, 16] with
// 512 <= C*L <= 8192 complex elements (three such buffers per CTA: 13 KB to 204 KB).
constexpr bool col_tile_ok(int L, int C) { return C >= 1 && C <= 16 && C * L >= 512 && C * L <= 8192; }
template <int L, int C> struct ColCfg {
    static constexpr int NT = (C * L / 16) < 32 ? 32 : (C * L / 16);
    // CTAs per SM that the shared memory leaves room for (two at C*L = 4096)
    static constexpr int MINB = (8192 / (C * L)) > 8 ? 8 : ((8192 / (C * L)) < 1 ? 1 : 8192 / (C * L));
};

// C2 correlation kernel at |k| = sqrtf(ks), as the reference builds its float table
// (misfit_uniform_time_seed_fftw_early.cpp:700-750): exp in double of float arguments.
__device__ __forceinline__ float c2_ref(const C2Params &p, float ks) {
    const float s = __fsqrt_rn(ks);
    if (s <= p.kc) {
        const double d = (double)__fsub_rn(s, p.k1);
        return (float)(exp(-(double)p.q1 * (double)p.q1) * exp(-(d * d) / (double)p.gg1));
    }
    const double d = (double)__fsub_rn(s, p.k2);
    return (float)(exp(-(double)p.q2 * (double)p.q2) * exp(-(d * d) / (double)p.gg2));
}

static inline int log2i(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// Opt in to more than 48 KB of dynamic shared memory, once per kernel and device
// (the attribute call is not a stream operation, so it is also done before any
// graph capture through prepare_size()).
template <typename K> static inline cudaError_t set_smem(K kernel, size_t bytes, unsigned &mask) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (mask & (1u << dev)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) mask |= 1u << dev;
    return e;
}

template <int n> static constexpr size_t smem_bytes() { return sizeof(float2) * padded_len<n>::value; }

// Streaming multiprocessors of the current device (the persistent grid's width).
static inline int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

#define PFC_SIZE_SWITCH(n, FN, ...)             \
    switch (n) {                                \
        case 32: return FN<32>(__VA_ARGS__);    \
        case 64: return FN<64>(__VA_ARGS__);    \
        case 128: return FN<128>(__VA_ARGS__);  \
        case 256: return FN<256>(__VA_ARGS__);  \
        case 512: return FN<512>(__VA_ARGS__);  \
        case 1024: return FN<1024>(__VA_ARGS__); \
        case 2048: return FN<2048>(__VA_ARGS__); \
        default: return cudaErrorInvalidValue;  \
    }

}  // namespace pfc
