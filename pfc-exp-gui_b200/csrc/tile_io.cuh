// tile_io.cuh -- tile staging (cp.async into shared memory, float4 stores out) and the
// multipliers an inverse transform's first stage applies, used by the column kernel
// (col_kernel.cuh).
#pragma once

#include "fft_core.cuh"

namespace pfc {

// multiplier applied by an inverse transform's first stage: P * g(l, km)
struct ScaleByTable {
    const float2 *tab;  // kc2 tile (c2a, c2b)
    int C, which;       // which: 0 = .x, 1 = .y
    __device__ __forceinline__ float2 operator()(int e, int b, float2 v) const {
        const float2 t = tab[e * C + b];
        const float g = which == 0 ? t.x : t.y;
        return make_float2(v.x * g, v.y * g);
    }
};
// -i k P along l (which = 0, krefl) or m (which = 1, krefm)
struct GradientOf {
    const float *krefl, *krefm;
    int km0, H, which;
    __device__ __forceinline__ float2 operator()(int e, int b, float2 v) const {
        const int km = km0 + b;
        const float kv = which == 0 ? krefl[e] : krefm[km <= H ? km : 0];
        return make_float2(kv * v.y, -kv * v.x);
    }
};

// Asynchronous copy of one tile (L*C float2, 16-byte aligned) into the staging buffer q:
// 16 bytes per instruction, tracked per thread by a commit group.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
template <int L, int C, int NT> __device__ __forceinline__ void tile_prefetch(const float2 *__restrict__ g, float2 *q) {
    for (int i = threadIdx.x; i < L * C / 2; i += NT) cp_async16(q + 2 * i, g + 2 * i);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// this thread's copies have landed; the barrier makes every thread's visible
__device__ __forceinline__ void tile_wait() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
}
template <int L, int C, int NT> struct Prefetch {
    const float2 *src;
    float2 *q;
    __device__ __forceinline__ void operator()() const {
        if (src) tile_prefetch<L, C, NT>(src, q);
    }
};

template <int L, int C, int NT> __device__ __forceinline__ void tile_out(const float2 *sm, float2 *__restrict__ g) {
    float4 *g4 = reinterpret_cast<float4 *>(g);
    for (int i = threadIdx.x; i < L * C / 2; i += NT) {
        const float2 a = sm[spad(2 * i)], b = sm[spad(2 * i + 1)];
        g4[i] = make_float4(a.x, a.y, b.x, b.y);
    }
}

}  // namespace pfc
