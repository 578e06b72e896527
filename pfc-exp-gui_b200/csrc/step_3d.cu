// step_3d.cu -- the m-axis pass of the 3-D mixed-precision step (CVD on L x M x N grids).
//
// A 3-D run of the reference (src/experiment/cvd.cpp:389-454) transforms every field with
// a 3-D DFT (FFTW, n fastest).  Here the state is held as its DFT along n (Hermitian half,
// Hn = N/2 + 1 bins padded to Hp = Tn*CT), and one step is four sweeps:
//   the mixed row kernel on the L*M rows of length N (layout A, step_mixed.cu);
//   this kernel, forward: psi, con, inn, inc transformed along m, layout A -> B;
//   the mixed column kernel on the (n-tile, km) tiles of layout B: transforms along l and
//     the semi-implicit update with k^2 = kl^2 + km^2 + kn^2 (the 3-D table);
//   this kernel, inverse: psi', con', c2a, c2b, B -> A (at checkpoints too: the column
//     kernel sums the energy's gradient term in k-space).
// Layouts (pfc_internal.h, MPassArgs): A puts each (t, l) M x CT tile in one block, B each
// (t, km) L x CT tile.  A work item is one (array, t, l): the A block is copied (or the B
// chunks of CT values gathered) by cp.async into an FP32 staging buffer, transformed along
// m in FP64 (the first stage reads the staging buffer, shared memory holds the rest), and
// written as CT-value chunks of B (or as the contiguous A block); the next item's copies
// run behind the current transform.  The inverse is unnormalised; the 1/(L*M) of both l
// and m inverses is folded into the column kernel's factors.
#include "pfc_b200.h"
#include "step_common.cuh"

namespace pfc {

template <int M, int C> struct MPassCfg {
    static constexpr int NT = (M * C / 16) < 32 ? 32 : (M * C / 16);  // one radix-16 butterfly per thread
    // padded double2 transform buffer + the unpadded FP32 staging buffer
    static constexpr int SMEM = (int)sizeof(double2) * padded_len<M * C>::value + (int)sizeof(float2) * M * C;
    static constexpr int FIT = (228 * 1024) / (SMEM + 1024);  // CTAs per SM the shared memory leaves room for
    static constexpr int MINB = FIT > 4 ? 4 : (FIT < 1 ? 1 : FIT);
};

__device__ __forceinline__ void mpass_cp8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// All threads: start the copies of item `item` into the staging buffer q, one commit
// group.  Forward: the A block, contiguous.  Inverse: the item's CT-value chunk of every
// km of layout B.  Element m of sequence c lands at m*C + c, the transform's input order.
template <int M, int C, int NT, bool FWD>
__device__ __forceinline__ void mpass_issue(const MPassArgs &a, long item, float2 *q) {
    const long per_arr = (long)a.Tn * a.L;
    const int arr = (int)(item / per_arr);
    const int rem = (int)(item % per_arr);
    const int t = rem / a.L, l = rem % a.L;
    const float2 *src = a.src[arr];
    if (FWD) {
        const float2 *g = src + ((long)t * a.L + l) * M * C;
        for (int i = threadIdx.x; i < M * C / 2; i += NT) cp_async16(q + 2 * i, g + 2 * i);
    } else if (C >= 2) {  // 16-byte pieces within a chunk (C is even)
        for (int i = threadIdx.x; i < M * C / 2; i += NT) {
            const int e = 2 * i, km = e / C, c = e % C;
            cp_async16(q + e, src + (((long)t * M + km) * a.L + l) * C + c);
        }
    } else {
        for (int i = threadIdx.x; i < M; i += NT) mpass_cp8(q + i, src + ((long)t * M + i) * a.L + l);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// a transform's hook: start the next item's copies once the first stage has read q
template <int M, int C, int NT, bool FWD> struct MPassPrefetch {
    const MPassArgs *a;
    long next, items;
    float2 *q;
    __device__ __forceinline__ void operator()() const {
        if (next < items) mpass_issue<M, C, NT, FWD>(*a, next, q);
    }
};

// Persistent over items (array, t, l): the item's input is staged (FP32) by cp.async into
// q, which the transform's first stage reads directly; the next item's copies are issued
// as soon as that stage has read q, so they stream in while the transform and the
// output stores of this item run.
template <int M, int C, bool FWD>
__global__ void __launch_bounds__(MPassCfg<M, C>::NT, MPassCfg<M, C>::MINB)
    k_mpass(MPassArgs a, const double2 *__restrict__ tw) {
    constexpr int NT = MPassCfg<M, C>::NT;
    typedef RegOut<M, C, NT, double2> RO;
    extern __shared__ __align__(16) double2 sd[];
    float2 *q = reinterpret_cast<float2 *>(sd + padded_len<M * C>::value);  // 16-byte aligned
    const int L = a.L;
    const long per_arr = (long)a.Tn * L, items = (long)a.narr * per_arr;
    long item = blockIdx.x;
    if (item >= items) return;
    double2 last[RO::PER_T][RO::R];
    mpass_issue<M, C, NT, FWD>(a, item, q);
    for (; item < items; item += gridDim.x) {
        const int arr = (int)(item / per_arr);
        const int rem = (int)(item % per_arr);
        const int t = rem / L, l = rem % L;
        float2 *__restrict__ dst = a.dst[arr];
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();  // every thread's copies have landed; the previous item's stores have read sd
        // sequences c interleaved: element m of c at m*C + c
        fft<M, C, NT, FWD, SP_GLOBAL, SP_SMEM>(q, sd, sd, tw, last, Identity(),
                                               MPassPrefetch<M, C, NT, FWD>{&a, item + gridDim.x, items, q});
        if (FWD) {
            for (int i = threadIdx.x; i < M * C; i += NT) {
                const int km = i / C, c = i % C;
                const double2 v = sd[spad(i)];
                dst[(((long)t * M + km) * L + l) * C + c] = make_float2((float)v.x, (float)v.y);
            }
        } else {
            float4 *g = reinterpret_cast<float4 *>(dst + ((long)t * L + l) * M * C);
            for (int i = threadIdx.x; i < M * C / 2; i += NT) {
                const double2 u = sd[spad(2 * i)], v = sd[spad(2 * i + 1)];
                g[i] = make_float4((float)u.x, (float)u.y, (float)v.x, (float)v.y);
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // the last item issues no copy
}

template <int M, int C>
static cudaError_t mpass_impl(const MPassArgs &a, bool fwd, const TwiddleSet &tw, cudaStream_t s) {
    constexpr int NT = MPassCfg<M, C>::NT;
    constexpr size_t smem = MPassCfg<M, C>::SMEM;
    static unsigned mask_f = 0, mask_i = 0;
    cudaError_t e = fwd ? set_smem(k_mpass<M, C, true>, smem, mask_f) : set_smem(k_mpass<M, C, false>, smem, mask_i);
    if (e != cudaSuccess) return e;
    const long items = (long)a.narr * a.Tn * a.L;
    const long cap = (long)MPassCfg<M, C>::MINB * sm_count();
    const unsigned grid = (unsigned)(items < cap ? items : cap);
    if (fwd)
        k_mpass<M, C, true><<<grid, NT, smem, s>>>(a, tw.f64[log2i(M)]);
    else
        k_mpass<M, C, false><<<grid, NT, smem, s>>>(a, tw.f64[log2i(M)]);
    return cudaGetLastError();
}

// M * C <= 4096 complex doubles (101.6 KB of shared memory per CTA with the staging buffer)
template <int M>
static cudaError_t mpass_width(const MPassArgs &a, bool fwd, const TwiddleSet &tw, cudaStream_t s) {
    switch (a.CT) {
        case 1: return mpass_impl<M, 1>(a, fwd, tw, s);
        case 2: return mpass_impl<M, 2>(a, fwd, tw, s);
        case 4:
            if constexpr (M * 4 <= 4096) return mpass_impl<M, 4>(a, fwd, tw, s);
            break;
        case 8:
            if constexpr (M * 8 <= 4096) return mpass_impl<M, 8>(a, fwd, tw, s);
            break;
        case 16:
            if constexpr (M * 16 <= 4096) return mpass_impl<M, 16>(a, fwd, tw, s);
            break;
        default: break;
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_mpass(const MPassArgs &a, bool forward, const TwiddleSet &tw, cudaStream_t s) {
    if (a.narr < 1 || a.narr > 8 || a.L < 1 || a.Tn < 1) return cudaErrorInvalidValue;
    PFC_SIZE_SWITCH(a.M, mpass_width, a, forward, tw, s)
}

}  // namespace pfc
