// step_3d.cu -- the m-axis pass of the 3-D mixed-precision step (CVD on L x M x N grids).
//
// A 3-D run of the reference (src/experiment/cvd.cpp:389-454) transforms every field with
// a 3-D DFT (FFTW, n fastest).  Here the state is held as its DFT along n (Hermitian half,
// Hn = N/2 + 1 bins padded to Hp = Tn*CT), and one step is four sweeps:
//   the mixed row kernel on the L*M rows of length N (layout A, step_mixed.cu);
//   this kernel, forward: psi, con, inn, inc transformed along m, layout A -> B;
//   the mixed column kernel on the (n-tile, km) tiles of layout B: transforms along l and
//     the semi-implicit update with k^2 = kl^2 + km^2 + kn^2 (the 3-D table);
//   this kernel, inverse: psi', con', c2a, c2b (and the gradients at checkpoints), B -> A.
// Layouts (pfc_internal.h, MPassArgs): A puts each (t, l) M x CT tile in one block, B each
// (t, km) L x CT tile.  A work item is one (array, t, l): the A block is read (or the B
// chunks of CT values gathered), transformed along m in shared memory in FP64, and written
// as CT-value chunks of B (or as the contiguous A block).  The inverse is unnormalised;
// the 1/(L*M) of both l and m inverses is folded into the column kernel's factors.
#include "pfc_b200.h"
#include "step_common.cuh"

namespace pfc {

template <int M, int C> struct MPassCfg {
    static constexpr int NT = (M * C / 16) < 32 ? 32 : (M * C / 16);  // one radix-16 butterfly per thread
};

template <int M, int C, bool FWD>
__global__ void __launch_bounds__(MPassCfg<M, C>::NT) k_mpass(MPassArgs a, const double2 *__restrict__ tw) {
    constexpr int NT = MPassCfg<M, C>::NT;
    extern __shared__ double2 sd[];
    const int L = a.L, Tn = a.Tn;
    const long per_arr = (long)Tn * L, items = (long)a.narr * per_arr;
    for (long item = blockIdx.x; item < items; item += gridDim.x) {
        const int arr = (int)(item / per_arr);
        const int rem = (int)(item % per_arr);
        const int t = rem / L, l = rem % L;
        const float2 *__restrict__ src = a.src[arr];
        float2 *__restrict__ dst = a.dst[arr];
        const long blockA = ((long)t * L + l) * M * C;  // the (t, l) tile in layout A
        __syncthreads();  // the previous item's stores have read sd
        if (FWD) {
            const float4 *g = reinterpret_cast<const float4 *>(src + blockA);
            for (int i = threadIdx.x; i < M * C / 2; i += NT) {
                const float4 v = g[i];
                sd[spad(2 * i)] = make_double2(v.x, v.y);
                sd[spad(2 * i + 1)] = make_double2(v.z, v.w);
            }
        } else {
            for (int i = threadIdx.x; i < M * C; i += NT) {
                const int km = i / C, c = i % C;
                const float2 v = src[(((long)t * M + km) * L + l) * C + c];
                sd[spad(i)] = make_double2(v.x, v.y);
            }
        }
        __syncthreads();
        fft_smem<M, C, NT, FWD>(sd, tw);  // sequences c interleaved: element m of c at m*C + c
        if (FWD) {
            for (int i = threadIdx.x; i < M * C; i += NT) {
                const int km = i / C, c = i % C;
                const double2 v = sd[spad(i)];
                dst[(((long)t * M + km) * L + l) * C + c] = make_float2((float)v.x, (float)v.y);
            }
        } else {
            float4 *g = reinterpret_cast<float4 *>(dst + blockA);
            for (int i = threadIdx.x; i < M * C / 2; i += NT) {
                const double2 u = sd[spad(2 * i)], v = sd[spad(2 * i + 1)];
                g[i] = make_float4((float)u.x, (float)u.y, (float)v.x, (float)v.y);
            }
        }
    }
}

template <int M, int C>
static cudaError_t mpass_impl(const MPassArgs &a, bool fwd, const TwiddleSet &tw, cudaStream_t s) {
    constexpr int NT = MPassCfg<M, C>::NT;
    constexpr size_t smem = sizeof(double2) * padded_len<M * C>::value;
    static unsigned mask_f = 0, mask_i = 0;
    cudaError_t e = fwd ? set_smem(k_mpass<M, C, true>, smem, mask_f) : set_smem(k_mpass<M, C, false>, smem, mask_i);
    if (e != cudaSuccess) return e;
    const long items = (long)a.narr * a.Tn * a.L;
    const long cap = 8L * sm_count();
    const unsigned grid = (unsigned)(items < cap ? items : cap);
    if (fwd)
        k_mpass<M, C, true><<<grid, NT, smem, s>>>(a, tw.f64[log2i(M)]);
    else
        k_mpass<M, C, false><<<grid, NT, smem, s>>>(a, tw.f64[log2i(M)]);
    return cudaGetLastError();
}

// M * C <= 4096 complex doubles (69.6 KB of padded shared memory per CTA)
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
