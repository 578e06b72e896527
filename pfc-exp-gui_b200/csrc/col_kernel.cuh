// col_kernel.cuh -- the column kernel of the fused FP32 step, and its launchers.
//
// Instantiated one row length L per translation unit (col_inst.cu compiled with
// PFC_COL_L = L); step_fp32.cu reaches it through launch_col_f32_L<L>.
#pragma once

#include "step_common.cuh"

namespace pfc {

// Work item: a tile of L rows x C packed columns of one run (a contiguous block of
// the row-space layout).  CTAs are persistent and take items in turn.  For phi and
// then con:
//   the field's tile is transformed forward into the parked buffer P,
//   its nonlinear term's tile is transformed forward in place in the scratch s,
//   the semi-implicit update runs in place in P (MAINEQUATIONC2_NOI / C2MIX,
//     MIS:983-1014, CVD:865-886) with the FP64-built factors of the shared
//     coefficient table (and the noise term when axx > 0),
//   each output is an inverse transform whose first stage reads P through a
//     multiplier (1, C2A, C2B for phi, MIS:807-810; 1 and the -i k gradients for
//     con at checkpoints, MIS:884-889) into s, copied s -> HBM (float4).
// Inputs are staged into an unpadded buffer Q, which a transform's first stage reads
// directly, by 16-byte cp.async copies (STAGE_ASYNC) or by one TMA bulk copy per tile
// completing on a shared-memory mbarrier (STAGE_BULK; waits bounded in time, a CTA
// whose copy does not arrive sets the context's fault word and returns); the
// autotuner picks the method with the width.  Each load is issued as soon as the
// previous transform's first stage has consumed Q, so it streams in while that
// transform, the update and the output transforms run; the next item's phi tile
// streams in during the current item's con work.  Two CTAs of 256 threads
// per SM at C*L = 4096 (2 x 100 KB of shared memory, 128 registers); the tile width C
// of a grid is chosen per device by the autotuner (engine.cu).

// Tile staging (Stager, Prefetch, tile_out) and the
// ScaleByTable / GradientOf multipliers come from tile_io.cuh.

// noise_mode (the spectrum of the noise field of step t) comes from step_common.cuh.

template <int L, int C, int MODE, int STAGE>
__global__ void __launch_bounds__(ColCfg<L, C>::NT, ColCfg<L, C>::MINB)
    k_col_step(const RunDesc *__restrict__ runs, int nruns, const float2 *__restrict__ tw, int *fault) {
    constexpr int NT = ColCfg<L, C>::NT;
    constexpr int SPAD = padded_len<C * L>::value;
    typedef RegOut<L, C, NT> RO;  // register scratch the transforms need for their last stage
    extern __shared__ __align__(16) float2 smem[];
    __shared__ __align__(8) unsigned long long stage_bar;  // completion barrier of the tile copies
    float2 *s = smem;               // FFT scratch
    float2 *Pk = smem + SPAD;       // parked spectrum
    float2 *Q = smem + 2 * SPAD;    // staging buffer (16-byte aligned: 2*SPAD float2)
    const int T = runs[0].T;        // all runs of a launch share L and M
    const int items = nruns * T;
    float2 b[RO::PER_T][RO::R];
    int item = blockIdx.x;
    if (item >= items) return;
    typedef Stager<L, C, NT, STAGE> ST;
    const ST st{smem_u32(&stage_bar), Q};
    st.init();
    auto tile_of = [&](int it) { return (long)(it % T) * L * C; };
    st.issue(runs[item / T].psi + tile_of(item));
    for (; item < items; item += gridDim.x) {
        const RunDesc &d = runs[item / T];
        const int H = d.M / 2;
        const long tile = tile_of(item);
        const int km0 = (item % T) * C;
        const int next = item + gridDim.x;
        const float2 *next_psi = next < items ? runs[next / T].psi + tile_of(next) : nullptr;
        const float invL = 1.0f / (float)L;
        // barrier phase of this item's first wait: an item of the step modes waits four
        // times (phases 0, 1, 0, 1), a COL_PREPARE item once (the iteration's parity)
        const unsigned p0 = MODE == COL_PREPARE ? (unsigned)((item - (int)blockIdx.x) / (int)gridDim.x) & 1u : 0u;
        const float mn_dt = d.k.dynamic_mn * d.dt, mc_dt = d.k.dynamic_mc * d.dt;

        // ---- phi ----
        if (!st.wait(p0, fault)) return;
        if (MODE == COL_PREPARE) {
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, next_psi});
        } else {
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, d.inn + tile});
            if (!st.wait(1u, fault)) return;
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, s, tw, b, Identity(), Prefetch<ST>{st, d.con + tile});
        }
        const int nstep = (MODE != COL_PREPARE && d.noise_amp != 0.0f) ? *d.step_ctr : -1;
        for (int e = threadIdx.x; e < L * C; e += NT) {
            const int l = e / C, c = e % C, km = km0 + c;
            const int pi = spad(e);
            float2 v = Pk[pi];
            if (MODE != COL_PREPARE) {
                // (psi^ - Mn dt k^2 N^ [+ dt b0 xi^ |k| lowpass]) / (1 + Mn dt k^2) / L; the
                // FP64-built factor is 0 at k = 0
                const float kl = d.krefl[l], kmv = d.krefm[km <= H ? km : 0];
                const float ks = kl * kl + kmv * kmv;
                const float an = mn_dt * ks;
                const float2 nh = s[pi];
                const float f = d.kden[tile + e].x;
                float rx = v.x - an * nh.x, ry = v.y - an * nh.y;
                if (nstep >= 0 && km <= H) {
                    // MAINEQUATIONC2_NOI's noise term (MIS:1002-1003), lowpass at |k| = 2 pi
                    const float2 xi = noise_mode(d.noise_key, nstep, l, km, L, d.M);
                    const float sk = sqrtf(ks);
                    const float w = d.noise_amp * sk * (0.5f - 0.5f * tanhf((sk - 6.2831852f) / 0.1f));
                    rx += w * xi.x;
                    ry += w * xi.y;
                }
                v = make_float2(rx * f, ry * f);
            } else {
                v = (l == 0 && km == 0) ? make_float2(0.f, 0.f) : cscale(v, invL);
            }
            Pk[pi] = v;
        }
        __syncthreads();
        if (MODE != COL_PREPARE) {
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b);
            tile_out<L, C, NT>(s, d.psi + tile);
        }
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, ScaleByTable{d.kc2 + tile, C, 0});
        tile_out<L, C, NT>(s, d.ca + tile);
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, ScaleByTable{d.kc2 + tile, C, 1});
        tile_out<L, C, NT>(s, d.cb + tile);
        if (MODE == COL_PREPARE) continue;

        // ---- con ----
        if (!st.wait(0u, fault)) return;
        fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, d.inc + tile});
        if (!st.wait(1u, fault)) return;
        fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, s, tw, b, Identity(), Prefetch<ST>{st, next_psi});
        for (int e = threadIdx.x; e < L * C; e += NT) {
            const int l = e / C, c = e % C, km = km0 + c;
            const int pi = spad(e);
            // (c^ - Mc dt k^2 I^) / (1 + Mc dt alpha k^4) / L; the FP64-built factor is 0 at k = 0
            const float kl = d.krefl[l], kmv = d.krefm[km <= H ? km : 0];
            const float ac = mc_dt * (kl * kl + kmv * kmv);
            const float f = d.kden[tile + e].y;
            const float2 ih = s[pi];
            const float2 v = Pk[pi];
            Pk[pi] = make_float2((v.x - ac * ih.x) * f, (v.y - ac * ih.y) * f);
        }
        __syncthreads();
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b);
        tile_out<L, C, NT>(s, d.con + tile);
        if (MODE == COL_STEP_CHECKPOINT) {
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, GradientOf{d.krefl, d.krefm, km0, H, 0});
            tile_out<L, C, NT>(s, d.gx + tile);
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, GradientOf{d.krefl, d.krefm, km0, H, 1});
            tile_out<L, C, NT>(s, d.gy + tile);
        }
    }
    st.finish();  // every copy issued has been waited for: the last item issues none (next_psi = null)
}

template <int L, int C, int MODE, int STAGE>
static cudaError_t col_impl(const RunDesc *d_runs, int nruns, int M, const TwiddleSet &tw, cudaStream_t st) {
    constexpr int NT = ColCfg<L, C>::NT;
    constexpr size_t smem = 2 * smem_bytes<C * L>() + sizeof(float2) * C * L;  // s, P (padded) and Q
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_col_step<L, C, MODE, STAGE>, smem, mask);
    if (nruns == 0) return e;
    if (e != cudaSuccess) return e;
    const int H = M / 2;
    const int items = ((H + 1 + C - 1) / C) * nruns;
    const int cap = ColCfg<L, C>::MINB * sm_count();
    const int grid = items < cap ? items : cap;
    k_col_step<L, C, MODE, STAGE><<<grid, NT, smem, st>>>(d_runs, nruns, tw.f32[log2i(L)], tw.fault);
    return cudaGetLastError();
}

template <int L, int C, int STAGE>
static cudaError_t col_modes(const RunDesc *d_runs, int nruns, int M, int mode, const TwiddleSet &tw,
                             cudaStream_t s) {
    switch (mode) {
        case COL_STEP: return col_impl<L, C, COL_STEP, STAGE>(d_runs, nruns, M, tw, s);
        case COL_PREPARE: return col_impl<L, C, COL_PREPARE, STAGE>(d_runs, nruns, M, tw, s);
        case COL_STEP_CHECKPOINT: return col_impl<L, C, COL_STEP_CHECKPOINT, STAGE>(d_runs, nruns, M, tw, s);
        default: return cudaErrorInvalidValue;
    }
}
template <int L, int C>
static cudaError_t col_stages(const RunDesc *d_runs, int nruns, int M, int stage, int mode, const TwiddleSet &tw,
                              cudaStream_t s) {
    switch (stage) {
        case STAGE_ASYNC: return col_modes<L, C, STAGE_ASYNC>(d_runs, nruns, M, mode, tw, s);
        case STAGE_BULK: return col_modes<L, C, STAGE_BULK>(d_runs, nruns, M, mode, tw, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int L>
static cudaError_t col_dispatch(const RunDesc *d_runs, int nruns, int M, int C, int stage, int mode,
                                const TwiddleSet &tw, cudaStream_t s) {
    switch (C) {
        case 1:
            if constexpr (col_tile_ok(L, 1)) return col_stages<L, 1>(d_runs, nruns, M, stage, mode, tw, s);
            break;
        case 2:
            if constexpr (col_tile_ok(L, 2)) return col_stages<L, 2>(d_runs, nruns, M, stage, mode, tw, s);
            break;
        case 4:
            if constexpr (col_tile_ok(L, 4)) return col_stages<L, 4>(d_runs, nruns, M, stage, mode, tw, s);
            break;
        case 8:
            if constexpr (col_tile_ok(L, 8)) return col_stages<L, 8>(d_runs, nruns, M, stage, mode, tw, s);
            break;
        case 16:
            if constexpr (col_tile_ok(L, 16)) return col_stages<L, 16>(d_runs, nruns, M, stage, mode, tw, s);
            break;
        default: break;
    }
    return cudaErrorInvalidValue;
}

template <int L>
cudaError_t launch_col_f32_L(const RunDesc *d_runs, int nruns, int M, int C, int stage, int mode,
                             const TwiddleSet &tw, cudaStream_t s) {
    return col_dispatch<L>(d_runs, nruns, M, C, stage, mode, tw, s);
}

}  // namespace pfc
