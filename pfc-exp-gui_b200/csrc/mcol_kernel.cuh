// mcol_kernel.cuh -- the column kernel of the mixed-precision fused step (FP32 tiles in
// HBM, FP64 arithmetic), and its launchers.
//
// Instantiated one row length L per translation unit (col_inst.cu compiled with
// PFC_COL_L = L); step_mixed.cu reaches it through launch_col_mixed_L<L>, whose `tiles`
// is the number of column tiles per run (T of the runs' descriptors).
#pragma once

#include "step_common.cuh"

namespace pfc {

// Column tile of the mixed path (mcol_tile_ok, step_common.cuh): two padded double2
// buffers, an FP32 staging buffer and a coefficient plane slot, 47 KB to 205 KB.
template <int L, int C> struct MColCfg {
    static constexpr int NT = (C * L / 16) < 32 ? 32 : (C * L / 16);  // one radix-16 butterfly per thread
    static_assert(NT % C == 0, "a thread's elements share one tile column");
    static constexpr int SMEM = 2 * (int)sizeof(double2) * padded_len<C * L>::value + (int)sizeof(float2) * C * L +
                                (int)sizeof(double) * C * L;
    static constexpr int FIT = (228 * 1024) / (SMEM + 1024);  // CTAs per SM the shared memory leaves room for
    static constexpr int MINB = FIT > 8 ? 8 : (FIT < 1 ? 1 : FIT);
};

__device__ __forceinline__ double2 wide(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ float2 narrow(double2 v) { return make_float2((float)v.x, (float)v.y); }

// ---------------------------------------------------------------------------
// Column kernel.
// ---------------------------------------------------------------------------
// multiplier of an inverse transform's first stage: P * C2A or C2B (one plane of the table)
struct ScaleByTableD {
    const double *tab;
    int C;
    __device__ __forceinline__ double2 operator()(int e, int b, double2 v) const {
        const double g = tab[e * C + b];
        return make_double2(v.x * g, v.y * g);
    }
};
// The column part of k^2 for tile column b: km^2 of column km0 + b (2-D; 0 past M/2, the
// padding), or km^2 + kn^2 of a 3-D column view's tile (km = km3, kn = kn0 + b, 0 past N/2).
__device__ __forceinline__ double col_k2(const RunDesc &d, int b, int km0, int km3, int kn0) {
    if (km3 < 0) {
        const int km = km0 + b;
        const double k = km <= d.M / 2 ? d.kdm[km] : 0.0;
        return k * k;
    }
    const int kn = kn0 + b;
    const double km = d.kdm[km3], kz = kn <= d.N / 2 ? d.kdn[kn] : 0.0;
    return km * km + kz * kz;
}
// padded shared double2 tile -> FP32 tile in HBM (16-byte stores)
template <int L, int C, int NT> __device__ __forceinline__ void tile_out_d(const double2 *sm, float2 *__restrict__ g) {
    float4 *g4 = reinterpret_cast<float4 *>(g);
    for (int i = threadIdx.x; i < L * C / 2; i += NT) {
        const double2 a = sm[spad(2 * i)], b = sm[spad(2 * i + 1)];
        g4[i] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
    }
}

// Work item = (tile, run), tile-major: item i is tile i / nruns of run i % nruns.  CTA j
// takes items [j*per, (j+1)*per).  Per item, as the FP32 column kernel: for phi and then
// con, the field's tile is transformed forward into the parked buffer P, the nonlinear
// term's tile forward into s, the update runs in P, and each output is an inverse
// transform whose first stage reads P through a multiplier.  Inputs are staged (FP32)
// into Q by cp.async or one TMA bulk copy per tile, each issued as soon as the previous
// transform's first stage has read Q.  The coefficient planes the item reads (fn, C2A,
// C2B, fc; C2A and C2B only in the set-up mode) pass through the shared slot Tt, one TMA
// bulk copy each on a second barrier, each issued once the previous plane's last reader
// has passed a barrier, so that a transform's time covers the copy.  Waits are bounded: a
// CTA whose copy does not arrive sets the context's fault word, gives the copies still in
// flight a last bounded wait, and returns.
template <int L, int C, int MODE, int STAGE>
__global__ void __launch_bounds__(MColCfg<L, C>::NT, MColCfg<L, C>::MINB)
    k_mcol_step(const RunDesc *__restrict__ runs, int nruns, int per, const double2 *__restrict__ tw, int *fault) {
    constexpr int NT = MColCfg<L, C>::NT;
    constexpr int SPAD = padded_len<C * L>::value;
    typedef RegOut<L, C, NT, double2> RO;
    extern __shared__ __align__(16) double2 smd[];
    __shared__ __align__(8) unsigned long long stage_bar, table_bar;
    double2 *s = smd;                                                  // FFT scratch
    double2 *Pk = smd + SPAD;                                          // parked spectrum
    float2 *Q = reinterpret_cast<float2 *>(smd + 2 * SPAD);           // FP32 staging buffer (16-byte aligned)
    double *Tt = reinterpret_cast<double *>(Q + L * C);                // coefficient plane slot (16-byte aligned)
    const int T = runs[0].T;                                           // all runs of a launch share L, M and CT
    const int items = nruns * T;
    const int first = blockIdx.x * per;
    const int end = first + per < items ? first + per : items;
    if (first >= end) return;
    double2 b[RO::PER_T][RO::R];
    typedef Stager<L, C, NT, STAGE> ST;
    const ST st{smem_u32(&stage_bar), Q, true, smem_u32(&table_bar)};
    const TableStager ts{smem_u32(&table_bar), Tt, (unsigned)(L * C * sizeof(double)), smem_u32(&stage_bar),
                         STAGE == STAGE_BULK};
    st.init();
    ts.init();
    auto run_of = [&](int it) { return it % nruns; };
    auto tile_of = [&](int it) { return (long)(it / nruns) * L * C; };
    // a table wait that gave up: cp.async input copies in flight land before the return
    auto table_failed = [&]() { st.finish(); };
    // k_l of row l in a run of spacing dkl (its kdl table's entry, formed without a load)
    auto kl_of = [](int l, double dkl) { return (double)(l <= L / 2 ? l : l - L) * dkl; };
    st.issue(runs[run_of(first)].psi + tile_of(first));
    ts.issue(MODE == COL_PREPARE ? runs[run_of(first)].kc2a + tile_of(first) : runs[run_of(first)].kfn + tile_of(first));
    for (int item = first; item < end; ++item) {
        const RunDesc &d = runs[run_of(item)];
        const int H = d.M / 2;
        const long tile = tile_of(item);
        const int tile_i = item / nruns;
        const int km0 = tile_i * C;                      // 2-D: first column's km
        const int km3 = d.col3d ? tile_i % d.M : -1;     // 3-D column view: the tile's km
        // this thread's column (NT is a multiple of C: the same b for all its elements)
        const double kb2 = MODE == COL_PREPARE ? 0.0 : col_k2(d, threadIdx.x % C, km0, km3, (tile_i / d.M) * C);
        const double dkl = d.dkl;
        const bool more = item + 1 < end;
        const RunDesc *dn = more ? &runs[run_of(item + 1)] : nullptr;
        const float2 *next_psi = more ? dn->psi + tile_of(item + 1) : nullptr;
        // barrier phases: an item of the step modes waits four times on each barrier
        // (phases 0, 1, 0, 1); a COL_PREPARE item once on the input barrier (the
        // iteration's parity) and twice on the table barrier (0, 1)
        const unsigned p0 = MODE == COL_PREPARE ? (unsigned)(item - first) & 1u : 0u;

        // ---- phi ----
        if (!st.wait(p0, fault)) return;
        if (MODE == COL_PREPARE) {
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, next_psi});
        } else {
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, d.inn + tile});
            if (!st.wait(1u, fault)) return;
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, s, tw, b, Identity(), Prefetch<ST>{st, d.con + tile});
            if (!ts.wait(0u, fault)) return table_failed();  // fn
        }
        const int nstep = (MODE != COL_PREPARE && d.noise_amp != 0.0f) ? *d.step_ctr : -1;
        for (int e = threadIdx.x; e < L * C; e += NT) {
            const int pi = spad(e);
            double2 v = Pk[pi];
            if (MODE != COL_PREPARE) {
                // (psi^ - Mn dt k^2 N^ [+ dt b0 xi^ |k| lowpass]) / (1 + Mn dt k^2) / L as
                // fn/L * (psi^ - an N^), an = Mn dt k^2; fn is 0 at k = 0 and past M/2
                const double fn = Tt[e];
                const int l = e / C, km = km0 + e % C;
                const double kl = kl_of(l, dkl);
                const double ks = fma(kl, kl, kb2), an = d.mn_dt * ks;
                const double2 nh = s[pi];
                double rx = fn * (v.x - an * nh.x), ry = fn * (v.y - an * nh.y);
                if (nstep >= 0 && km <= H) {
                    // MAINEQUATIONC2_NOI's noise term (MIS:1002-1003), lowpass at |k| = 2 pi
                    const float2 xi = noise_mode(d.noise_key, nstep, l, km, L, d.M);
                    const double sk = sqrt(ks);
                    const double wn = d.noise_amp_d * sk * (0.5 - 0.5 * tanh((sk - 2.0 * 3.1415926) / 0.1)) * fn;
                    rx += wn * (double)xi.x;
                    ry += wn * (double)xi.y;
                }
                v = make_double2(rx, ry);
            } else {
                // k = 0 is row 0 of column 0 of tile 0, in 2-D and in the 3-D column view
                const bool k0 = e / C == 0 && tile_i == 0 && e % C == 0;
                v = k0 ? make_double2(0.0, 0.0) : cscale(v, d.col_scale);
            }
            Pk[pi] = v;
        }
        __syncthreads();
        if (MODE != COL_PREPARE) {
            ts.issue(d.kc2a + tile);  // every thread has read fn
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b);
            tile_out_d<L, C, NT>(s, d.psi + tile);
        }
        if (!ts.wait(MODE == COL_PREPARE ? 0u : 1u, fault)) return table_failed();  // C2A
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, ScaleByTableD{Tt, C}, TableFetch{ts, d.kc2b + tile});
        tile_out_d<L, C, NT>(s, d.ca + tile);
        if (!ts.wait(MODE == COL_PREPARE ? 1u : 0u, fault)) return table_failed();  // C2B
        const double *after_c2b = MODE == COL_PREPARE ? (more ? dn->kc2a + tile_of(item + 1) : nullptr) : d.kfc + tile;
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, ScaleByTableD{Tt, C}, TableFetch{ts, after_c2b});
        tile_out_d<L, C, NT>(s, d.cb + tile);
        if (MODE == COL_PREPARE) continue;

        // ---- con ----
        if (!st.wait(0u, fault)) return;
        fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, d.inc + tile});
        if (!st.wait(1u, fault)) return;
        fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, s, tw, b, Identity(), Prefetch<ST>{st, next_psi});
        if (!ts.wait(1u, fault)) return table_failed();  // fc
        for (int e = threadIdx.x; e < L * C; e += NT) {
            const int pi = spad(e);
            // (c^ - Mc dt k^2 I^) / (1 + Mc dt alpha k^4) / L as fc/L * (c^ - ac I^), ac = Mc dt k^2
            const double fc = Tt[e];
            const double kl = kl_of(e / C, dkl);
            const double ac = d.mc_dt * fma(kl, kl, kb2);
            const double2 ih = s[pi];
            const double2 v = Pk[pi];
            Pk[pi] = make_double2(fc * (v.x - ac * ih.x), fc * (v.y - ac * ih.y));
        }
        __syncthreads();
        if (more) ts.issue(dn->kfn + tile_of(item + 1));  // every thread has read fc
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b);
        tile_out_d<L, C, NT>(s, d.con + tile);
        if (MODE == COL_STEP_CHECKPOINT) {
            // The energy's gradient term alpha sum_x (gx^2 + 2 gy^2) of the new c (ENERGYC2
            // with grao2 twice, MIS:915), as a k-space sum (Parseval): Pk = S C^ (S the
            // inverse-transform scale), so sum_x gx^2 = sum_k w kl^2 |Pk|^2 / (P S^2) over this
            // half spectrum, w = 1 on the self-conjugate column (km = 0, M/2 in 2-D; kn = 0,
            // N/2 in 3-D), 2 on the others.  The reference keeps the real part of the complex
            // inverse transform of -i k C^, which has no derivative along an axis at that
            // axis's Nyquist index: kl = 0 at l = L/2, the m wavenumber 0 at M/2.
            // One partial per spectral column, summed in an order that does not depend on the
            // tile width: a column's L/16 threads take rows t, t + L/16, ... in turn (thread
            // t*C + b of column b), and one thread adds their sums in t order.
            const int b0 = threadIdx.x % C;
            const int kc0 = km3 >= 0 ? (tile_i / d.M) * C + b0 : km0 + b0;  // the half-spectrum column
            const int hc = km3 >= 0 ? d.N / 2 : H;
            const int kmi = km3 >= 0 ? km3 : kc0;                            // its m index
            const double ky = (kc0 > hc || kmi == d.M / 2) ? 0.0 : d.kdm[kmi];
            const double ky2 = dmul(2.0, dmul(ky, ky));
            double g = 0.0;
            for (int e = threadIdx.x; e < L * C; e += NT) {
                const int l = e / C;
                const double kl = l == L / 2 ? 0.0 : kl_of(l, dkl);
                const double2 v = Pk[spad(e)];
                g = fma(fma(kl, kl, ky2), fma(v.x, v.x, dmul(v.y, v.y)), g);
            }
            double *gs = reinterpret_cast<double *>(s);  // s is free: con' has been stored
            __syncthreads();
            gs[threadIdx.x] = g;
            __syncthreads();
            if (threadIdx.x < C) {
                const int kc = km3 >= 0 ? (tile_i / d.M) * C + threadIdx.x : km0 + threadIdx.x;
                if (kc <= hc) {
                    double t = 0.0;
                    for (int i = 0; i < NT / C; ++i) t = dadd(t, gs[i * C + threadIdx.x]);
                    const double w = (kc == 0 || kc == hc) ? 1.0 : 2.0;
                    const int col = km3 >= 0 ? kc * d.M + km3 : kc;  // (kn, km) in 3-D, km in 2-D
                    d.partials[2 * (d.gpart_off + col)] = dmul(dmul(t, w), d.gscale);
                    d.partials[2 * (d.gpart_off + col) + 1] = 0.0;
                }
            }
        }
    }
    st.finish();  // every copy issued has been waited for: the last item issues none
}

template <int L, int C, int MODE, int STAGE>
static cudaError_t mcol_impl(const RunDesc *d_runs, int nruns, int tiles, const TwiddleSet &tw, cudaStream_t st) {
    constexpr int NT = MColCfg<L, C>::NT;
    constexpr size_t smem = MColCfg<L, C>::SMEM;
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_mcol_step<L, C, MODE, STAGE>, smem, mask);
    if (nruns == 0 || e != cudaSuccess) return e;
    const int items = tiles * nruns;
    const int cap = MColCfg<L, C>::MINB * sm_count();
    const int g0 = items < cap ? items : cap;
    const int per = (items + g0 - 1) / g0;
    const int grid = (items + per - 1) / per;
    k_mcol_step<L, C, MODE, STAGE><<<grid, NT, smem, st>>>(d_runs, nruns, per, tw.f64[log2i(L)], tw.fault);
    return cudaGetLastError();
}

template <int L, int C, int STAGE>
static cudaError_t mcol_modes(const RunDesc *d_runs, int nruns, int tiles, int mode, const TwiddleSet &tw,
                              cudaStream_t s) {
    switch (mode) {
        case COL_STEP: return mcol_impl<L, C, COL_STEP, STAGE>(d_runs, nruns, tiles, tw, s);
        case COL_PREPARE: return mcol_impl<L, C, COL_PREPARE, STAGE>(d_runs, nruns, tiles, tw, s);
        case COL_STEP_CHECKPOINT: return mcol_impl<L, C, COL_STEP_CHECKPOINT, STAGE>(d_runs, nruns, tiles, tw, s);
        default: return cudaErrorInvalidValue;
    }
}
template <int L, int C>
static cudaError_t mcol_stages(const RunDesc *d_runs, int nruns, int tiles, int stage, int mode, const TwiddleSet &tw,
                               cudaStream_t s) {
    switch (stage) {
        case STAGE_ASYNC: return mcol_modes<L, C, STAGE_ASYNC>(d_runs, nruns, tiles, mode, tw, s);
        case STAGE_BULK: return mcol_modes<L, C, STAGE_BULK>(d_runs, nruns, tiles, mode, tw, s);
        default: return cudaErrorInvalidValue;
    }
}
template <int L>
static cudaError_t mcol_dispatch(const RunDesc *d_runs, int nruns, int tiles, int C, int stage, int mode,
                                 const TwiddleSet &tw, cudaStream_t s) {
    switch (C) {
        case 1:
            if constexpr (mcol_tile_ok(L, 1)) return mcol_stages<L, 1>(d_runs, nruns, tiles, stage, mode, tw, s);
            break;
        case 2:
            if constexpr (mcol_tile_ok(L, 2)) return mcol_stages<L, 2>(d_runs, nruns, tiles, stage, mode, tw, s);
            break;
        case 4:
            if constexpr (mcol_tile_ok(L, 4)) return mcol_stages<L, 4>(d_runs, nruns, tiles, stage, mode, tw, s);
            break;
        case 8:
            if constexpr (mcol_tile_ok(L, 8)) return mcol_stages<L, 8>(d_runs, nruns, tiles, stage, mode, tw, s);
            break;
        case 16:
            if constexpr (mcol_tile_ok(L, 16)) return mcol_stages<L, 16>(d_runs, nruns, tiles, stage, mode, tw, s);
            break;
        default: break;
    }
    return cudaErrorInvalidValue;
}

template <int L>
cudaError_t launch_col_mixed_L(const RunDesc *d_runs, int nruns, int tiles, int C, int stage, int mode,
                               const TwiddleSet &tw, cudaStream_t s) {
    return mcol_dispatch<L>(d_runs, nruns, tiles, C, stage, mode, tw, s);
}

}  // namespace pfc
