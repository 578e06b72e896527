// mrow_kernel.cuh -- the row kernels of the mixed-precision fused step (FP32 rows in
// HBM, FP64 arithmetic) and their launchers: the row step, the row forward (real fields
// to row space) and the checkpoint analysis.
//
// Instantiated one row length M per translation unit (row_inst.cu compiled with
// PFC_ROW_M = M); step_mixed.cu reaches them through launch_mrow_M<M>.
#pragma once

#include "mcol_kernel.cuh"

namespace pfc {

template <int M> struct MRowCfg {
    static constexpr int RPC = mrow_rpc(M);  // rows per CTA
    static constexpr int NB = 2 * RPC;
    static constexpr int NT = (NB * M / 16) < 512 ? (NB * M / 16) : 512;  // one radix-16 butterfly per thread
    static constexpr int MINB = 512 / NT;  // 128 registers per thread
};

// ---------------------------------------------------------------------------
// Pointwise terms (MIS:773-874) and the energy density (MIS:1043-1092) in double.
// ---------------------------------------------------------------------------
struct TermsD {
    double inn, inc;
};
struct CoefsD {
    double niu, ksi, w, alpha, inv_c0, inv_1mc0;
    double ksi_3, mniu_2;  // ksi / 3 and -niu / 2
};
__device__ __forceinline__ CoefsD coefs_d(const ModelCoefs &k) {
    CoefsD c;
    c.niu = k.niu;
    c.ksi = k.ksi;
    c.w = k.para_w;
    c.alpha = k.para_alpha;
    c.inv_c0 = 1.0 / (double)k.para_c0;
    c.inv_1mc0 = 1.0 / (1.0 - (double)k.para_c0);
    c.ksi_3 = c.ksi / 3.0;
    c.mniu_2 = -0.5 * c.niu;
    return c;
}
// Pointwise arithmetic of the mixed path is written as explicit fma() and the __d*_rn
// operations, which the compiler never fuses or splits.  Left as a*b + c, the choice of
// fusing is the compiler's for each inlined copy (a thread evaluates several points
// through unrolled copies), so equal inputs could round differently from point to point.
// With every rounding fixed, equal inputs give equal terms: a 3-D state that does not
// depend on n (the CVD initial condition) stays exactly independent of n, as in the
// reference, whose row transforms of a constant row are exact.
// 1 - 3 c^2 + 2 c^3 = 1 + c^2 (2 c - 3), c2 = c^2
__device__ __forceinline__ double cubic_d(double c, double c2) { return fma(c2, fma(2.0, c, -3.0), 1.0); }
__device__ __forceinline__ TermsD point_terms_d(const CoefsD &k, double psi, double c, double a, double b,
                                              const double2 *__restrict__ lt) {
    const double psi2 = dmul(psi, psi);
    const double in1 = dmul(psi2, fma(k.ksi_3, psi, k.mniu_2));  // -niu psi^2 / 2 + ksi psi^3 / 3
    const double lc = log_tab(dmul(c, k.inv_c0), lt);
    const double omc = dsub(1.0, c);
    const double l1c = log_tab(dmul(omc, k.inv_1mc0), lt);
    const double in2 = dmul(k.w, fma(c, lc, dmul(omc, l1c)));
    const double c2 = dmul(c, c), omc2 = dmul(omc, omc);
    const double in3 = -fma(cubic_d(c, c2), a, dmul(cubic_d(omc, omc2), b));
    TermsD t;
    t.inn = dadd(dadd(in1, in2), in3);
    // w (psi + 1)(lc - l1c) - 3 psi (a - b)(c^2 - c)
    t.inc = fma(dmul(-3.0, dmul(psi, dsub(a, b))), dsub(c2, c), dmul(dmul(k.w, dadd(psi, 1.0)), dsub(lc, l1c)));
    return t;
}

// Hermitian pairs in double (the FP32 path's separate / build_pair).
__device__ __forceinline__ void separate_d(double2 zk, double2 zm, double2 &X, double2 &Y) {
    X = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
    Y = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
}
__device__ __forceinline__ void build_pair_d(double2 *s, int NB, int b, int k, int M, double2 X, double2 Y) {
    const int H = M / 2;
    if (k == 0 || k == H) {
        s[spad(k * NB + b)] = make_double2(X.x, Y.x);
    } else {
        s[spad(k * NB + b)] = make_double2(X.x - Y.y, X.y + Y.x);
        s[spad((M - k) * NB + b)] = make_double2(X.x + Y.y, Y.x - X.y);
    }
}

// ---------------------------------------------------------------------------
// Row step: 4 row-space arrays in, 2 out.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(MRowCfg<M>::NT, MRowCfg<M>::MINB)
    k_mrow_step(const RunDesc *__restrict__ runs, const double2 *__restrict__ tw, const double2 *__restrict__ lt) {
    constexpr int RPC = MRowCfg<M>::RPC, NB = MRowCfg<M>::NB, NT = MRowCfg<M>::NT, H = M / 2;
    extern __shared__ double2 sd[];
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    // the noise stream's step index: advanced once per step, read by this step's column kernel
    if (d.noise_amp != 0.0f && blockIdx.x == 0 && threadIdx.x == 0) *d.step_ctr += 1;
    ROW_TILE_LOOP(RPC, H, NT, {
        float2 P = make_float2(0.f, 0.f), Cc = P, A = P, B = P;
        if (l < L) {
            const long o = rs_index(d, l, k);
            P = d.psi[o];
            Cc = d.con[o];
            A = d.ca[o];
            B = d.cb[o];
        }
        build_pair_d(sd, NB, 2 * r, k, M, wide(P), wide(Cc));
        build_pair_d(sd, NB, 2 * r + 1, k, M, wide(A), wide(B));
    })
    __syncthreads();
    fft_smem<M, NB, NT, false>(sd, tw);

    constexpr int PTS = (RPC * M + NT - 1) / NT;
    const double invM = 1.0 / (double)M;
    const CoefsD kc = coefs_d(d.k);
    double2 out[PTS];
    bool bad = false;
#pragma unroll
    for (int q = 0; q < PTS; ++q) {
        const int w = threadIdx.x + q * NT;
        if (w < RPC * M) {
            const int r = w % RPC, m = w / RPC;
            const double2 z1 = sd[spad(m * NB + 2 * r)], z2 = sd[spad(m * NB + 2 * r + 1)];
            const TermsD t = point_terms_d(kc, fma(z1.x, invM, d.psi_mean), fma(z1.y, invM, d.con_mean),
                                           dmul(z2.x, invM), dmul(z2.y, invM), lt);
            out[q] = make_double2(t.inn, t.inc);
            bad |= !(isfinite(t.inn) && isfinite(t.inc));
        }
    }
    // every thread has read the inverse transforms; a non-finite term marks the run
    if (__syncthreads_or(bad) && threadIdx.x == 0) *d.nonfinite = 1;
#pragma unroll
    for (int q = 0; q < PTS; ++q) {
        const int w = threadIdx.x + q * NT;
        if (w < RPC * M) sd[spad(w)] = out[q];  // w = m*RPC + r: RPC interleaved sequences
    }
    __syncthreads();
    fft_smem<M, RPC, NT, true>(sd, tw);
    ROW_TILE_LOOP(RPC, H, NT, {
        if (l < L) {
            double2 X, Y;
            separate_d(sd[spad(k * RPC + r)], sd[spad(((M - k) & (M - 1)) * RPC + r)], X, Y);
            const long o = rs_index(d, l, k);
            d.inn[o] = narrow(X);
            d.inc[o] = narrow(Y);
        }
    })
}

// ---------------------------------------------------------------------------
// Row forward: real psi/con (FP32, [L][M]) minus their FP64 means -> row space.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(MRowCfg<M>::NT) k_mrow_forward(const RunDesc *__restrict__ runs,
                                                                 const double2 *__restrict__ tw) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowCfg<M>::NT, H = M / 2;
    extern __shared__ double2 sd[];
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    for (int w = threadIdx.x; w < RPC * M; w += NT) {
        const int r = w % RPC, m = w / RPC, l = l0 + r;
        double2 z = make_double2(0.0, 0.0);
        if (l < L) {
            const size_t o = (size_t)l * M + m;
            z = make_double2((double)d.psi_real[o] - d.psi_mean, (double)d.con_real[o] - d.con_mean);
        }
        sd[spad(w)] = z;
    }
    __syncthreads();
    fft_smem<M, RPC, NT, true>(sd, tw);
    ROW_TILE_LOOP(RPC, H, NT, {
        if (l < L) {
            double2 X, Y;
            separate_d(sd[spad(k * RPC + r)], sd[spad(((M - k) & (M - 1)) * RPC + r)], X, Y);
            const long o = rs_index(d, l, k);
            d.psi[o] = narrow(X);
            d.con[o] = narrow(Y);
        }
    })
}

// ---------------------------------------------------------------------------
// Analysis row kernel (checkpoints): real fields (rounded once to FP32), and the energy
// density (ENERGYC2, MIS:1043-1092, every term in double) and mass summed in double.  The
// gradient term (the grao2-twice gradient of MIS:915) is summed in k-space by the
// checkpoint column kernel; its per-tile partials follow this kernel's.
// ---------------------------------------------------------------------------
// the analysis transforms two sequences per row (psi + i con, c2a + i c2b): one radix-16
// butterfly per thread
template <int M> struct MRowACfg {
    static constexpr int NT = (2 * MRowCfg<M>::RPC * M / 16) < 1024 ? (2 * MRowCfg<M>::RPC * M / 16) : 1024;
    static constexpr int MINB = 512 / NT >= 1 ? 512 / NT : 1;  // 128 registers per thread, as the step kernel
    static constexpr int MINB_STEP = MINB;                      // the analysis with the next step's row work
};
// STEP = false: the analysis of the state.  STEP = true: the same analysis (the same
// arithmetic, so the same sums), and then the next step's row work from the transforms it
// already holds: the pointwise terms, their forward transform and the inn/inc row-space
// arrays, as k_mrow_step computes them (the same operations in the same order, so the same
// bits).  The next step then starts at its m-axis pass (3-D) or column kernel (2-D).
template <int M, bool STEP>
__global__ void __launch_bounds__(MRowACfg<M>::NT, STEP ? MRowACfg<M>::MINB_STEP : MRowACfg<M>::MINB)
    k_mrow_analysis(const RunDesc *__restrict__ runs, const double2 *__restrict__ tw, const double2 *__restrict__ lt) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowACfg<M>::NT, H = M / 2;
    constexpr int NB = 2 * RPC;
    constexpr int PTS = (RPC * M + NT - 1) / NT;
    extern __shared__ double2 sd[];
    __shared__ double red[2][32];
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    if (STEP && d.noise_amp != 0.0f && blockIdx.x == 0 && threadIdx.x == 0) *d.step_ctr += 1;
    ROW_TILE_LOOP(RPC, H, NT, {
        float2 z[4] = {};
        if (l < L) {
            const long o = rs_index(d, l, k);
            z[0] = d.psi[o];
            z[1] = d.con[o];
            z[2] = d.ca[o];
            z[3] = d.cb[o];
        }
        build_pair_d(sd, NB, 2 * r, k, M, wide(z[0]), wide(z[1]));
        build_pair_d(sd, NB, 2 * r + 1, k, M, wide(z[2]), wide(z[3]));
    })
    __syncthreads();
    fft_smem<M, NB, NT, false>(sd, tw);
    const double invM = 1.0 / (double)M;
    const CoefsD kc = coefs_d(d.k);
    double acc_e = 0.0, acc_m = 0.0;
    double2 out[STEP ? PTS : 1];
    bool bad = false;
#pragma unroll
    for (int q = 0; q < PTS; ++q) {
        const int w = threadIdx.x + q * NT;
        if (STEP) out[q] = make_double2(0.0, 0.0);
        if (w >= RPC * M) continue;
        const int r = w % RPC, m = w / RPC, l = l0 + r;
        if (l >= L) continue;
        const double2 z1 = sd[spad(m * NB + 2 * r)], z2 = sd[spad(m * NB + 2 * r + 1)];
        // explicit roundings, as in point_terms_d: equal inputs give equal outputs
        const double dpsi = dmul(z1.x, invM);
        const double psi = dadd(dpsi, d.psi_mean), c = fma(z1.y, invM, d.con_mean);
        const double a = dmul(z2.x, invM), b = dmul(z2.y, invM);
        d.psi_real[(size_t)l * M + m] = (float)psi;
        d.con_real[(size_t)l * M + m] = (float)c;
        const double psi2 = dmul(psi, psi);
        // psi^2 / 2 - niu psi^3 / 6 + ksi psi^4 / 12 = psi^2 (1/2 + psi (ksi psi / 12 - niu / 6))
        const double e_id = dmul(psi2, fma(psi, fma(dmul(kc.ksi_3, 0.25), psi, dmul(kc.mniu_2, 1.0 / 3.0)), 0.5));
        const double lc = log_tab(dmul(c, kc.inv_c0), lt), omc = dsub(1.0, c), l1c = log_tab(dmul(omc, kc.inv_1mc0), lt);
        const double e_mix = dmul(dmul(dadd(psi, 1.0), kc.w), fma(c, lc, dmul(omc, l1c)));
        const double c2 = dmul(c, c), omc2 = dmul(omc, omc);
        const double in3 = -fma(cubic_d(c, c2), a, dmul(cubic_d(omc, omc2), b));
        // the gradient term alpha (gx^2 + 2 gy^2) is summed in k-space by the checkpoint
        // column kernel (its per-tile partials follow this kernel's in d.partials)
        const double e_ex = dmul(dmul(0.5, psi), in3);
        acc_e += dadd(dadd(e_id, e_mix), e_ex);
        acc_m += dpsi;
        if constexpr (STEP) {
            // the row step's inputs: psi as k_mrow_step forms it (one rounding), c, a, b as above
            const TermsD t = point_terms_d(kc, fma(z1.x, invM, d.psi_mean), c, a, b, lt);
            out[q] = make_double2(t.inn, t.inc);
            bad |= !(isfinite(t.inn) && isfinite(t.inc));
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc_e += __shfl_down_sync(0xffffffffu, acc_e, off);
        acc_m += __shfl_down_sync(0xffffffffu, acc_m, off);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][warp] = acc_e;
        red[1][warp] = acc_m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double se = 0.0, sm = 0.0;
        for (int i = 0; i < NT / 32; ++i) {
            se += red[0][i];
            sm += red[1][i];
        }
        const int lrows = (L - l0) < RPC ? (L - l0) : RPC;
        d.partials[2 * blockIdx.x] = se;
        d.partials[2 * blockIdx.x + 1] = sm + d.psi_mean * (double)lrows * (double)M;
    }
    if constexpr (STEP) {
        // every thread has read the inverse transforms (the barrier above); a non-finite
        // term marks the run
        if (__syncthreads_or(bad) && threadIdx.x == 0) *d.nonfinite = 1;
#pragma unroll
        for (int q = 0; q < PTS; ++q) {
            const int w = threadIdx.x + q * NT;
            if (w < RPC * M) sd[spad(w)] = out[q];  // w = m*RPC + r: RPC interleaved sequences
        }
        __syncthreads();
        fft_smem<M, RPC, NT, true>(sd, tw);
        ROW_TILE_LOOP(RPC, H, NT, {
            if (l < L) {
                double2 X, Y;
                separate_d(sd[spad(k * RPC + r)], sd[spad(((M - k) & (M - 1)) * RPC + r)], X, Y);
                const long o = rs_index(d, l, k);
                d.inn[o] = narrow(X);
                d.inc[o] = narrow(Y);
            }
        })
    }
}

// The column kernel (mcol_kernel.cuh) is instantiated per row length L in col_inst.cu.

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <int n> static constexpr size_t dsmem_bytes() { return sizeof(double2) * padded_len<n>::value; }

template <int M>
static cudaError_t mrow_step_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw, cudaStream_t st) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowCfg<M>::NT;
    constexpr size_t smem = dsmem_bytes<MRowCfg<M>::NB * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_mrow_step<M>, smem, mask);
    if (nruns == 0 || e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_mrow_step<M><<<grid, NT, smem, st>>>(d_runs, tw.f64[log2i(M)], tw.logt);
    return cudaGetLastError();
}

template <int M>
static cudaError_t mrow_forward_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw,
                                     cudaStream_t st) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowCfg<M>::NT;
    constexpr size_t smem = dsmem_bytes<RPC * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_mrow_forward<M>, smem, mask);
    if (nruns == 0 || e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_mrow_forward<M><<<grid, NT, smem, st>>>(d_runs, tw.f64[log2i(M)]);
    return cudaGetLastError();
}

template <int M, bool STEP>
static cudaError_t mrow_analysis_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw,
                                      cudaStream_t st) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowACfg<M>::NT;
    constexpr size_t smem = dsmem_bytes<2 * RPC * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_mrow_analysis<M, STEP>, smem, mask);
    if (nruns == 0 || e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_mrow_analysis<M, STEP><<<grid, NT, smem, st>>>(d_runs, tw.f64[log2i(M)], tw.logt);
    return cudaGetLastError();
}

template <int M>
cudaError_t launch_mrow_M(int kind, const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw, cudaStream_t s) {
    switch (kind) {
        case MROW_STEP: return mrow_step_impl<M>(d_runs, nruns, L, tw, s);
        case MROW_FORWARD: return mrow_forward_impl<M>(d_runs, nruns, L, tw, s);
        case MROW_ANALYSIS: return mrow_analysis_impl<M, false>(d_runs, nruns, L, tw, s);
        case MROW_ANALYSIS_STEP: return mrow_analysis_impl<M, true>(d_runs, nruns, L, tw, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pfc
