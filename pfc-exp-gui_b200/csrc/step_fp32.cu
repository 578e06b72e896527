// step_fp32.cu -- fused FP32 semi-implicit spectral step (2-D Misfit / CVD).
//
// Restates, as two fused sweeps, one time step of the reference
// (src/experiment/misfit_uniform_time_seed_fftw_early.cpp:479-501 and
// src/experiment/cvd.cpp:400-422):
//
//   row kernel (one CTA per RPC rows l):
//     inverse row FFTs of psi+i*con and c2a+i*c2b   (p2/p7 and p10/p11 of the reference)
//     pointwise UPDATEINN3 + UPDATEINFMIX + UPDATEINFCMIX tail + UPDATEINC2MIX(C)
//       (MIS:773-874) -> inn, inc
//     forward row FFT of inn+i*inc                  (first half of p8/p9)
//   column kernel (one CTA per tile of CT packed columns km):
//     forward column FFTs of psi, inn, con, inc     (second half of p1/p8/p6/p9)
//     semi-implicit update MAINEQUATIONC2_NOI/C2MIX (MIS:983-1014, CVD:865-886) with
//       the denominators built in FP64 and rounded, k = 0 held out in FP64
//     C2A/C2B multiply (MIS:807-810) and inverse column FFTs of psi', c2a, c2b, con'
//
// Row-space arrays are stored column-tile-major: element (l, km) at
// ((km / CT) * L + l) * CT + km % CT, so a column kernel tile (L rows x CT columns)
// is one contiguous block, and RPC consecutive rows of one tile are RPC*CT
// contiguous elements for the row kernel.
//
// Compulsory HBM traffic: row kernel reads 4 and writes 2 row-space arrays, column
// kernel reads 4 and writes 4; a row-space array is 4 bytes per grid point, so one
// step moves 56 bytes per point.
#include "step_common.cuh"

namespace pfc {

constexpr int ROW_TILE = 8192;  // complex elements per row-kernel CTA (64 KB in FP32)

template <int M> struct RowCfg {
    static constexpr int RPC = (ROW_TILE / 2) / M >= 1 ? (ROW_TILE / 2) / M : 1;  // rows per CTA
    static constexpr int NB = 2 * RPC;
    static constexpr int NT = (NB * M / 16) < 512 ? (NB * M / 16) : 512;
};

int col_tile_width(int L) {
    int c = COL_TILE / L;
    return c > 16 ? 16 : (c < 1 ? 1 : c);
}

int col_tile_candidates(int L, int *out) {
    const int d = col_tile_width(L);
    int n = 0;
    for (int c : {d / 4, d / 2, d, 2 * d})
        if (col_tile_ok(L, c)) out[n++] = c;
    return n;
}

// Per k-point coefficients of one run (RunDesc::kcoef), built once in FP64 and rounded.
// ks and the k^4 product use the reference's float operation order (ks, MAINEQUATIONC2_NOI,
// MIS:1002-1010); the intrinsics keep them from being contracted into FMAs.
__global__ void k_build_kcoef(const RunDesc *__restrict__ run, float2 *__restrict__ den, float2 *__restrict__ c2) {
    const RunDesc &d = *run;
    const int H = d.M / 2;
    const long tile = (long)d.L * d.CT, total = (long)d.T * tile;
    const float mn_dt = __fmul_rn(d.k.dynamic_mn, d.dt), mc_dt = __fmul_rn(d.k.dynamic_mc, d.dt);
    const float mc_dt_alpha = __fmul_rn(mc_dt, d.k.para_alpha);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int t = (int)(i / tile), rem = (int)(i % tile);
        const int l = rem / d.CT, km = t * d.CT + rem % d.CT;
        if (km > H || (l == 0 && km == 0)) {
            den[i] = make_float2(0.f, 0.f);
            c2[i] = make_float2(0.f, 0.f);
            continue;
        }
        const float kl = d.krefl[l], kmv = d.krefm[km];
        const float ks = __fadd_rn(__fmul_rn(kl, kl), __fmul_rn(kmv, kmv));
        const float an = __fmul_rn(mn_dt, ks);
        const float dc = __fmul_rn(__fmul_rn(mc_dt_alpha, ks), ks);
        const float fn = (float)((1.0 / (1.0 + (double)an)) / (double)d.L);
        const float fc = (float)((1.0 / (1.0 + (double)dc)) / (double)d.L);
        den[i] = make_float2(fn, fc);
        c2[i] = make_float2(c2_ref(d.c2a, ks), c2_ref(d.c2b, ks));
    }
}

cudaError_t launch_build_kcoef(const RunDesc *d_run, float2 *kden, float2 *kc2, cudaStream_t s) {
    k_build_kcoef<<<148 * 4, 256, 0, s>>>(d_run, kden, kc2);
    return cudaGetLastError();
}

// Nonlinear chemical-potential terms at one grid point (MIS:773-874), FP32.
struct PointTerms {
    float inn, inc;
};
__device__ __forceinline__ PointTerms point_terms(const ModelCoefs &k, float inv_c0, float inv_1mc0, float psi,
                                                   float c, float a, float b) {
    const float psi2 = psi * psi;
    const float in1 = -k.niu * psi2 * 0.5f + k.ksi * psi2 * psi * (1.0f / 3.0f);
    const float lc = logf(c * inv_c0);
    const float omc = 1.0f - c;
    const float l1c = logf(omc * inv_1mc0);
    const float in2 = k.para_w * (c * lc + omc * l1c);
    const float c2 = c * c, omc2 = omc * omc;
    const float in3 = -(1.0f - 3.0f * c2 + 2.0f * c2 * c) * a - (1.0f - 3.0f * omc2 + 2.0f * omc2 * omc) * b;
    const float wp = k.para_w * (psi + 1.0f);
    PointTerms t;
    t.inn = in1 + in2 + in3;
    t.inc = wp * (lc - l1c) - 3.0f * psi * (a - b) * (c2 - c);
    return t;
}

// Hermitian separation of Z = FFT(x + i y) into X[k], Y[k] (k = 0..M/2).
__device__ __forceinline__ void separate(float2 zk, float2 zm, float2 &X, float2 &Y) {
    X = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    Y = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
}

// Write Z[k], Z[M-k] of Z = IFFT-input for the real pair (x, y) from half spectra X, Y.
__device__ __forceinline__ void build_pair(float2 *s, int NB, int b, int k, int M, float2 X, float2 Y) {
    const int H = M / 2;
    if (k == 0 || k == H) {
        s[spad(k * NB + b)] = make_float2(X.x, Y.x);
    } else {
        s[spad(k * NB + b)] = make_float2(X.x - Y.y, X.y + Y.x);
        s[spad((M - k) * NB + b)] = make_float2(X.x + Y.y, Y.x - X.y);
    }
}

// Balancing the two members of a packed transform.  The rounding error a transform
// adds to either member of x + i y is set by the larger of the two, so a member that
// is much smaller than its partner (con beside phi in Misfit runs: deviations about
// 60 times smaller) loses that many bits.  The smaller member therefore rides as
// 2^e * y, e = exponent(max|x|) - exponent(max|y|); multiplying by 2^e and 2^-e is
// exact, so the balancing adds no rounding of its own.
// The exponent is chosen in the same kernel from the values being packed: the
// fields change by orders of magnitude within a few steps early in a run, so an
// exponent carried over from the previous step can push y far past x.
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }  // |e| <= 30
__device__ __forceinline__ int balance_exp(unsigned ax, unsigned ay) {  // bit patterns of max|x|, max|y|
    if (ax == 0u || ay == 0u) return 0;
    const int e = (int)(ax >> 23) - (int)(ay >> 23);
    return e < -30 ? -30 : (e > 30 ? 30 : e);
}
// Block-wide maximum of non-negative floats: every thread calls block_max_put, each
// warp leaves its maximum (float bits) in wm[warp], and after the next
// __syncthreads block_max_get<NT / 32> combines the warps' slots.
__device__ __forceinline__ void block_max_put(unsigned *wm, float v) {
    const unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(v));
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = u;
}
template <int NW> __device__ __forceinline__ unsigned block_max_get(const unsigned *wm) {
    unsigned u = 0u;
#pragma unroll
    for (int i = 0; i < NW; ++i) u = u > wm[i] ? u : wm[i];
    return u;
}
__device__ __forceinline__ float absmax2(float2 v) { return fmaxf(fabsf(v.x), fabsf(v.y)); }

// The row-space walk (ROW_TILE_LOOP, step_common.cuh) unrolled over a fixed bound IT of
// iterations per thread; the body sees the iteration index `it`, so values can stay in
// registers from one walk to the next.  A run's Hp = round_up(M/2 + 1, CT) with
// CT <= COL_TILE_MAX, so T * CT * RPC <= (M/2 + COL_TILE_MAX) * RPC and
// IT = ceil((M/2 + COL_TILE_MAX) * RPC / NT) covers every element.
template <int M, int RPC, int NT> struct RowWalk {
    static constexpr int IT = ((M / 2 + COL_TILE_MAX) * RPC + NT - 1) / NT;
};
#define ROW_TILE_LOOP_REG(RPC, H, NT, IT, ...)                             \
    {                                                                       \
        const int _ct = d.CT, _lct = d.lct;                                 \
        const int _lblk = ilog2<(RPC)>::value + _lct;                       \
        const int _total = d.T << _lblk;                                    \
        _Pragma("unroll") for (int it = 0; it < (IT); ++it) {               \
            const int w = threadIdx.x + it * (NT);                          \
            if (w >= _total) continue;                                      \
            const int t = w >> _lblk, rem = w & ((1 << _lblk) - 1);         \
            const int r = rem >> _lct, k = (t << _lct) + (rem & (_ct - 1)); \
            if (k > (H)) continue;                                          \
            const int l = l0 + r;                                           \
            (void)l;                                                        \
            __VA_ARGS__                                                     \
        }                                                                   \
    }

// ---------------------------------------------------------------------------
// Row kernel: 4 row-space arrays in, 2 out.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(RowCfg<M>::NT, 2) k_row_step(const RunDesc *__restrict__ runs,
                                                             const float2 *__restrict__ tw) {
    constexpr int RPC = RowCfg<M>::RPC, NB = RowCfg<M>::NB, NT = RowCfg<M>::NT, H = M / 2;
    constexpr int NW = NT / 32;
    extern __shared__ float2 s[];
    __shared__ unsigned wmax[4][NW];  // per-warp maxima of |phi^|, |con^|, |inn|, |inc| (float bits)
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    // the noise stream's step index: advanced once per step, read by this step's column kernel
    if (d.noise_amp != 0.0f && blockIdx.x == 0 && threadIdx.x == 0) *d.step_ctr += 1;
    // phi^ and con^ stay in registers until the block's maxima give the balance
    // exponent; ca^ and cb^ go straight into their packed pair
    constexpr int LIT = RowWalk<M, RPC, NT>::IT;
    float2 Pr[LIT], Cr[LIT];
    float mp = 0.f, mc = 0.f;
    ROW_TILE_LOOP_REG(RPC, H, NT, LIT, {
        float2 P = make_float2(0.f, 0.f), Cc = P, A = P, B = P;
        if (l < L) {
            const long o = rs_index(d, l, k);
            P = d.psi[o];
            Cc = d.con[o];
            A = d.ca[o];
            B = d.cb[o];
        }
        Pr[it] = P;
        Cr[it] = Cc;
        build_pair(s, NB, 2 * r + 1, k, M, A, B);
        mp = fmaxf(mp, absmax2(P));
        mc = fmaxf(mc, absmax2(Cc));
    })
    block_max_put(wmax[0], mp);
    block_max_put(wmax[1], mc);
    __syncthreads();
    // con rides as 2^e1 * con beside phi (balance_exp)
    const float g1 = pow2f(balance_exp(block_max_get<NW>(wmax[0]), block_max_get<NW>(wmax[1])));
    ROW_TILE_LOOP_REG(RPC, H, NT, LIT,
                      { build_pair(s, NB, 2 * r, k, M, Pr[it], make_float2(Cr[it].x * g1, Cr[it].y * g1)); })
    __syncthreads();
    fft_smem<M, NB, NT, false>(s, tw);

    constexpr int PTS = (RPC * M + NT - 1) / NT;
    const float invM = 1.0f / (float)M;
    const float cs = invM / g1;  // 2^-e1 / M, exact
    const float inv_c0 = 1.0f / d.k.para_c0, inv_1mc0 = 1.0f / (1.0f - d.k.para_c0);
    float2 out[PTS];
    float mi = 0.f, mj = 0.f;
    bool bad = false;
#pragma unroll
    for (int q = 0; q < PTS; ++q) {
        const int w = threadIdx.x + q * NT;
        if (w < RPC * M) {
            const int r = w % RPC, m = w / RPC;
            const float2 z1 = s[spad(m * NB + 2 * r)], z2 = s[spad(m * NB + 2 * r + 1)];
            const float psi = z1.x * invM + d.psi_mean_f, c = z1.y * cs + d.con_mean_f;
            const PointTerms t = point_terms(d.k, inv_c0, inv_1mc0, psi, c, z2.x * invM, z2.y * invM);
            out[q] = make_float2(t.inn, t.inc);
            mi = fmaxf(mi, fabsf(t.inn));
            mj = fmaxf(mj, fabsf(t.inc));
            bad |= !(isfinite(t.inn) && isfinite(t.inc));
        }
    }
    block_max_put(wmax[2], mi);
    block_max_put(wmax[3], mj);
    // a non-finite term marks the run (fmaxf would pass over a NaN)
    if (__syncthreads_or(bad) && threadIdx.x == 0) *d.nonfinite = 1;
    // inc rides as 2^e2 * inc beside inn
    const int e2 = balance_exp(block_max_get<NW>(wmax[2]), block_max_get<NW>(wmax[3]));
    const float s2 = pow2f(e2);
#pragma unroll
    for (int q = 0; q < PTS; ++q) {
        const int w = threadIdx.x + q * NT;
        if (w < RPC * M) s[spad(w)] = make_float2(out[q].x, out[q].y * s2);  // w = m*RPC + r: NB' = RPC
    }
    __syncthreads();
    fft_smem<M, RPC, NT, true>(s, tw);
    const float is2 = pow2f(-e2);
    ROW_TILE_LOOP(RPC, H, NT, {
        if (l < L) {
            float2 X, Y;
            separate(s[spad(k * RPC + r)], s[spad(((M - k) & (M - 1)) * RPC + r)], X, Y);
            const long o = rs_index(d, l, k);
            d.inn[o] = X;
            d.inc[o] = make_float2(Y.x * is2, Y.y * is2);
        }
    })
}

// ---------------------------------------------------------------------------
// Row forward: real psi/con (FP32, [L][M]) minus their FP64 means -> row space.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(RowCfg<M>::NT) k_row_forward(const RunDesc *__restrict__ runs,
                                                                const float2 *__restrict__ tw) {
    constexpr int RPC = RowCfg<M>::RPC, NT = RowCfg<M>::NT, H = M / 2;
    constexpr int NW = NT / 32;
    extern __shared__ float2 s[];
    __shared__ unsigned wmax[2][NW];
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    // deviations from the FP64 means; con rides as 2^e * con beside phi (balance_exp)
    float mp = 0.f, mc = 0.f;
    for (int w = threadIdx.x; w < RPC * M; w += NT) {
        const int r = w % RPC, m = w / RPC, l = l0 + r;
        float2 z = make_float2(0.f, 0.f);
        if (l < L) {
            const size_t o = (size_t)l * M + m;
            z = make_float2((float)((double)d.psi_real[o] - d.psi_mean), (float)((double)d.con_real[o] - d.con_mean));
        }
        s[spad(w)] = z;
        mp = fmaxf(mp, fabsf(z.x));
        mc = fmaxf(mc, fabsf(z.y));
    }
    block_max_put(wmax[0], mp);
    block_max_put(wmax[1], mc);
    __syncthreads();
    const int e = balance_exp(block_max_get<NW>(wmax[0]), block_max_get<NW>(wmax[1]));
    const float sc = pow2f(e);
    for (int w = threadIdx.x; w < RPC * M; w += NT) s[spad(w)].y *= sc;
    __syncthreads();
    fft_smem<M, RPC, NT, true>(s, tw);
    const float isc = pow2f(-e);
    ROW_TILE_LOOP(RPC, H, NT, {
        if (l < L) {
            float2 X, Y;
            separate(s[spad(k * RPC + r)], s[spad(((M - k) & (M - 1)) * RPC + r)], X, Y);
            const long o = rs_index(d, l, k);
            d.psi[o] = X;
            d.con[o] = make_float2(Y.x * isc, Y.y * isc);
        }
    })
}

// The column kernel (col_kernel.cuh) is instantiated per row length L in col_inst.cu.

// ---------------------------------------------------------------------------
// Analysis row kernel (checkpoints): real fields, energy density and mass.
// ENERGYC2 (MIS:1043-1092): float energy terms, double accumulation.  The mass is
// accumulated as sum(phi - mean) plus the FP64 mean, so it carries no rounding of
// the mean itself.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(RowCfg<M>::NT) k_row_analysis(const RunDesc *__restrict__ runs,
                                                                 const float2 *__restrict__ tw) {
    constexpr int RPC = RowCfg<M>::RPC, NT = RowCfg<M>::NT, H = M / 2;
    constexpr int NB = 3 * RPC;
    constexpr int NW = NT / 32;
    extern __shared__ float2 s[];
    __shared__ double red[2][32];
    __shared__ unsigned wmax[2][NW];
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    // phi^ and con^ stay in registers until the block's maxima give the balance exponent
    constexpr int LIT = RowWalk<M, RPC, NT>::IT;
    float2 Pr[LIT], Cr[LIT];
    float mp = 0.f, mc = 0.f;
    ROW_TILE_LOOP_REG(RPC, H, NT, LIT, {
        float2 z[6] = {};
        if (l < L) {
            const long o = rs_index(d, l, k);
            z[0] = d.psi[o];
            z[1] = d.con[o];
            z[2] = d.ca[o];
            z[3] = d.cb[o];
            z[4] = d.gx[o];
            z[5] = d.gy[o];
        }
        Pr[it] = z[0];
        Cr[it] = z[1];
        build_pair(s, NB, 3 * r + 1, k, M, z[2], z[3]);
        build_pair(s, NB, 3 * r + 2, k, M, z[4], z[5]);
        mp = fmaxf(mp, absmax2(z[0]));
        mc = fmaxf(mc, absmax2(z[1]));
    })
    block_max_put(wmax[0], mp);
    block_max_put(wmax[1], mc);
    __syncthreads();
    // con rides as 2^e1 * con beside phi (balance_exp)
    const float g1 = pow2f(balance_exp(block_max_get<NW>(wmax[0]), block_max_get<NW>(wmax[1])));
    ROW_TILE_LOOP_REG(RPC, H, NT, LIT,
                      { build_pair(s, NB, 3 * r, k, M, Pr[it], make_float2(Cr[it].x * g1, Cr[it].y * g1)); })
    __syncthreads();
    fft_smem<M, NB, NT, false>(s, tw);
    const float invM = 1.0f / (float)M;
    const ModelCoefs &k = d.k;
    const float inv_c0 = 1.0f / k.para_c0, inv_1mc0 = 1.0f / (1.0f - k.para_c0);
    double acc_e = 0.0, acc_m = 0.0;
    for (int w = threadIdx.x; w < RPC * M; w += NT) {
        const int r = w % RPC, m = w / RPC, l = l0 + r;
        if (l >= L) continue;
        const float2 z1 = s[spad(m * NB + 3 * r)], z2 = s[spad(m * NB + 3 * r + 1)], z3 = s[spad(m * NB + 3 * r + 2)];
        const float dpsi = z1.x * invM;
        const float psi = dpsi + d.psi_mean_f, c = z1.y * (invM / g1) + d.con_mean_f;  // invM / g1 = 2^-e1 / M, exact
        const float a = z2.x * invM, b = z2.y * invM, gx = z3.x * invM, gy = z3.y * invM;
        d.psi_real[(size_t)l * M + m] = psi;
        d.con_real[(size_t)l * M + m] = c;
        const float psi2 = psi * psi;
        const float e_id = psi2 * 0.5f - k.niu * psi2 * psi * (1.0f / 6.0f) + k.ksi * psi2 * psi2 * (1.0f / 12.0f);
        const float lc = logf(c * inv_c0), omc = 1.0f - c, l1c = logf(omc * inv_1mc0);
        const float e_mix = (psi + 1.0f) * k.para_w * (c * lc + omc * l1c);
        const float c2 = c * c, omc2 = omc * omc;
        const float in3 = -(1.0f - 3.0f * c2 + 2.0f * c2 * c) * a - (1.0f - 3.0f * omc2 + 2.0f * omc2 * omc) * b;
        const float e_ex = 0.5f * psi * in3 + k.para_alpha * (gx * gx + gy * gy + gy * gy);
        acc_e += (double)(e_id + e_mix + e_ex);
        acc_m += (double)dpsi;
    }
    // deterministic block reduction
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
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <int M>
static cudaError_t row_step_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw, cudaStream_t st) {
    constexpr int RPC = RowCfg<M>::RPC, NT = RowCfg<M>::NT;
    constexpr size_t smem = smem_bytes<RowCfg<M>::NB * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_row_step<M>, smem, mask);
    if (nruns == 0) return e;
    if (e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_row_step<M><<<grid, NT, smem, st>>>(d_runs, tw.f32[log2i(M)]);
    return cudaGetLastError();
}

template <int M>
static cudaError_t row_forward_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw, cudaStream_t st) {
    constexpr int RPC = RowCfg<M>::RPC, NT = RowCfg<M>::NT;
    constexpr size_t smem = smem_bytes<RPC * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_row_forward<M>, smem, mask);
    if (nruns == 0) return e;
    if (e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_row_forward<M><<<grid, NT, smem, st>>>(d_runs, tw.f32[log2i(M)]);
    return cudaGetLastError();
}

template <int M>
static cudaError_t row_analysis_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw,
                                     cudaStream_t st) {
    constexpr int RPC = RowCfg<M>::RPC, NT = RowCfg<M>::NT;
    constexpr size_t smem = smem_bytes<3 * RPC * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_row_analysis<M>, smem, mask);
    if (nruns == 0) return e;
    if (e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_row_analysis<M><<<grid, NT, smem, st>>>(d_runs, tw.f32[log2i(M)]);
    return cudaGetLastError();
}

cudaError_t launch_row_step_f32(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw, cudaStream_t s) {
    PFC_SIZE_SWITCH(M, row_step_impl, d_runs, nruns, L, tw, s)
}

cudaError_t launch_row_forward_f32(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                   cudaStream_t s) {
    PFC_SIZE_SWITCH(M, row_forward_impl, d_runs, nruns, L, tw, s)
}

cudaError_t launch_row_analysis_f32(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                    cudaStream_t s) {
    PFC_SIZE_SWITCH(M, row_analysis_impl, d_runs, nruns, L, tw, s)
}

cudaError_t launch_col_step_f32(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode,
                                const TwiddleSet &tw, cudaStream_t s) {
    PFC_SIZE_SWITCH(L, launch_col_f32_L, d_runs, nruns, M, C, stage, mode, tw, s)
}

// Self-test of the column kernel's tile staging (one CTA of 128 threads): with issue,
// thread 0 stages n float2 of src into shared memory by one bulk copy, every thread
// waits (bounded by limit_ns) and the tile is written back to dst; without issue no
// copy is started, so the wait runs out, the CTA sets *fault and returns.
__global__ void k_stage_selftest(const float2 *src, float2 *dst, int n, int issue, unsigned long long limit_ns,
                                 int *fault) {
    extern __shared__ __align__(16) float2 q[];
    __shared__ __align__(8) unsigned long long bar_word;
    const unsigned bar = smem_u32(&bar_word);
    stage_init(bar);
    if (issue) stage_issue(bar, src, q, (unsigned)(n * sizeof(float2)));
    if (!tile_wait(bar, 0u, fault, limit_ns)) return;
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = q[i];
}

cudaError_t launch_stage_selftest(const float2 *src, float2 *dst, int n, int issue, unsigned long long limit_ns,
                                  int *fault, cudaStream_t s) {
    if (n < 2 || n > 8192 || (n & 1)) return cudaErrorInvalidValue;  // whole 16-byte units, <= 64 KB
    const size_t smem = sizeof(float2) * n;
    cudaError_t e = cudaFuncSetAttribute(k_stage_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_stage_selftest<<<1, 128, smem, s>>>(src, dst, n, issue, limit_ns, fault);
    return cudaGetLastError();
}

cudaError_t prepare_rows_f32(int M) {
    // nruns == 0: only the shared-memory attributes are set, nothing is launched
    TwiddleSet none{};
    cudaError_t e;
    if ((e = launch_row_step_f32(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    if ((e = launch_row_forward_f32(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    return launch_row_analysis_f32(nullptr, 0, 0, M, none, 0);
}

int analysis_partials_f32(int L, int M) {
    int rpc = (ROW_TILE / 2) / M;
    if (rpc < 1) rpc = 1;
    return (L + rpc - 1) / rpc;
}

}  // namespace pfc
