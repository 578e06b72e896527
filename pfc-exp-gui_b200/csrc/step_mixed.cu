// step_mixed.cu -- mixed-precision fused step: FP32 storage in HBM, FP64 arithmetic.
//
// The same two sweeps per step as the FP32 path (step_fp32.cu) over the same row-space
// arrays (FP32 complex, column-tile-major), restating one time step of the reference
// (src/experiment/misfit_uniform_time_seed_fftw_early.cpp:479-501, src/experiment/cvd.cpp:400-422):
//
//   row kernel: inverse row FFTs of psi+i*con and c2a+i*c2b, the pointwise terms
//     UPDATEINN3 / UPDATEINFMIX / UPDATEINFCMIX tail / UPDATEINC2MIX(C) (MIS:773-874),
//     forward row FFT of inn+i*inc;
//   column kernel: forward column FFTs of psi, inn, con, inc; the semi-implicit update
//     MAINEQUATIONC2_NOI / C2MIX (MIS:983-1014, CVD:865-886); inverse column FFTs of
//     psi', C2A psi', C2B psi', con' (and the -i k gradients of con' at checkpoints).
//
// Every value is widened to double when it is loaded and rounded to float once, when it
// is stored: the transforms, the pointwise terms and the update run in FP64, and the
// operator is the pure-FP64 one (k-vectors, k^2, the C2 kernel and the denominators in
// double, as the oracle's pure mode).  What separates this path from a pure-FP64 run is
// therefore only the FP32 storage of the six arrays that cross HBM between the sweeps;
// in the PFC dynamics those roundings stay below 1e-5 after 200 steps, where FP32
// arithmetic in any of the transforms, the pointwise terms or the update does not.
// The k = 0 modes stay in FP64 per run, as on the FP32 path.
//
// HBM traffic is that of the FP32 path, 56 bytes per grid point per step.  Shared
// memory holds double2 values, so the tiles are half as long (MROW_TILE, MCOL_TILE).
// Column-kernel work items are ordered tile-major (all runs of one tile, then the next
// tile) and each CTA takes a contiguous range, so a tile of the shared coefficient
// table is read once from HBM and then from L2 by the other runs of a batch.
#include "pfc_b200.h"
#include "mcol_kernel.cuh"

namespace pfc {

constexpr int MROW_TILE = 2048;  // complex doubles per row-kernel CTA (row step: 2 sequences per row)
constexpr int MCOL_TILE = 2048;  // complex doubles per column tile by default

template <int M> struct MRowCfg {
    static constexpr int RPC = (MROW_TILE / 2) / M >= 1 ? (MROW_TILE / 2) / M : 1;  // rows per CTA
    static constexpr int NB = 2 * RPC;
    static constexpr int NT = (NB * M / 16) < 512 ? (NB * M / 16) : 512;
    static constexpr int MINB = 512 / NT;  // 128 registers per thread
};

int mixed_col_tile_width(int L) {
    int c = MCOL_TILE / L;
    return c > COL_TILE_MAX ? COL_TILE_MAX : (c < 1 ? 1 : c);
}

int mixed_col_tile_candidates(int L, int *out) {
    const int d = mixed_col_tile_width(L);
    int n = 0;
    for (int c : {d / 4, d / 2, d, 2 * d})
        if (mcol_tile_ok(L, c)) out[n++] = c;
    return n;
}

// ---------------------------------------------------------------------------
// Coefficient table (pure FP64 operator), built once per run shape.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double c2_pure(const C2ParamsD &p, double ks) {
    const double s = sqrt(ks);
    if (s <= p.kc) return p.e1 * exp(-(s - p.k1) * (s - p.k1) / p.gg1);
    return p.e2 * exp(-(s - p.k2) * (s - p.k2) / p.gg2);
}

__global__ void k_build_kmix(const RunDesc *__restrict__ run, double mn_dt, double mc_dt, double alpha, C2ParamsD ca,
                             C2ParamsD cb, double4 *__restrict__ kmix, double2 *__restrict__ kc2d) {
    const RunDesc &d = *run;
    const int H = d.M / 2;
    const long tile = (long)d.L * d.CT, total = (long)d.T * tile;
    const double invL = 1.0 / (double)d.L;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int t = (int)(i / tile), rem = (int)(i % tile);
        const int l = rem / d.CT, km = t * d.CT + rem % d.CT;
        if (km > H || (l == 0 && km == 0)) {
            kmix[i] = make_double4(0.0, 0.0, 0.0, 0.0);
            kc2d[i] = make_double2(0.0, 0.0);
            continue;
        }
        const double kl = d.kdl[l], kmv = d.kdm[km];
        const double ks = kl * kl + kmv * kmv;
        const double an = mn_dt * ks, ac = mc_dt * ks, dc = mc_dt * alpha * ks * ks;
        const double fn = 1.0 / (1.0 + an) * invL, fc = 1.0 / (1.0 + dc) * invL;
        kmix[i] = make_double4(fn, an * fn, fc, ac * fc);
        kc2d[i] = make_double2(c2_pure(ca, ks), c2_pure(cb, ks));
    }
}

cudaError_t launch_build_kmix(const RunDesc *d_run, double mn_dt, double mc_dt, double alpha, C2ParamsD a,
                              C2ParamsD b, double4 *kmix, double2 *kc2d, cudaStream_t s) {
    k_build_kmix<<<148 * 4, 256, 0, s>>>(d_run, mn_dt, mc_dt, alpha, a, b, kmix, kc2d);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Pointwise terms (MIS:773-874) and the energy density (MIS:1043-1092) in double.
// ---------------------------------------------------------------------------
struct TermsD {
    double inn, inc;
};
struct CoefsD {
    double niu, ksi, w, alpha, inv_c0, inv_1mc0;
};
__device__ __forceinline__ CoefsD coefs_d(const ModelCoefs &k) {
    CoefsD c;
    c.niu = k.niu;
    c.ksi = k.ksi;
    c.w = k.para_w;
    c.alpha = k.para_alpha;
    c.inv_c0 = 1.0 / (double)k.para_c0;
    c.inv_1mc0 = 1.0 / (1.0 - (double)k.para_c0);
    return c;
}
__device__ __forceinline__ TermsD point_terms_d(const CoefsD &k, double psi, double c, double a, double b) {
    const double psi2 = psi * psi;
    const double in1 = -k.niu * psi2 * 0.5 + k.ksi * psi2 * psi * (1.0 / 3.0);
    const double lc = log(c * k.inv_c0);
    const double omc = 1.0 - c;
    const double l1c = log(omc * k.inv_1mc0);
    const double in2 = k.w * (c * lc + omc * l1c);
    const double c2 = c * c, omc2 = omc * omc;
    const double in3 = -(1.0 - 3.0 * c2 + 2.0 * c2 * c) * a - (1.0 - 3.0 * omc2 + 2.0 * omc2 * omc) * b;
    TermsD t;
    t.inn = in1 + in2 + in3;
    t.inc = k.w * (psi + 1.0) * (lc - l1c) - 3.0 * psi * (a - b) * (c2 - c);
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
__global__ void __launch_bounds__(MRowCfg<M>::NT, MRowCfg<M>::MINB) k_mrow_step(const RunDesc *__restrict__ runs,
                                                                                const double2 *__restrict__ tw) {
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
            const TermsD t =
                point_terms_d(kc, z1.x * invM + d.psi_mean, z1.y * invM + d.con_mean, z2.x * invM, z2.y * invM);
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
// density (ENERGYC2, MIS:1043-1092, every term in double, the grao2-twice gradient of
// MIS:915) and mass summed in double.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(MRowCfg<M>::NT) k_mrow_analysis(const RunDesc *__restrict__ runs,
                                                                  const double2 *__restrict__ tw) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowCfg<M>::NT, H = M / 2;
    constexpr int NB = 3 * RPC;
    extern __shared__ double2 sd[];
    __shared__ double red[2][32];
    const RunDesc &d = runs[blockIdx.y];
    const int L = d.L;
    const int l0 = blockIdx.x * RPC;
    ROW_TILE_LOOP(RPC, H, NT, {
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
        build_pair_d(sd, NB, 3 * r, k, M, wide(z[0]), wide(z[1]));
        build_pair_d(sd, NB, 3 * r + 1, k, M, wide(z[2]), wide(z[3]));
        build_pair_d(sd, NB, 3 * r + 2, k, M, wide(z[4]), wide(z[5]));
    })
    __syncthreads();
    fft_smem<M, NB, NT, false>(sd, tw);
    const double invM = 1.0 / (double)M;
    const CoefsD kc = coefs_d(d.k);
    double acc_e = 0.0, acc_m = 0.0;
    for (int w = threadIdx.x; w < RPC * M; w += NT) {
        const int r = w % RPC, m = w / RPC, l = l0 + r;
        if (l >= L) continue;
        const double2 z1 = sd[spad(m * NB + 3 * r)], z2 = sd[spad(m * NB + 3 * r + 1)],
                      z3 = sd[spad(m * NB + 3 * r + 2)];
        const double dpsi = z1.x * invM;
        const double psi = dpsi + d.psi_mean, c = z1.y * invM + d.con_mean;
        const double a = z2.x * invM, b = z2.y * invM, gx = z3.x * invM, gy = z3.y * invM;
        d.psi_real[(size_t)l * M + m] = (float)psi;
        d.con_real[(size_t)l * M + m] = (float)c;
        const double psi2 = psi * psi;
        const double e_id = psi2 * 0.5 - kc.niu * psi2 * psi * (1.0 / 6.0) + kc.ksi * psi2 * psi2 * (1.0 / 12.0);
        const double lc = log(c * kc.inv_c0), omc = 1.0 - c, l1c = log(omc * kc.inv_1mc0);
        const double e_mix = (psi + 1.0) * kc.w * (c * lc + omc * l1c);
        const double c2 = c * c, omc2 = omc * omc;
        const double in3 = -(1.0 - 3.0 * c2 + 2.0 * c2 * c) * a - (1.0 - 3.0 * omc2 + 2.0 * omc2 * omc) * b;
        const double e_ex = 0.5 * psi * in3 + kc.alpha * (gx * gx + gy * gy + gy * gy);
        acc_e += e_id + e_mix + e_ex;
        acc_m += dpsi;
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
    k_mrow_step<M><<<grid, NT, smem, st>>>(d_runs, tw.f64[log2i(M)]);
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

template <int M>
static cudaError_t mrow_analysis_impl(const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw,
                                      cudaStream_t st) {
    constexpr int RPC = MRowCfg<M>::RPC, NT = MRowCfg<M>::NT;
    constexpr size_t smem = dsmem_bytes<3 * RPC * M>();
    static unsigned mask = 0;
    cudaError_t e = set_smem(k_mrow_analysis<M>, smem, mask);
    if (nruns == 0 || e != cudaSuccess) return e;
    dim3 grid((L + RPC - 1) / RPC, nruns);
    k_mrow_analysis<M><<<grid, NT, smem, st>>>(d_runs, tw.f64[log2i(M)]);
    return cudaGetLastError();
}

cudaError_t launch_row_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                  cudaStream_t s) {
    PFC_SIZE_SWITCH(M, mrow_step_impl, d_runs, nruns, L, tw, s)
}
cudaError_t launch_row_forward_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                     cudaStream_t s) {
    PFC_SIZE_SWITCH(M, mrow_forward_impl, d_runs, nruns, L, tw, s)
}
cudaError_t launch_row_analysis_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                      cudaStream_t s) {
    PFC_SIZE_SWITCH(M, mrow_analysis_impl, d_runs, nruns, L, tw, s)
}
cudaError_t launch_col_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode,
                                  const TwiddleSet &tw, cudaStream_t s) {
    PFC_SIZE_SWITCH(L, launch_col_mixed_L, d_runs, nruns, M, C, stage, mode, tw, s)
}

cudaError_t prepare_rows_mixed(int M) {
    TwiddleSet none{};
    cudaError_t e;
    if ((e = launch_row_step_mixed(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    if ((e = launch_row_forward_mixed(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    return launch_row_analysis_mixed(nullptr, 0, 0, M, none, 0);
}

int analysis_partials_mixed(int L, int M) {
    int rpc = (MROW_TILE / 2) / M;
    if (rpc < 1) rpc = 1;
    return (L + rpc - 1) / rpc;
}

// ---------------------------------------------------------------------------
// Dispatch on the precision of the runs (FP32 or mixed).
// ---------------------------------------------------------------------------
static bool is_mixed(int prec) { return prec == PFC_PRECISION_MIXED; }

cudaError_t launch_row_step(const RunDesc *d_runs, int nruns, int L, int M, int prec, const TwiddleSet &tw,
                            cudaStream_t s) {
    return is_mixed(prec) ? launch_row_step_mixed(d_runs, nruns, L, M, tw, s)
                          : launch_row_step_f32(d_runs, nruns, L, M, tw, s);
}
cudaError_t launch_col_step(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode, int prec,
                            const TwiddleSet &tw, cudaStream_t s) {
    return is_mixed(prec) ? launch_col_step_mixed(d_runs, nruns, L, M, C, stage, mode, tw, s)
                          : launch_col_step_f32(d_runs, nruns, L, M, C, stage, mode, tw, s);
}
cudaError_t launch_row_forward(const RunDesc *d_runs, int nruns, int L, int M, int prec, const TwiddleSet &tw,
                               cudaStream_t s) {
    return is_mixed(prec) ? launch_row_forward_mixed(d_runs, nruns, L, M, tw, s)
                          : launch_row_forward_f32(d_runs, nruns, L, M, tw, s);
}
cudaError_t launch_row_analysis(const RunDesc *d_runs, int nruns, int L, int M, int prec, const TwiddleSet &tw,
                                cudaStream_t s) {
    return is_mixed(prec) ? launch_row_analysis_mixed(d_runs, nruns, L, M, tw, s)
                          : launch_row_analysis_f32(d_runs, nruns, L, M, tw, s);
}
cudaError_t prepare_rows(int M, int prec) { return is_mixed(prec) ? prepare_rows_mixed(M) : prepare_rows_f32(M); }
int analysis_partials(int L, int M, int prec) {
    return is_mixed(prec) ? analysis_partials_mixed(L, M) : analysis_partials_f32(L, M);
}

cudaError_t prepare_size(int L, int M, int C, int stage, int prec) {
    TwiddleSet none{};
    cudaError_t e;
    if ((e = prepare_rows(M, prec)) != cudaSuccess) return e;
    for (int mode = 0; mode < 3; ++mode)
        if ((e = launch_col_step(nullptr, 0, L, M, C, stage, mode, prec, none, 0)) != cudaSuccess) return e;
    return cudaSuccess;
}

}  // namespace pfc
