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
//     psi', C2A psi', C2B psi', con'; at checkpoints also the energy's gradient term of
//     con' as a k-space sum (one partial per spectral column).
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
// memory holds double2 values, so the tiles are half as long (MROW_TILE, MCOL_TILE),
// except that a row-kernel CTA takes two rows of M = 1024 (mrow_rpc).
// Column-kernel work items are ordered tile-major (all runs of one tile, then the next
// tile) and each CTA takes a contiguous range, so a tile of the shared coefficient
// table is read once from HBM and then from L2 by the other runs of a batch.
#include "pfc_b200.h"
#include "step_common.cuh"

namespace pfc {

constexpr int MCOL_TILE = 2048;  // complex doubles per column tile by default


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

// Plane p of a table of n points: kfn, kfc, kc2a, kc2b (p = 0 .. 3).
__device__ __forceinline__ void put_kmix(double *planes, long n, long i, double fn, double fc, double c2a, double c2b) {
    planes[i] = fn;
    planes[n + i] = fc;
    planes[2 * n + i] = c2a;
    planes[3 * n + i] = c2b;
}

__global__ void k_build_kmix(const RunDesc *__restrict__ run, double mn_dt, double mc_dt, double alpha, C2ParamsD ca,
                             C2ParamsD cb, double *__restrict__ planes) {
    const RunDesc &d = *run;
    const int H = d.M / 2;
    const long tile = (long)d.L * d.CT, total = (long)d.T * tile;
    const double invL = 1.0 / (double)d.L;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int t = (int)(i / tile), rem = (int)(i % tile);
        const int l = rem / d.CT, km = t * d.CT + rem % d.CT;
        if (km > H || (l == 0 && km == 0)) {
            put_kmix(planes, total, i, 0.0, 0.0, 0.0, 0.0);
            continue;
        }
        const double kl = d.kdl[l], kmv = d.kdm[km];
        const double ks = kl * kl + kmv * kmv;
        const double an = mn_dt * ks, dc = mc_dt * alpha * ks * ks;
        put_kmix(planes, total, i, 1.0 / (1.0 + an) * invL, 1.0 / (1.0 + dc) * invL, c2_pure(ca, ks), c2_pure(cb, ks));
    }
}

cudaError_t launch_build_kmix(const RunDesc *d_run, double mn_dt, double mc_dt, double alpha, C2ParamsD a,
                              C2ParamsD b, double *planes, cudaStream_t s) {
    k_build_kmix<<<148 * 4, 256, 0, s>>>(d_run, mn_dt, mc_dt, alpha, a, b, planes);
    return cudaGetLastError();
}

// The 3-D table in layout B of the column view d (T = Tn*M tiles of L x CT): tile t*M + km,
// row l, column c holds k = (kl, km, kn = t*CT + c), zero at k = 0 and past kn = N/2; the
// factors carry the 1/(L*M) of the unnormalised l and m inverse transforms.
__global__ void k_build_kmix3(const RunDesc *__restrict__ run, double mn_dt, double mc_dt, double alpha, C2ParamsD ca,
                              C2ParamsD cb, double *__restrict__ planes) {
    const RunDesc &d = *run;
    const int N = d.N;
    const long tile = (long)d.L * d.CT, total = (long)d.T * tile;
    const double scale = 1.0 / ((double)d.L * (double)d.M);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int ti = (int)(i / tile), rem = (int)(i % tile);
        const int tn = ti / d.M, km = ti % d.M, l = rem / d.CT, kn = tn * d.CT + rem % d.CT;
        if (kn > N / 2 || (l == 0 && km == 0 && kn == 0)) {
            put_kmix(planes, total, i, 0.0, 0.0, 0.0, 0.0);
            continue;
        }
        const double kl = d.kdl[l], kmv = d.kdm[km], knv = d.kdn[kn];
        const double ks = kl * kl + kmv * kmv + knv * knv;
        const double an = mn_dt * ks, dc = mc_dt * alpha * ks * ks;
        put_kmix(planes, total, i, 1.0 / (1.0 + an) * scale, 1.0 / (1.0 + dc) * scale, c2_pure(ca, ks),
                 c2_pure(cb, ks));
    }
}

cudaError_t launch_build_kmix3(const RunDesc *d_col, double mn_dt, double mc_dt, double alpha, C2ParamsD a,
                               C2ParamsD b, double *planes, cudaStream_t s) {
    k_build_kmix3<<<148 * 4, 256, 0, s>>>(d_col, mn_dt, mc_dt, alpha, a, b, planes);
    return cudaGetLastError();
}

__global__ void k_log_selftest(const double *__restrict__ x, double *__restrict__ y, int n,
                               const double2 *__restrict__ tab) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = log_tab(x[i], tab);
}

cudaError_t launch_log_selftest(const double *x, double *y, int n, const double2 *tab, cudaStream_t s) {
    const int blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    k_log_selftest<<<blocks, 256, 0, s>>>(x, y, n, tab);
    return cudaGetLastError();
}

// Row lengths of the mixed row kernels: 2-D rows (32 ... 2048) and the short n-rows of
// 3-D runs (8, 16).
#define PFC_MROW_SWITCH(n, FN, ...)             \
    switch (n) {                                \
        case 8: return FN<8>(__VA_ARGS__);      \
        case 16: return FN<16>(__VA_ARGS__);    \
        case 32: return FN<32>(__VA_ARGS__);    \
        case 64: return FN<64>(__VA_ARGS__);    \
        case 128: return FN<128>(__VA_ARGS__);  \
        case 256: return FN<256>(__VA_ARGS__);  \
        case 512: return FN<512>(__VA_ARGS__);  \
        case 1024: return FN<1024>(__VA_ARGS__); \
        case 2048: return FN<2048>(__VA_ARGS__); \
        default: return cudaErrorInvalidValue;  \
    }

bool mixed_row_len_ok(int n) { return n >= 8 && n <= 2048 && (n & (n - 1)) == 0; }


cudaError_t launch_row_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                  cudaStream_t s) {
    PFC_MROW_SWITCH(M, launch_mrow_M, MROW_STEP, d_runs, nruns, L, tw, s)
}
cudaError_t launch_row_forward_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                     cudaStream_t s) {
    PFC_MROW_SWITCH(M, launch_mrow_M, MROW_FORWARD, d_runs, nruns, L, tw, s)
}
cudaError_t launch_row_analysis_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                      cudaStream_t s) {
    PFC_MROW_SWITCH(M, launch_mrow_M, MROW_ANALYSIS, d_runs, nruns, L, tw, s)
}
cudaError_t launch_row_analysis_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                           cudaStream_t s) {
    PFC_MROW_SWITCH(M, launch_mrow_M, MROW_ANALYSIS_STEP, d_runs, nruns, L, tw, s)
}
cudaError_t launch_col_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode,
                                  const TwiddleSet &tw, cudaStream_t s) {
    const int tiles = (M / 2 + 1 + C - 1) / C;
    PFC_SIZE_SWITCH(L, launch_col_mixed_L, d_runs, nruns, tiles, C, stage, mode, tw, s)
}
cudaError_t launch_col_step_mixed_tiles(const RunDesc *d_runs, int nruns, int L, int tiles, int C, int stage,
                                        int mode, const TwiddleSet &tw, cudaStream_t s) {
    PFC_SIZE_SWITCH(L, launch_col_mixed_L, d_runs, nruns, tiles, C, stage, mode, tw, s)
}

cudaError_t prepare_rows_mixed(int M) {
    TwiddleSet none{};
    cudaError_t e;
    if ((e = launch_row_step_mixed(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    if ((e = launch_row_forward_mixed(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    if ((e = launch_row_analysis_step_mixed(nullptr, 0, 0, M, none, 0)) != cudaSuccess) return e;
    return launch_row_analysis_mixed(nullptr, 0, 0, M, none, 0);
}

int analysis_partials_mixed(int L, int M) {
    const int rpc = mrow_rpc(M);
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
