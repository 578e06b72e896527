// pfc_internal.h -- device-side run descriptors and internal launch interfaces.
//
// A "run" is one Misfit or CVD simulation.  Its FP32 state lives in row space:
// every field f[l][m] (m fastest, the reference's n + N*(m + M*l) layout with N = 1,
// misfit_uniform_time_seed_fftw_early.cpp:600) is stored as its unnormalised DFT
// along m, bins 0..M/2 (Hermitian half), in a row of Hp >= M/2 + 1 complex floats.
// The k = 0 mode of phi and con is held separately in FP64 and kept out of the
// FP32 arrays (their DC bin is zero), so the mass is conserved exactly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pfc {

enum Model : int { MODEL_MISFIT = 0, MODEL_CVD = 1 };

// Model coefficients of the reference (float statics at
// misfit_uniform_time_seed_fftw_early.cpp:116-143 and cvd.cpp:26-53).
struct ModelCoefs {
    float niu, ksi, para_w, para_c0, para_alpha, dynamic_mn, dynamic_mc;
    float gaa1, gaa2, gab1, gab2;
    float ka0, ka1, ka2, kb0, kb1, kb2;
    float sigMa1, sigMa2, sigMb1, sigMb2;
};

// Two-peak correlation kernel parameters (misfit_uniform_time_seed_fftw_early.cpp:700-750):
// C2(k) = e1 * exp(-(|k| - k1)^2 * i1) for |k| <= kc, else e2 * exp(-(|k| - k2)^2 * i2).
struct C2Params {
    float kc, e1, e2, k1, k2, i1, i2;
    float q1, q2;    // sig / sigM1, sig / sigM2 (float quotients, as the reference forms them)
    float gg1, gg2;  // 2 * g1 * g1, 2 * g2 * g2 (float products)
};

struct RunDesc {
    int L, M, N;      // grid (N = 1 for 2-D)
    int Hp;           // padded number of packed columns (T * CT >= M/2 + 1)
    int CT, lct, T;   // column-tile width (power of two), its log2, number of tiles
    int stage;        // column-kernel tile staging (ColStage; a launch choice, results do not depend on it)
    int model;
    // row-space arrays, T tiles of [L][CT] float2 each: (l, km) at ((km/CT)*L + l)*CT + km%CT
    float2 *psi, *con, *ca, *cb, *inn, *inc, *gx, *gy;
    // real-space checkpoint outputs, [L][M] float
    float *psi_real, *con_real;
    // reference k-vectors (float), lengths L and M
    const float *krefl, *krefm;
    // per k-point coefficients in the row-space tile layout (0 at k = 0, the FP64-held mode):
    //   kden = ((float)(1/(1 + Mn dt k^2) / L), (float)(1/(1 + Mc dt alpha k^4) / L))
    //   kc2  = (C2A(k), C2B(k)) as the reference's float tables
    const float2 *kden, *kc2;
    // FP64 means of phi and con (the k = 0 modes / P), and their float roundings
    double psi_mean, con_mean;
    float psi_mean_f, con_mean_f;
    float dt;
    ModelCoefs k;
    C2Params c2a, c2b;
    // mixed-precision runs (FP32 storage, FP64 arithmetic) only, pure-FP64 operator, one
    // double per k-point in four planes of the column kernel's tile layout (0 at k = 0 and
    // in the padding columns): kfn = fn*S, kfc = fc*S, kc2a = C2A(k), kc2b = C2B(k), with
    // fn = 1/(1 + Mn dt k^2), fc = 1/(1 + Mc dt alpha k^4) and S the scale of the
    // unnormalised inverse transforms (1/L, or 1/(L*M) for a 3-D column view);
    // mn_dt = Mn dt and mc_dt = Mc dt (the column kernel forms an = mn_dt k^2 and
    // ac = mc_dt k^2 from the k-vectors); kdl, kdm, kdn: the k-vectors in double, entry
    // i = s(i) * dkl (dkm, dkn) with s(i) = i for i <= n/2, else i - n, and dk = 2 pi / (n dx)
    const double *kfn, *kfc, *kc2a, *kc2b;
    double mn_dt, mc_dt;
    const double *kdl, *kdm, *kdn;
    double dkl, dkm, dkn;
    // column view of a 3-D run (col3d = 1): the column kernel's tiles are (n-tile t, km)
    // pairs, tile index t*M + km, each L rows x CT columns kn = t*CT + c; col_scale is the
    // inverse-transform scale its set-up mode applies (1/L for 2-D runs, 1/(L*M) for 3-D)
    int col3d;
    double col_scale;
    double noise_amp_d;  // dt * b0 in double (0 = off)
    // set to 1 (device-visible, mapped pinned host memory) by a row-step kernel that met a
    // non-finite nonlinear term (NaN / Inf in the run's fields); the engine fails the run
    int *nonfinite;
    // per-CTA partial sums written by the analysis row kernel: [2 * L] doubles; on the
    // mixed path followed, from pair gpart_off on, by one (energy, 0) pair per spectral
    // column (km in 2-D, kn*M + km in 3-D) that the checkpoint column kernel writes: the
    // gradient term of the energy summed in k-space, times gscale = alpha / (P S^2) (S the
    // column view's inverse-transform scale)
    double *partials;
    int gpart_off;
    double gscale;
    // batched runs only: slots of (energy sum, mass sum) that launch_reduce_runs fills
    double *ehist;
    // stochastic noise (axx > 0): amplitude dt * b0 (0 = off), stream key, and the
    // device step counter the row kernel advances once per step (the column kernel of
    // step t reads t)
    float noise_amp;
    unsigned long long noise_key;
    int *step_ctr;
};

// Twiddle tables exp(-2 pi i j / n) for n = 2^1 .. 2^11, FP32 and FP64, the logarithm
// table of the mixed path's pointwise terms, and the
// context's fault word: a device-visible int in mapped pinned host memory that a
// kernel sets to nonzero when one of its bounded waits gives up (the host reads it
// after synchronising and reports PFC_E_CUDA).
constexpr int LOG_TABLE_SIZE = 129;  // breakpoints j = 0 .. 128 of log_tab
struct TwiddleSet {
    const float2 *f32[12];
    const double2 *f64[12];
    const double2 *logt;  // log_tab's table (step_common.cuh): (log F_j, 1/F_j), F_j = 1 + j/128
    int *fault;
};

// Fused step (two sweeps per step).  All runs of one call share (L, M) and the
// precision prec: PFC_PRECISION_FP32 (step_fp32.cu, FP32 arithmetic) or
// PFC_PRECISION_MIXED (step_mixed.cu, FP64 arithmetic on the same FP32 arrays).
cudaError_t launch_row_step(const RunDesc *d_runs, int nruns, int L, int M, int prec, const TwiddleSet &tw,
                            cudaStream_t s);
// C: column tile width of the runs' layout (RunDesc::CT, the same for all nruns runs);
// stage: how input tiles are staged (COL_STAGE_*; the results do not depend on it)
cudaError_t launch_col_step(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode, int prec,
                            const TwiddleSet &tw, cudaStream_t s);
cudaError_t launch_row_forward(const RunDesc *d_runs, int nruns, int L, int M, int prec, const TwiddleSet &tw,
                               cudaStream_t s);
cudaError_t launch_row_analysis(const RunDesc *d_runs, int nruns, int L, int M, int prec, const TwiddleSet &tw,
                                cudaStream_t s);
// The column kernels of one row length L (instantiated per L in col_inst.cu).
template <int L>
cudaError_t launch_col_f32_L(const RunDesc *d_runs, int nruns, int M, int C, int stage, int mode,
                             const TwiddleSet &tw, cudaStream_t s);
template <int L>
cudaError_t launch_col_mixed_L(const RunDesc *d_runs, int nruns, int tiles, int C, int stage, int mode,
                               const TwiddleSet &tw, cudaStream_t s);
// The mixed column kernel over `tiles` column tiles per run (the 3-D column view: Tn*M).
cudaError_t launch_col_step_mixed_tiles(const RunDesc *d_runs, int nruns, int L, int tiles, int C, int stage,
                                        int mode, const TwiddleSet &tw, cudaStream_t s);
// The mixed-precision row kernels of one row length M (instantiated per M in row_inst.cu).
enum MRowKind : int { MROW_STEP = 0, MROW_FORWARD = 1, MROW_ANALYSIS = 2, MROW_ANALYSIS_STEP = 3 };
template <int M>
cudaError_t launch_mrow_M(int kind, const RunDesc *d_runs, int nruns, int L, const TwiddleSet &tw, cudaStream_t s);
// The FP32 and mixed-precision kernels behind them.
cudaError_t launch_row_step_f32(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw, cudaStream_t s);
cudaError_t launch_col_step_f32(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode,
                                const TwiddleSet &tw, cudaStream_t s);
cudaError_t launch_row_forward_f32(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                   cudaStream_t s);
cudaError_t launch_row_analysis_f32(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                    cudaStream_t s);
cudaError_t launch_row_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                  cudaStream_t s);
cudaError_t launch_col_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, int C, int stage, int mode,
                                  const TwiddleSet &tw, cudaStream_t s);
cudaError_t launch_row_forward_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                     cudaStream_t s);
cudaError_t launch_row_analysis_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                      cudaStream_t s);
// The analysis followed by the next step's row work (k_mrow_analysis<M, true>): the
// energy sums of the current state, and inn/inc for the next step, whose row kernel is
// then not launched.
cudaError_t launch_row_analysis_step_mixed(const RunDesc *d_runs, int nruns, int L, int M, const TwiddleSet &tw,
                                           cudaStream_t s);

// For each of nruns runs: (sum of the analysis row kernel's nparts partial pairs) ->
// runs[i].ehist[2*slot], [2*slot+1]; the same additions in the same fixed order as the
// single-run reduction (launch_reduce_fixed), so the sums are identical.
cudaError_t launch_reduce_runs(const RunDesc *d_runs, int nruns, int nparts, int slot, cudaStream_t s);

// Build the per k-point coefficient table of one run (layout and values as RunDesc::kcoef).
cudaError_t launch_build_kcoef(const RunDesc *d_run, float2 *kden, float2 *kc2, cudaStream_t s);
// Pure-FP64 correlation kernel C2(|k|) (misfit_uniform_time_seed_fftw_early.cpp:700-750 with
// every intermediate in double): e1 * exp(-(|k| - k1)^2 / gg1) for |k| <= kc, else with 2.
struct C2ParamsD {
    double kc, e1, e2, k1, k2, gg1, gg2;
};
// The mixed-precision table of one run, from its double k-vectors: planes = four planes
// of T*L*CT doubles (kfn, kfc, kc2a, kc2b in that order; RunDesc's mixed-path fields).
cudaError_t launch_build_kmix(const RunDesc *d_run, double mn_dt, double mc_dt, double alpha, C2ParamsD a,
                              C2ParamsD b, double *planes, cudaStream_t s);

// column-kernel modes
enum ColMode : int { COL_STEP = 0, COL_PREPARE = 1, COL_STEP_CHECKPOINT = 2 };
// column-kernel tile staging: 16-byte cp.async copies, or one TMA bulk copy per tile
// completing on an mbarrier (tile_io.cuh)
enum ColStage : int { COL_STAGE_ASYNC = 0, COL_STAGE_BULK = 1 };

// The m-axis pass of a 3-D mixed-precision run (step_3d.cu).  Its n-space arrays live in
// two layouts of the same size, L*M*Hp complex floats with Hp = Tn*CT:
//   A (the row kernel's): element (l, m, kn) at ((t*L + l)*M + m)*CT + c, kn = t*CT + c,
//     so the rows of length N are the row view's L*M rows and every (t, l) is one
//     contiguous M x CT tile;
//   B (the column kernel's): element (l, km, kn) at ((t*M + km)*L + l)*CT + c, so every
//     (t, km) is one contiguous L x CT column tile.
// The forward pass transforms each (t, l) tile of an A array along m and writes it to B;
// the inverse pass reads B, transforms back (unnormalised) and writes A.
struct MPassArgs {
    const float2 *src[8];
    float2 *dst[8];
    int narr;
    int L, M, Tn, CT;
};
cudaError_t launch_mpass(const MPassArgs &a, bool forward, const TwiddleSet &tw, cudaStream_t s);
// y[i] = log_tab(x[i]) (step_common.cuh) for device arrays of n doubles.
cudaError_t launch_log_selftest(const double *x, double *y, int n, const double2 *tab, cudaStream_t s);
// The 3-D mixed-precision coefficient table in layout B (the four planes of the column
// view, fn and fc scaled by 1/(L*M)), from the double k-vectors kdl, kdm, kdn.
cudaError_t launch_build_kmix3(const RunDesc *d_col, double mn_dt, double mc_dt, double alpha, C2ParamsD a,
                               C2ParamsD b, double *planes, cudaStream_t s);
// Row lengths the mixed row kernels take: powers of two 8 ... 2048 (3-D rows of N points
// as short as 8).
bool mixed_row_len_ok(int n);

// Self-test of the column kernel's tile staging (k_stage_selftest): n float2 (even,
// <= 8192) staged from src by one bulk copy and written back to dst, or, without
// issue, a wait that runs out after limit_ns and sets *fault.
cudaError_t launch_stage_selftest(const float2 *src, float2 *dst, int n, int issue, unsigned long long limit_ns,
                                  int *fault, cudaStream_t s);

// Kernel attribute setup (before graph capture) of the row kernels of row length M.
cudaError_t prepare_rows(int M, int prec);
cudaError_t prepare_rows_f32(int M);
cudaError_t prepare_rows_mixed(int M);

// Number of partial-sum slots the analysis kernel of precision prec writes per run (2
// doubles each).
int analysis_partials(int L, int M, int prec);
int analysis_partials_f32(int L, int M);
int analysis_partials_mixed(int L, int M);
// Default column-tile width of the row-space layout for a grid with L rows, and the
// widths the autotuner may choose from (out[] holds up to 4; returns their number).
int col_tile_width(int L);
int col_tile_candidates(int L, int *out);
// The same for the mixed-precision column kernel (double2 tiles, half as long).
int mixed_col_tile_width(int L);
int mixed_col_tile_candidates(int L, int *out);

}  // namespace pfc
