/*
 * pfc_b200.h -- C ABI of libpfc_b200.so, the B200 (sm_100a) engine for the
 * pfc-exp-cli hot path of zhiqing0205/PFC-Exp-GUI.
 *
 * Plain C types only: pointers, sizes and status codes.  Every function returns
 * PFC_OK (0) on success or a negative PFC_E_* code, and pfc_last_error() then
 * describes the failure (thread-local).  Nothing here calls exit().
 *
 * Reference interfaces replaced (paths within zhiqing0205/PFC-Exp-GUI):
 *   src/experiment/main_cli.cpp:24-88          main() / --model dispatch
 *   src/experiment/pfc_common.h:348-350        int run_misfit/run_cvd/run_elastic(int, char**)
 *   src/experiment/misfit_uniform_time_seed_fftw_early.cpp:464-501   INITIAL_dis + one time step
 *   src/experiment/cvd.cpp:377-422             INITIAL_C2 + one time step
 *   src/experiment/misfit_uniform_time_seed_fftw_early.cpp:1043-1092 ENERGYC2
 *   src/experiment/misfit_uniform_time_seed_fftw_early.cpp:3261-3556 phimax_atmposi (Misfit)
 *   src/experiment/elastic.cpp:2802-2921       phimax_atmposi (Elastic)
 *   src/experiment/elastic.cpp:3586-3729       elastic3D
 *   src/experiment/elastic.cpp:3013-3319       cryst_order
 *   src/experiment/misfit_uniform_time_seed_fftw_early.cpp:438-452   fftw_plan_dft_3d / fftw_execute
 */
#ifndef PFC_B200_H
#define PFC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFC_OK 0
#define PFC_E_INVALID (-1)   /* bad argument or unsupported size */
#define PFC_E_CUDA (-2)      /* CUDA runtime error */
#define PFC_E_NOMEM (-3)     /* device or host allocation failed */
#define PFC_E_IO (-4)        /* file read/write failure */
#define PFC_E_STATE (-5)     /* call not valid in the object's current state */
#define PFC_E_NONFINITE (-6) /* a run's fields became non-finite (NaN or Inf) */

#define PFC_MODEL_MISFIT 0
#define PFC_MODEL_CVD 1

#define PFC_PRECISION_FP32 0 /* fused path in FP32 arithmetic, FP64 k=0 mode and reductions */
#define PFC_PRECISION_FP64 1 /* plain FP64 path with the reference's float roundings */
#define PFC_PRECISION_FP64_PURE 2 /* plain FP64 path, every intermediate in double */
#define PFC_PRECISION_MIXED 3 /* fused path: the FP32 path's FP32 complex arrays in HBM, FP64
                                 arithmetic and the pure-FP64 operator in the kernels (Misfit
                                 within 1e-5 of pure FP64 after 200 steps; CVD amplifies the FP32
                                 storage roundings, and PFC_PRECISION_FP64 follows the reference's
                                 own trajectory); the default */

/* Parameters of one run.  Field meanings and defaults follow the reference CLI
 * (misfit_uniform_time_seed_fftw_early.cpp:17-35, 125-143; cvd.cpp:111-125, 33-53). */
typedef struct pfc_run_params {
    int model;      /* PFC_MODEL_MISFIT or PFC_MODEL_CVD */
    int L, M, N;    /* grid; L, M powers of two in [32, 2048]; N = 1 (2-D), or for 3-D CVD
                       runs a power of two: 8 <= N <= 2048 on the mixed path, N <= 2048 on
                       the FP64 paths (the FP32 path takes 2-D grids only) */
    float u0, con0, sig, dt, dx, axx;
    int grainx, grainy, grainz; /* Misfit initial grains */
    uint32_t seed;
    int precision;  /* PFC_PRECISION_MIXED, _FP32, _FP64 or _FP64_PURE */
    int device;     /* CUDA device ordinal */
} pfc_run_params;

typedef struct pfc_run pfc_run;
typedef struct pfc_batch pfc_batch;

/* Last error message of the calling thread ("" if none). */
const char *pfc_last_error(void);

/* Fill *p with the reference defaults of `model` (grid 256 x 256 x 1, mixed precision). */
int pfc_default_params(int model, pfc_run_params *p);

/* Allocate a run on the device and set its initial condition (INITIAL_dis for
 * Misfit, MIS:610-682; INITIAL_C2 for CVD, CVD:587-642). */
int pfc_run_create(const pfc_run_params *p, pfc_run **out);
int pfc_run_destroy(pfc_run *r);

/* Advance nsteps time steps (MIS:475-501 / CVD:389-422).  With analysis != 0 the
 * last step also prepares the checkpoint analysis (real fields, energy, mass). */
int pfc_run_advance(pfc_run *r, int nsteps, int analysis);

/* pfc_run_advance(r, nsteps, 0) bracketed by CUDA events on the run's stream;
 * *ms receives the device time.  (Measurement hook; no reference counterpart.) */
int pfc_run_advance_timed(pfc_run *r, int nsteps, float *ms);

/* Column tile width (packed columns per column-kernel tile, 1..16) that fused-path
 * runs (precision PFC_PRECISION_MIXED or PFC_PRECISION_FP32) of an L x M grid use on
 * `device`.  The first run of a grid and precision times each candidate width with
 * each tile staging method (a batch of Misfit runs, row and column sweeps, CUDA
 * events) and keeps the fastest pair for the process; neither changes the results of
 * a step, only its speed.  This call tunes the grid if it has not been tuned, returns
 * the width and, when the pointers are not NULL, the candidates (up to 4) and their
 * trial times (ms per 8 steps, the faster staging; *ntrials is 0 when no trial ran).
 * PFC_AUTOTUNE=0 in the environment keeps the default widths with bulk staging.
 * (Autotuner of the batched FFT sweeps; the reference uses FFTW and has no
 * counterpart.) */
int pfc_tile_width(int device, int L, int M, int precision, int *width, int *candidates, float *trial_ms,
                   int *ntrials);
/* Fix the tile width of a grid and precision for the rest of the process (one of the
 * candidates; the staging becomes the faster one of that width's trial, bulk without
 * one); runs created before keep their own. */
int pfc_set_tile_width(int device, int L, int M, int precision, int width);

#define PFC_STAGE_ASYNC 0 /* column kernel stages tiles by 16-byte cp.async copies */
#define PFC_STAGE_BULK 1  /* ... by one TMA bulk copy per tile, completing on an mbarrier */
/* Tile staging method (PFC_STAGE_*) that fused-path runs of an L x M grid and
 * precision use, tuning the grid first if needed; when not NULL, ms_async / ms_bulk
 * receive each candidate width's trial time with either method (order of
 * pfc_tile_width's candidates). */
int pfc_col_staging(int device, int L, int M, int precision, int *stage, float *ms_async, float *ms_bulk,
                    int *ntrials);
/* Fix the staging method of a grid and precision for the rest of the process; runs
 * created before keep their own. */
int pfc_set_col_staging(int device, int L, int M, int precision, int stage);

/* Self-test of the column kernel's tile staging on one device (not a reference
 * interface; the reference has no device code).  With issue = 1, n complex floats
 * (even, 2..8192) are staged into shared memory by one TMA bulk copy, waited for on
 * an mbarrier and written back; *match = 1 when they came back unchanged.  With
 * issue = 0 no copy is started, so the bounded wait runs out after limit_ms and the
 * kernel reports it (*timed_out = 1) and returns; the device stays usable.  *ms is
 * the kernel's device time.  Uses its own fault word, not the device's. */
int pfc_selftest_tile_stage(int device, int issue, int n, double limit_ms, int *timed_out, int *match, double *ms);

/* Self-test of the mixed path's double-precision logarithm (the table-driven log of its
 * pointwise terms): y[i] = that log of x[i] for n host doubles (1 <= n <= 2^24),
 * evaluated on the device. */
int pfc_selftest_log(int device, const double *x, double *y, int n);

/* Steps taken so far. */
int pfc_run_steps(const pfc_run *r, int *steps);

/* Real fields of the current state in the reference layout n + N*(m + M*l)
 * (double, P = L*M*N each); either pointer may be NULL. */
int pfc_run_get_fields(pfc_run *r, double *phi, double *con);
/* Same, as the FP32 values the checkpoint writer stores. */
int pfc_run_get_fields_f32(pfc_run *r, float *phi, float *con);
/* Replace the state with the given real fields (double, reference layout). */
int pfc_run_set_fields(pfc_run *r, const double *phi, const double *con);
/* Same from FP32 fields (the values a VTI checkpoint holds): copied to the device as
 * they are (asynchronously from pinned host memory), the means summed on the device.
 * Returns when the new state is in place. */
int pfc_run_set_fields_f32(pfc_run *r, const float *phi, const float *con);

/* ENERGYC2 of the current state: sum(e)/L/M/N and sum(phi)/L/M/N as written to
 * energy.txt (MIS:1081-1085).  Valid after pfc_run_advance(..., analysis=1). */
int pfc_run_energy(pfc_run *r, double *e_over_p, double *mass_over_p);

/* n time steps, each followed by the energy analysis, as n calls of
 * pfc_run_advance(r, 1, 1) + pfc_run_energy (the same kernels and values); the n
 * energies and masses (e_over_p[i], mass_over_p[i] after step i + 1) come back with one
 * synchronisation.  CVD writes ENERGYC2 of every step to energy.txt (CVD:442, 979-1039).
 * Returns PFC_E_NONFINITE, with the arrays written all the same, when the run's
 * non-finite flag is set (see pfc_run_nonfinite; the flag stays set). */
int pfc_run_advance_energies(pfc_run *r, int n, double *e_over_p, double *mass_over_p);

/* Whether a fused-path (mixed or FP32) run has met a non-finite nonlinear term since it
 * was created or since the last call (*flag = 1: its fields hold NaN or Inf).  Waits for
 * the run's queued steps.  The engine fails such a run alone (PFC_EV_FAILED with
 * PFC_E_NONFINITE) and keeps the others running.  (No reference counterpart: the
 * reference keeps stepping and writes the NaN fields.) */
int pfc_run_nonfinite(pfc_run *r, int *flag);

/* FP64 k = 0 modes of phi and con divided by P (the conserved means). */
int pfc_run_means(const pfc_run *r, double *phi_mean, double *con_mean);

/* Batched execution: runs of any of the supported grid sizes advanced together
 * (one launch per size class and precision per sweep).  Runs must be on the fused
 * paths (mixed or FP32) and on one device; the batch does not own them. */
int pfc_batch_create(pfc_run *const *runs, int nruns, pfc_batch **out);
int pfc_batch_destroy(pfc_batch *b);
/* Advance every run of the batch by nsteps (captured once into a CUDA graph). */
int pfc_batch_advance(pfc_batch *b, int nsteps);

/* Same as pfc_batch_advance, bracketed by CUDA events on the batch's stream;
 * *ms receives the device time of the nsteps.  (Measurement hook; no reference
 * counterpart.) */
int pfc_batch_advance_timed(pfc_batch *b, int nsteps, float *ms);

/* Advance reps steps with each sweep's kernels launched individually and timed
 * with CUDA events; *row_ms and *col_ms receive the mean device time of the row
 * and column kernel launches of one step.  (Measurement hook; no reference
 * counterpart.) */
int pfc_batch_kernel_times(pfc_batch *b, int reps, double *row_ms, double *col_ms);

/* Misfit peak finder (MIS:3261-3556) on a 2-D field (N = 1, layout m + M*l).
 * Writes up to cap atoms as 5 doubles (x, y, z, phimax, con) in the reference's
 * emission order; *count receives the number of atoms (the global-maximum
 * fallback counts as one). */
int pfc_phimax_misfit(const float *phi, const float *con, int L, int M, float dx, float con0, double *out5, int cap,
                      int *count);

/* Allocation-free variant of pfc_phimax_misfit, with no counterpart in the
 * reference.  It is for callers that cannot allocate device memory: a serving loop
 * whose admission controller has already committed the whole HBM budget to
 * resident runs, or a host thread that must not trigger the device-wide
 * synchronisation that cudaMalloc and cudaFree imply while other streams run.
 *
 * The caller passes DEVICE buffers: d_phi and d_con (float[L*M], layout m + M*l)
 * and d_out5 (cap x 5 doubles, the same records as pfc_phimax_misfit).  The
 * compaction scratch is a fixed array inside the library (about 32 KB on every GPU
 * that loads it, held until exit).  L*M must not exceed 4194304 (2048 x 2048);
 * larger fields are rejected with PFC_E_INVALID.  The function calls no cudaMalloc,
 * cudaFree or other allocating routine.  It runs on `stream` (a cudaStream_t;
 * NULL = the default stream), waits for that stream to finish, and returns after the
 * atoms are written and *count is set.  *count is the number of atoms found, which
 * may exceed cap; only the first cap records are written.
 *
 * Every call synchronises `stream` (it reads the atom count back to the host), so
 * it cannot be part of a CUDA graph: never call it while `stream`, or the legacy
 * default stream, is being captured.  All calls on a device share the scratch
 * array, so calls that overlap on the GPU (from several host threads or streams)
 * race: serialise them. */
int pfc_phimax_misfit_noalloc(const float *d_phi, const float *d_con, int L, int M, float dx, float con0,
                              double *d_out5, int cap, int *count, void *stream);

/* Elastic peak finder (ELA:2802-2921) on a field read from a VTI (layout
 * n + N*(m + M*l)); writes up to cap atoms as 4 doubles (x, y, z, phimax). */
int pfc_phimax_elastic(const float *phi, int L, int M, int N, float dx, double *out4, int cap, int *count);

/* elastic3D (ELA:3586-3729): per-atom strain magnitude and neighbour count
 * (0.7 < r < benchel, first 16 neighbours in ascending index contribute). */
int pfc_elastic3d(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                  float benchel, double *strain, uint32_t *nb);

/* cryst_order (ELA:3013-3319): per-atom q4 and q6 as written to q4q6_<kd>.txt. */
int pfc_cryst_order(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                    double *q4, double *q6);

/* CVD checkpoint analysis, atompositionCFGC2 (CVD:1067-1275): the peak finder on phi
 * (float[L*M*N], layout n + N*(m + M*l)).  Writes up to cap records (x, y, z, phi) as
 * the reference's pc_x / pc_y / pc_z / pc_phi (fractional y, z and x positions); a
 * field without atoms gives the one record (-1, -1, -1, 0) as in the reference.
 * *phic and *phimax receive the threshold u0 + (max - u0) * 0.618 and the maximum. */
int pfc_cvd_atoms(const float *phi, int L, int M, int N, float dx, float u0, float *out4, int cap, int *count,
                  float *phic, float *phimax);
/* GR (CVD:1277-1347): pair-distance histogram of n records (the x, y, z columns of
 * pfc_cvd_atoms); *maxbin receives its length, hist must hold cap >= maxbin entries. */
int pfc_cvd_gr_hist(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx,
                    uint32_t *hist, int cap, int *maxbin);
/* Q6_GLO (CVD:1349-1520): per-record neighbour counts and local Q6, and the global Q6. */
int pfc_cvd_q6(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, uint32_t *nb,
               float *ql, float *ql_global);

/* 3-D complex-double DFT with FFTW's conventions (row-major, n2 fastest,
 * sign -1 = forward exp(-2 pi i jk/n), +1 = backward, unnormalised): the transform
 * the reference obtains from fftw_plan_dft_3d + fftw_execute (MIS:438-452).
 * in/out: host arrays of n0*n1*n2 interleaved (re, im) doubles. */
int pfc_dft3d(const double *in, double *out, int n0, int n1, int n2, int sign);

/* The pfc-exp-cli process interface (main_cli.cpp:24-88): same flags, files,
 * progress lines and exit codes, plus the additive --grid LxMxN and
 * --precision fp32|fp64 options.  Returns the process exit code. */
int pfc_run_cli(int argc, char **argv);

/* ------------------------------------------------------------------------------
 * Engine: many Misfit / CVD runs and Elastic analyses on one GPU, submitted and
 * polled from any thread.  It replaces the GUI's one-process-per-run queue
 * (src/gui/MainWindow.cpp:3453-3522 starts pfc-exp-cli once per parameter set) and
 * has no direct counterpart in the reference.  Runs whose memory fits the HBM
 * budget are admitted in submission order and advanced together (continuous
 * batching: runs join and leave between scheduling quanta); each run's kernels
 * and results are the same as when it runs alone.  Checkpoint files (the same
 * files and formats as pfc-exp-cli) are written by an engine-owned writer thread.
 * ------------------------------------------------------------------------------ */
typedef struct pfc_engine pfc_engine;

#define PFC_JOB_MISFIT 0  /* same values as PFC_MODEL_* */
#define PFC_JOB_CVD 1
#define PFC_JOB_ELASTIC 2

#define PFC_EV_ADMITTED 1   /* job's memory reserved, run created */
#define PFC_EV_CHECKPOINT 2 /* a checkpoint's results are available (its files are written) */
#define PFC_EV_DONE 3       /* job finished; its files are written */
#define PFC_EV_FAILED 4     /* job failed; status holds the PFC_E_* code */
#define PFC_EV_CANCELLED 5

typedef struct pfc_engine_opts {
    int device;               /* CUDA device ordinal */
    double hbm_budget_bytes;  /* device memory the engine may commit to runs; <= 0: 150e9,
                                 capped by the memory free when the engine starts */
    int max_active;           /* most runs resident at once; <= 0: no limit */
    int quantum_steps;        /* most steps between scheduling decisions; <= 0: 64 */
} pfc_engine_opts;

typedef struct pfc_job {
    int kind;                 /* PFC_JOB_MISFIT, PFC_JOB_CVD or PFC_JOB_ELASTIC */
    pfc_run_params params;    /* Misfit / CVD: the run (precision must be FP32, N = 1);
                                 Elastic: dx is the lattice spacing, L/M/N unused */
    int steps;                /* Misfit / CVD: time steps (> 0) */
    int mod;                  /* checkpoint interval as in --mod (> 0) */
    const char *outdir;       /* NULL: no files; else the directory pfc-exp-cli --outdir
                                 would write (created if missing) */
    /* Elastic only: the fields to analyse are either the final state of an earlier
     * job (source_job != 0; the analysis waits until that job is done) or every
     * phi/con checkpoint pair found in input_dir (as pfc-exp-cli --model elastic). */
    uint64_t source_job;
    const char *input_dir;
    float benchel;            /* Elastic neighbour cutoff (--benchel; <= 0: 1.7) */
} pfc_job;

typedef struct pfc_event {
    uint64_t job;             /* id returned by pfc_submit */
    int type;                 /* PFC_EV_* */
    int status;               /* PFC_OK or a PFC_E_* code */
    int step;                 /* checkpoint step (kd), or the job's steps when done */
    int atoms;                /* Misfit / Elastic: atoms found at this checkpoint */
    double energy, mass;      /* energy.txt values of this checkpoint (e/P, sum(phi)/P) */
    double t_submit, t_admit, t_event; /* seconds on the engine's clock */
    double t_finish;          /* DONE / FAILED / CANCELLED: when the job left the GPU and
                                 its memory was returned (its files are written after
                                 that, before the event is posted) */
} pfc_event;

/* Start an engine (its scheduler and writer threads) on opts->device (NULL: defaults). */
int pfc_engine_create(const pfc_engine_opts *opts, pfc_engine **out);
/* Cancel queued and running jobs, finish writing files, join the threads and free
 * all device memory. */
int pfc_engine_destroy(pfc_engine *e);
/* Queue a job; *id receives its id (never 0).  The job's strings are copied. */
int pfc_submit(pfc_engine *e, const pfc_job *job, uint64_t *id);
/* Queue n jobs at once, in order (a whole sweep: the scheduler sees them together and
 * admits as many as fit in one pass); ids[i] receives job i's id.  All or nothing: if
 * any job is invalid, none is queued and the error names its index.  An Elastic job
 * may name an earlier job of the same call as its source. */
int pfc_submit_many(pfc_engine *e, const pfc_job *jobs, int n, uint64_t *ids);
/* Copy up to max pending events into ev (oldest first) without waiting; *n
 * receives the number copied. */
int pfc_poll(pfc_engine *e, pfc_event *ev, int max, int *n);
/* Same, waiting up to timeout_ms (< 0: forever) for at least one event. */
int pfc_wait(pfc_engine *e, pfc_event *ev, int max, int *n, int timeout_ms);
/* Cancel a queued or running job (a PFC_EV_CANCELLED event follows). */
int pfc_cancel(pfc_engine *e, uint64_t id);
/* Final real fields of a finished Misfit / CVD job (P floats each, layout
 * m + M*l); either pointer may be NULL.  Kept until pfc_release. */
int pfc_job_fields(pfc_engine *e, uint64_t id, float *phi, float *con);
/* Forget a finished job's kept fields. */
int pfc_release(pfc_engine *e, uint64_t id);
/* Device bytes a Misfit / CVD run with these parameters reserves. */
int pfc_run_bytes(const pfc_run_params *p, double *bytes);

#ifdef __cplusplus
}
#endif

#endif
