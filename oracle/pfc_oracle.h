/*
 * pfc_oracle.h -- CPU restatement of the reference's hot path (TEST INFRASTRUCTURE).
 *
 * This library is the parity oracle: tests, the smoke check and the CPU leg of
 * the benchmark call it as the checker.  It is never linked into, loaded by or
 * called from the product library (pfc-exp-gui_b200/), whose GPU path fails
 * loudly rather than fall back to anything here.
 *
 * Reference files restated (paths within zhiqing0205/PFC-Exp-GUI):
 *   MIS = src/experiment/misfit_uniform_time_seed_fftw_early.cpp
 *   CVD = src/experiment/cvd.cpp
 *   ELA = src/experiment/elastic.cpp
 *   COM = src/experiment/pfc_common.h
 *
 * Two arithmetic modes:
 *   exact = 1  reproduces the reference's mixed precision (float k-vectors, float
 *              C2A/C2B tables, float Rhat in the semi-implicit update, float cmix
 *              terms, float energy terms) operation by operation, so that with
 *              the same FFT it is bit-identical to the reference binary;
 *   exact = 0  "pure FP64": the same scheme with every intermediate in double.
 * Both modes start from the same initial fields.
 */
#ifndef PFC_ORACLE_H
#define PFC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_MODEL_MISFIT = 0, ORC_MODEL_CVD = 1 };

typedef struct orc_params {
    int model; /* ORC_MODEL_MISFIT or ORC_MODEL_CVD */
    int L, M, N;
    float u0, con0, sig, dt, dx, axx;
    int grainx, grainy, grainz;
    uint32_t seed;
    int exact; /* 1: reference-exact roundings; 0: pure FP64 */
} orc_params;

typedef struct orc_run orc_run;

/* Fill *p with the reference CLI defaults of the given model (MIS:125-143, CVD:35-53). */
void orc_default_params(int model, orc_params *p);

orc_run *orc_create(const orc_params *p);
void orc_destroy(orc_run *r);

/* Initial condition (MIS:610-682 INITIAL_dis or CVD:587-642 INITIAL_C2), k-vectors
 * (MIS:455-462) and correlation kernels (MIS:700-750, CVD:658-708). */
void orc_init(orc_run *r);

/* One time step t (MIS:475-501 or CVD:400-422). */
void orc_step(orc_run *r, int t);

/* Real parts of the fields in reference layout n + N*(m + M*l). */
void orc_get_fields(const orc_run *r, double *phi, double *con);
void orc_set_fields(orc_run *r, const double *phi, const double *con);
/* Correlation kernel tables as the reference stores them (float, MIS:700-750). */
void orc_get_c2(const orc_run *r, float *c2a, float *c2b);
/* k-vectors as the reference stores them (float, MIS:455-462). */
void orc_get_kref(const orc_run *r, float *kl, float *km, float *kn);

/* ENERGYC2 (MIS:1043-1092) on the current state: returns sum(e)/L/M/N and
 * sum(phi)/L/M/N exactly as written to energy.txt.  Uses in3 and grac from the
 * last step, as the reference does. */
void orc_energy(const orc_run *r, double *e_over_p, double *mass_over_p);

/* Misfit peak finder (MIS:3261-3556).  phi, con: double[L*M] (N=1 layout m + M*l).
 * Writes up to cap atoms as 5 doubles (x, y, z, phimax, con) in emission order and
 * returns the atom count (the file lists each atom twice).  *num_found_raw receives
 * the number of local maxima before the global-max fallback. */
int orc_phimax_misfit(const double *phi, const double *con, int L, int M, float dx, float con0,
                      double *out5, int cap, int *num_found_raw);

/* Elastic peak finder (ELA:2802-2921).  phi: double[L*M*N] (values read from a
 * Float32 VTI).  Writes up to cap atoms as 4 doubles (x, y, z, phimax); returns count. */
int orc_phimax_elastic(const double *phi, int L, int M, int N, float dx, double *out4, int cap);

/* elastic3D (ELA:3586-3729).  The reference reads an uninitialised neighbour
 * strain term when 1.3 <= r < benchel (ELA:3711-3716); the oracle defines it as 0. */
void orc_elastic3d(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                   float benchel, double *strain, uint32_t *nb);

/* cryst_order (ELA:3013-3319): per-atom q4 and q6 as written to q4q6_<kd>.txt. */
void orc_cryst_order(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                     double *q4, double *q6);

/* CVD checkpoint analysis (CVD:1067-1520).
 * orc_cvd_atoms: atompositionCFGC2's peak finder on phi (float[L*M*N], layout
 * n + N*(m + M*l)).  *phic / *phimax receive the threshold and the field maximum (the
 * first line of phimax.txt); out4 receives up to cap records (x, y, z, phi) as the
 * reference's pc_x / pc_y / pc_z / pc_phi (fractional y, z, x coordinates); returns
 * the record count (>= 1: a (-1, -1, -1, 0) record stands for "no atoms"). */
int orc_cvd_atoms(const float *phi, int L, int M, int N, float dx, float u0, float *phic, float *phimax,
                  float *out4, int cap);
/* GR (CVD:1277-1312): pair-distance histogram of the records; returns maxbin and
 * fills hist[0..maxbin) (cap entries at most). */
int orc_cvd_gr_hist(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx,
                    unsigned *hist, int cap);
/* Q6_GLO (CVD:1349-1520): per-record neighbour count nb, local Q6 ql, the global
 * Q6 *ql_global and the 30-bin histogram of the local values. */
void orc_cvd_q6(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, unsigned *nb,
                float *ql, float *ql_global, unsigned *histq);

/* Splitmix64 helpers (COM:165-181), exposed for tests. */
uint64_t orc_splitmix64_next(uint64_t *state);
double orc_rng_u01(uint64_t *state);

/* Forward / backward 3-D DFT with FFTW conventions (the shim's transform). */
void orc_dft3d(int n0, int n1, int n2, const double *in, double *out, int sign);

#ifdef __cplusplus
}
#endif

#endif
