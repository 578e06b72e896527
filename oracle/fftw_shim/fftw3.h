/*
 * fftw3.h -- minimal FFTW-3 API shim (oracle / test infrastructure only).
 *
 * The reference program (zhiqing0205/PFC-Exp-GUI, the src/experiment sources) calls
 * five FFTW symbols: fftw_plan_dft_3d, fftw_execute, fftw_destroy_plan,
 * fftw_malloc and fftw_free (plans at misfit_uniform_time_seed_fftw_early.cpp:438-452,
 * cvd.cpp:334-348; the MPI wrappers in pfc_common.h:113-125 forward to
 * fftw_plan_dft_3d).  FFTW itself is not available in this environment, so this
 * header declares exactly that surface and fftw_shim.c implements it with
 * FFTW's conventions:
 *   - fftw_complex is double[2] (re, im);
 *   - FFTW_FORWARD (-1) computes out[k] = sum_j in[j] exp(-2 pi i j k / n),
 *     FFTW_BACKWARD (+1) the same with +i; neither is normalised;
 *   - the 3-D array is row-major with the last index (n2) fastest.
 *
 * This is never linked into the product library.  It exists so that the
 * unmodified reference sources and the CPU restatement in ../pfc_oracle.c can
 * be compiled and compared against each other and against the GPU engine.
 */
#ifndef PFC_ORACLE_FFTW3_SHIM_H
#define PFC_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

/* Shim extension used by the oracle: run the same transform on explicit arrays. */
void pfc_shim_dft_3d(int n0, int n1, int n2, const fftw_complex *in, fftw_complex *out, int sign);

#ifdef __cplusplus
}
#endif

#endif
