// pfc_engine.h -- host-side run object shared by engine.cu, step_fp64.cu and cli.cpp.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "pfc_b200.h"
#include "pfc_internal.h"

namespace pfc {
struct Fp64State;

// Per-device context: one non-blocking stream and the twiddle tables.
struct Context {
    int device = -1;
    cudaStream_t stream = nullptr;
    TwiddleSet tw{};
    void *tw_mem = nullptr;
    // pinned host staging for field uploads (pfc_run_set_fields), grown on demand
    std::mutex stage_mu;
    float *stage = nullptr;
    size_t stage_floats = 0;
    // host view of tw.fault (mapped pinned memory): set by a kernel whose bounded wait
    // gave up, cleared by fault_status when it reports the error
    volatile int *fault = nullptr;
};

int set_error(int code, const std::string &msg);
int cuda_error(cudaError_t e, const char *what);

// return the PFC_E_CUDA status of a failed CUDA call from the enclosing function
#define PFC_CUDA_TRY(expr)                                          \
    do {                                                            \
        cudaError_t _e = (expr);                                    \
        if (_e != cudaSuccess) return pfc::cuda_error(_e, #expr);   \
    } while (0)
// PFC_OK, or PFC_E_CUDA when a kernel of the context has set its fault word (read
// after the context's work has been synchronised; the word is then cleared)
int fault_status(const Context *c);
// synchronise a stream, then report a CUDA error or the context's fault word
#define PFC_SYNC_CHECKED(ctx, stream)                                          \
    do {                                                                       \
        PFC_CUDA_TRY(cudaStreamSynchronize(stream));                           \
        const int _rc = pfc::fault_status(ctx);                                \
        if (_rc != PFC_OK) return _rc;                                         \
    } while (0)
int get_context(int device, Context **out);
void model_coefs(int model, ModelCoefs *k);
void kref_table(int n, float dx, std::vector<float> &k);
float c2_kc(float sig, float g1, float g2, float k1, float k2, float s1, float s2);
bool is_supported_len(int n);
// PFC_PRECISION_FP32 or PFC_PRECISION_MIXED: the fused two-sweep kernels
bool fused_path(int prec);
}  // namespace pfc

struct pfc_run {
    pfc_run_params p;
    pfc::Context *ctx = nullptr;
    cudaStream_t stream = nullptr;
    int L = 0, M = 0, N = 0, Hp = 0;
    long P = 0;
    int nparts = 0;
    pfc::ModelCoefs k;
    pfc::C2Params c2a, c2b;
    std::vector<float> krefl, krefm, krefn;
    float b0 = 0.0f;
    void *dev_mem = nullptr;
    pfc::RunDesc desc;
    pfc::RunDesc *d_desc = nullptr;
    float *d_krefn = nullptr;
    double *d_scratch = nullptr;
    // pfc_run_advance_energies: per-step (energy sum, mass sum) slots on the device
    double *d_eslots = nullptr;
    int eslots_cap = 0;
    double psi_mean = 0.0, con_mean = 0.0;
    int t = 0;
    int step_ctr_init = -1;  // host staging of the device step counter
    bool fields_valid = false;
    bool energy_valid = false;
    pfc::Fp64State *f64 = nullptr;
    bool kcoef_held = false;        // holds a reference on the shared coefficient table
    // 3-D mixed-precision runs (d3): desc / d_desc are the row view (L*M rows of length N,
    // layout A), desc_col / d_desc_col the column view (layout B, Tn*M column tiles)
    bool d3 = false;
    int rows = 0, rowlen = 0;       // row view of the fused kernels: (L, M) in 2-D, (L*M, N) in 3-D
    pfc::RunDesc desc_col{};
    pfc::RunDesc *d_desc_col = nullptr;
    volatile int *h_nonfinite = nullptr;  // fused paths: host view of RunDesc::nonfinite (mapped pinned)
    std::vector<double> kd_host;    // mixed path: the double k-vectors (lengths L and M)
};

namespace pfc {
// Plain FP64 path (step_fp64.cu).
int fp64_create(pfc_run *r);
void fp64_destroy(Fp64State *s);
int fp64_init_from_real(pfc_run *r, bool from_device_real);
int fp64_advance(pfc_run *r, int nsteps);
int fp64_materialize(pfc_run *r);
int fp64_get_fields(pfc_run *r, double *phi, double *con);
int fp64_set_fields(pfc_run *r, const double *phi, const double *con);
int fp64_energy(pfc_run *r, double *e_over_p, double *mass_over_p);
// Kernel attribute setup for one grid size and precision (must precede graph capture).
cudaError_t prepare_size(int L, int M, int C, int stage, int prec);
}  // namespace pfc
