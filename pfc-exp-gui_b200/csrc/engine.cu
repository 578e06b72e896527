// engine.cu -- run objects, batching and the C ABI of libpfc_b200.so.
//
// Host-side restatement of the reference's setup (model constants, k-vectors,
// correlation-kernel parameters, grain seeding) feeding the device kernels.
// Reference: src/experiment/misfit_uniform_time_seed_fftw_early.cpp:116-179 (constants,
// RecomputeDerivedParams), :455-466 (k-vectors, INITIAL_dis, C2AK/C2BK), and
// src/experiment/cvd.cpp:26-53, 351-377.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pfc_b200.h"
#include "pfc_engine.h"
#include "pfc_internal.h"

namespace pfc {

cudaError_t launch_init_misfit(float *psi, float *con, int L, int M, int N, float u0, float con0, float dx,
                               const void *grains, int ngrains, double limx, double limy, const float *costab,
                               int xmin, int ntab, float A1x2, float A2x4, cudaStream_t s);
cudaError_t launch_init_cvd(float *psi, float *con, int L, int M, int N, float u0, float con0, const float *tab,
                            float A1x2, float A2x4, cudaStream_t s);
cudaError_t launch_sum_f32(const float *a, long n, double *scratch, int blocks, double *out, cudaStream_t s);
cudaError_t launch_reduce_fixed(const double *partials, int count, int stride, int width, double *out,
                                cudaStream_t s);

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_error(cudaError_t e, const char *what) {
    return set_error(PFC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static constexpr double PI_REF = 3.1415926;  // pfc_common.h:152

// ---------------------------------------------------------------------------
// Per-device context: stream and twiddle tables.
// ---------------------------------------------------------------------------
static std::mutex g_ctx_mu;
static std::map<int, Context *> g_ctx;

// The word is cleared once it has been reported: the call that synchronised the work
// whose wait gave up returns the error, and later work on the device starts clean.
int fault_status(const Context *c) {
    if (c && c->fault && *c->fault != 0) {
        *c->fault = 0;
        return set_error(PFC_E_CUDA, "column kernel: a tile copy did not arrive within its bounded wait");
    }
    return PFC_OK;
}

int get_context(int device, Context **out) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(device);
    if (it != g_ctx.end()) {
        *out = it->second;
        return PFC_OK;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_error(PFC_E_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return set_error(PFC_E_INVALID, "device ordinal out of range");
    PFC_CUDA_TRY(cudaSetDevice(device));
    // memory freed in stream order (the analysis calls' buffers) stays in this process's
    // default pool for the next call instead of being unmapped at each synchronisation
    {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    Context *c = new Context();
    c->device = device;
    PFC_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    {
        int *f = nullptr, *fd = nullptr;
        PFC_CUDA_TRY(cudaHostAlloc(reinterpret_cast<void **>(&f), sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable));
        *f = 0;
        PFC_CUDA_TRY(cudaHostGetDevicePointer(reinterpret_cast<void **>(&fd), f, 0));
        c->fault = f;
        c->tw.fault = fd;
    }
    // twiddles for n = 2^1 .. 2^11: the FP32 tables in the stage layout of the radix-16
    // transforms (twiddle_offset, fft_core.cuh), stage (Ns, R) entry k*R + r =
    // exp(-2 pi i j / n), j = r*k*n/(Ns*R), computed in double and rounded once; the FP64
    // tables plain, entry j = exp(-2 pi i j / n) for j < n (an FP64 stage loads its base
    // factor from them and forms the powers).  Each length gets 2n entries (enough for
    // every stage table up to n = 2048; 16-byte aligned starts).
    size_t total = 0;
    for (int lg = 1; lg <= 11; ++lg) total += (size_t)2 << lg;
    std::vector<double2> h64(total, make_double2(0.0, 0.0));
    std::vector<float2> h32(total, make_float2(0.f, 0.f));
    size_t off = 0;
    for (int lg = 1; lg <= 11; ++lg) {
        const int n = 1 << lg;
        int ns = 1, rem = n;
        size_t at = off;
        while (rem > 1) {
            const int R = rem >= 16 ? 16 : rem;  // radix-16 stages first, the small radix last
            if (ns > 1) {
                for (int k = 0; k < ns; ++k)
                    for (int r = 0; r < R; ++r) {
                        const long j = (long)r * k * (n / (ns * R));
                        const double a = 2.0 * M_PI * (double)j / (double)n;
                        h32[at + (size_t)k * R + r] = make_float2((float)std::cos(a), (float)-std::sin(a));
                    }
                at += (size_t)ns * R;
            }
            ns *= R;
            rem /= R;
        }
        if (at - off > (size_t)2 * n) return set_error(PFC_E_INVALID, "twiddle table overflow");
        for (int j = 0; j < n; ++j) {
            const double a = 2.0 * M_PI * (double)j / (double)n;
            h64[off + (size_t)j] = make_double2(std::cos(a), -std::sin(a));
        }
        off += (size_t)2 * n;
    }
    // log_tab's breakpoints F_j = 1 + j/128: (log F_j, 1/F_j), each rounded once
    std::vector<double2> hlog(LOG_TABLE_SIZE);
    for (int j = 0; j < LOG_TABLE_SIZE; ++j) {
        const double F = 1.0 + j / 128.0;
        hlog[j] = make_double2(std::log(F), 1.0 / F);
    }
    const size_t tw_bytes = total * (sizeof(double2) + sizeof(float2));
    char *mem = nullptr;
    PFC_CUDA_TRY(cudaMalloc(&mem, tw_bytes + LOG_TABLE_SIZE * sizeof(double2)));
    PFC_CUDA_TRY(cudaMemcpy(mem, h64.data(), total * sizeof(double2), cudaMemcpyHostToDevice));
    PFC_CUDA_TRY(cudaMemcpy(mem + total * sizeof(double2), h32.data(), total * sizeof(float2), cudaMemcpyHostToDevice));
    PFC_CUDA_TRY(cudaMemcpy(mem + tw_bytes, hlog.data(), LOG_TABLE_SIZE * sizeof(double2), cudaMemcpyHostToDevice));
    c->tw.logt = reinterpret_cast<const double2 *>(mem + tw_bytes);
    c->tw_mem = mem;
    off = 0;
    for (int lg = 1; lg <= 11; ++lg) {
        c->tw.f64[lg] = reinterpret_cast<const double2 *>(mem) + off;
        c->tw.f32[lg] = reinterpret_cast<const float2 *>(mem + total * sizeof(double2)) + off;
        off += (size_t)2 << lg;
    }
    c->tw.f64[0] = c->tw.f64[1];
    c->tw.f32[0] = c->tw.f32[1];
    g_ctx[device] = c;
    *out = c;
    return PFC_OK;
}

// ---------------------------------------------------------------------------
// Model constants (MIS:116-143, CVD:26-53) and derived parameters.
// ---------------------------------------------------------------------------
void model_coefs(int model, ModelCoefs *k) {
    const float a_lattice = 1.0f;
    k->gaa1 = 0.8f;
    k->gaa2 = (float)(k->gaa1 * std::sqrt(2.));
    k->gab1 = 0.8f;
    k->gab2 = (float)(k->gaa2 * std::sqrt(2.));
    k->niu = 1.4f;
    k->ksi = 1.f;
    k->ka0 = (float)(2.0 * PI_REF / a_lattice);
    k->ka1 = (float)(2.0 * PI_REF);
    k->ka2 = (float)(std::sqrt(2.0) * k->ka1);
    k->sigMa1 = k->sigMa2 = k->sigMb1 = k->sigMb2 = 0.55f;
    k->para_c0 = 0.5f;
    k->para_alpha = 0.5f;
    k->para_w = 0.02f;
    if (model == MODEL_CVD) {
        const float b_lattice = (float)(std::sqrt(3.0) / 2.0);
        k->kb0 = (float)(2.5 * PI_REF / b_lattice);
        k->kb1 = (float)(5.0 * PI_REF / std::sqrt(3.0));
        k->kb2 = (float)(k->kb1 * std::sqrt(2.0));
        k->dynamic_mn = 1.f;
        k->dynamic_mc = 1.f;
    } else {
        const float b_lattice = 0.88f;
        k->kb0 = (float)(2.0 * PI_REF / b_lattice);
        k->kb1 = k->kb0;
        k->kb2 = (float)(k->kb1 * std::sqrt(2.0));
        k->dynamic_mn = 0.1f;
        k->dynamic_mc = 10.f;
    }
}

// Crossover |k| of the two Gaussian peaks, float arithmetic of MIS:702-706.
float c2_kc(float sig, float g1, float g2, float k1, float k2, float s1, float s2) {
    const float aa1 = (float)std::pow(sig / s1, 2);
    const float aa2 = (float)std::pow(sig / s2, 2);
    const float bb1 = (float)(1. / (2. * g1 * g1));
    const float bb2 = (float)(1. / (2. * g2 * g2));
    const float D = bb1 * k1 - bb2 * k2;
    const float E = aa1 - aa2 + bb1 * k1 * k1 - bb2 * k2 * k2;
    float kc = (float)(((double)D + std::sqrt(std::pow((double)D, 2) - (double)((bb1 - bb2) * E))) / (double)(bb1 - bb2));
    if (g1 == g2) kc = (aa2 - aa1 + bb1 * (k2 * k2 - k1 * k1)) / (2 * bb1 * (k2 - k1));
    return kc;
}

static C2Params c2_params(float sig, float g1, float g2, float k1, float k2, float s1, float s2) {
    C2Params p;
    p.kc = c2_kc(sig, g1, g2, k1, k2, s1, s2);
    p.e1 = (float)std::exp(-std::pow((double)(sig / s1), 2));
    p.e2 = (float)std::exp(-std::pow((double)(sig / s2), 2));
    p.k1 = k1;
    p.k2 = k2;
    p.i1 = (float)(1.0 / (double)(2 * g1 * g1));
    p.i2 = (float)(1.0 / (double)(2 * g2 * g2));
    p.q1 = sig / s1;
    p.q2 = sig / s2;
    p.gg1 = 2 * g1 * g1;
    p.gg2 = 2 * g2 * g2;
    return p;
}

// ---------------------------------------------------------------------------
// Shared per k-point coefficient tables: runs with the same model, grid, sig, dt
// and dx use one table, so a batch of such runs reads it from L2.
// ---------------------------------------------------------------------------
struct KcoefKey {
    int device, model, prec, L, M, N, CT;
    uint32_t sig, dt, dx;
    bool operator<(const KcoefKey &o) const {
        return std::tie(device, model, prec, L, M, N, CT, sig, dt, dx) <
               std::tie(o.device, o.model, o.prec, o.L, o.M, o.N, o.CT, o.sig, o.dt, o.dx);
    }
};
struct KcoefEntry {
    void *ptr = nullptr;
    int refs = 0;
};
static std::mutex g_kcoef_mu;
static std::map<KcoefKey, KcoefEntry> g_kcoef;

static uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, sizeof(u));
    return u;
}

static KcoefKey kcoef_key(const pfc_run *r) {
    return KcoefKey{r->p.device, r->p.model, r->p.precision, r->L, r->M, r->N, r->desc.CT,
                    fbits(r->p.sig), fbits(r->p.dt), fbits(r->p.dx)};
}

// Bytes per k point of the shared table: (kden, kc2) float2 pairs on the FP32 path,
// four doubles (kfn, kfc, kc2a, kc2b) on the mixed path.
static size_t kcoef_point_bytes(int prec) {
    return prec == PFC_PRECISION_MIXED ? 4 * sizeof(double) : 2 * sizeof(float2);
}

// Pure-FP64 C2 parameters (the oracle's pure mode of MIS:700-750): crossover, peak
// heights exp(-(sig/sigM)^2), peak positions and Gaussian widths 2 g^2, all in double.
static C2ParamsD c2_params_pure(float sig, float g1, float g2, float k1, float k2, float s1, float s2) {
    const double daa1 = std::pow((double)sig / s1, 2), daa2 = std::pow((double)sig / s2, 2);
    const double dbb1 = 1. / (2. * g1 * g1), dbb2 = 1. / (2. * g2 * g2);
    const double dD = dbb1 * k1 - dbb2 * k2;
    const double dE = daa1 - daa2 + dbb1 * k1 * k1 - dbb2 * k2 * k2;
    double dkc = (dD + std::sqrt(dD * dD - (dbb1 - dbb2) * dE)) / (dbb1 - dbb2);
    if (g1 == g2) dkc = (daa2 - daa1 + dbb1 * ((double)k2 * k2 - (double)k1 * k1)) / (2 * dbb1 * ((double)k2 - k1));
    const double q1 = (double)sig / s1, q2 = (double)sig / s2;
    C2ParamsD p;
    p.kc = dkc;
    p.e1 = std::exp(-q1 * q1);
    p.e2 = std::exp(-q2 * q2);
    p.k1 = k1;
    p.k2 = k2;
    p.gg1 = 2.0 * g1 * g1;
    p.gg2 = 2.0 * g2 * g2;
    return p;
}

// Table for run r (its descriptor must already be on the device); built on first use.
static int acquire_kcoef(pfc_run *r) {
    std::lock_guard<std::mutex> lk(g_kcoef_mu);
    KcoefEntry &e = g_kcoef[kcoef_key(r)];
    // points of the table: the 2-D row space, or the 3-D column view's layout B
    const size_t npts = r->d3 ? (size_t)r->desc_col.T * r->L * r->desc.CT : (size_t)r->desc.T * r->L * r->desc.CT;
    const bool mixed = r->p.precision == PFC_PRECISION_MIXED;
    if (!e.ptr) {
        const size_t bytes = npts * kcoef_point_bytes(r->p.precision);
        cudaError_t ce = cudaMalloc(&e.ptr, bytes);
        if (ce != cudaSuccess) {
            e.ptr = nullptr;
            return set_error(PFC_E_NOMEM, std::string("cudaMalloc coefficient table: ") + cudaGetErrorString(ce));
        }
        if (mixed) {
            const ModelCoefs &k = r->k;
            const C2ParamsD ca = c2_params_pure(r->p.sig, k.gaa1, k.gaa2, k.ka1, k.ka2, k.sigMa1, k.sigMa2);
            const C2ParamsD cb = c2_params_pure(r->p.sig, k.gab1, k.gab2, k.kb1, k.kb2, k.sigMb1, k.sigMb2);
            if (r->d3)
                ce = launch_build_kmix3(r->d_desc_col, (double)k.dynamic_mn * (double)r->p.dt,
                                        (double)k.dynamic_mc * (double)r->p.dt, (double)k.para_alpha, ca, cb,
                                        (double *)e.ptr, r->stream);
            else
                ce = launch_build_kmix(r->d_desc, (double)k.dynamic_mn * (double)r->p.dt,
                                       (double)k.dynamic_mc * (double)r->p.dt, (double)k.para_alpha, ca, cb,
                                       (double *)e.ptr, r->stream);
        } else {
            ce = launch_build_kcoef(r->d_desc, (float2 *)e.ptr, (float2 *)e.ptr + npts, r->stream);
        }
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(r->stream);
        if (ce != cudaSuccess) {
            cudaFree(e.ptr);
            e.ptr = nullptr;
            return cuda_error(ce, "building the coefficient table");
        }
    }
    e.refs++;
    if (mixed) {
        RunDesc &t = r->d3 ? r->desc_col : r->desc;
        const double *pl = (const double *)e.ptr;
        t.kfn = pl;
        t.kfc = pl + npts;
        t.kc2a = pl + 2 * npts;
        t.kc2b = pl + 3 * npts;
    } else {
        r->desc.kden = (const float2 *)e.ptr;
        r->desc.kc2 = (const float2 *)e.ptr + npts;
    }
    r->kcoef_held = true;
    return PFC_OK;
}

static void release_kcoef(pfc_run *r) {
    if (!r->kcoef_held) return;
    r->kcoef_held = false;
    std::lock_guard<std::mutex> lk(g_kcoef_mu);
    auto it = g_kcoef.find(kcoef_key(r));
    if (it == g_kcoef.end()) return;
    if (--it->second.refs <= 0) {
        cudaFree(it->second.ptr);
        g_kcoef.erase(it);
    }
    r->desc.kden = nullptr;
    r->desc.kc2 = nullptr;
    for (RunDesc *t : {&r->desc, &r->desc_col}) t->kfn = t->kfc = t->kc2a = t->kc2b = nullptr;
}

// k-vectors exactly as MIS:455-462 (float storage, double arithmetic).
void kref_table(int n, float dx, std::vector<float> &k) {
    k.resize(n);
    const double len = (double)((float)n * dx);
    for (int i = 0; i < n / 2 + 1; i++) k[i] = (float)((double)i * 2.0 * PI_REF / len);
    for (int i = n / 2 + 1; i < n; i++) k[i] = (float)((double)(i - n) * 2.0 * PI_REF / len);
}

static uint64_t splitmix64_next(uint64_t &state) {  // pfc_common.h:165-170
    uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static double rng_u01(uint64_t &state) {  // pfc_common.h:172-176
    return (double)(splitmix64_next(state) >> 11) * (1.0 / 9007199254740992.0);
}

bool is_supported_len(int n) { return n >= 32 && n <= 2048 && (n & (n - 1)) == 0; }

static int round_up(int x, int a) { return (x + a - 1) / a * a; }

// Key of a run's noise stream: splitmix64's output function of the base seed.
static unsigned long long noise_key(uint32_t seed) {
    uint64_t z = (uint64_t)seed + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

bool fused_path(int prec) { return prec == PFC_PRECISION_FP32 || prec == PFC_PRECISION_MIXED; }

// Bytes of a run's own device allocation with column tile width ct: 8 row-space
// arrays (fused paths) + 2 real fields + k tables (float; and double on the mixed
// path) + partials + result slots + descriptor.
static size_t run_state_bytes(int L, int M, int N, int prec, int ct) {
    const bool fused = fused_path(prec);
    const bool d3 = fused && N > 1;  // 3-D: 8 arrays in layout A and 8 in layout B
    const int Hp = d3 ? round_up(N / 2 + 1, ct) : round_up(M / 2 + 1, ct);
    const size_t rs = (size_t)(d3 ? (size_t)L * M : (size_t)L) * Hp * sizeof(float2);
    const size_t real = (size_t)L * M * N * sizeof(float);
    const size_t ktab = (size_t)(L + M + N + 1) * sizeof(float);  // k-vectors + the step counter
    const size_t kdtab = prec == PFC_PRECISION_MIXED ? (size_t)(L + M + N) * sizeof(double) : 0;
    // mixed path: one (energy, 0) pair per spectral column follows the analysis partials
    const int gtiles = prec != PFC_PRECISION_MIXED ? 0 : (d3 ? (N / 2 + 1) * M : M / 2 + 1);
    const int parts_n = gtiles + (!fused ? analysis_partials(L, M, PFC_PRECISION_FP32)
                                         : (d3 ? analysis_partials(L * M, N, prec) : analysis_partials(L, M, prec)));
    const size_t parts = (size_t)(2 * parts_n + 4096) * sizeof(double);
    // row-space arrays: psi, con, ca, cb, inn, inc, and gx, gy on the FP32 path only (the
    // mixed path sums the energy's gradient term in k-space)
    const int narr = prec == PFC_PRECISION_MIXED ? 6 : 8;
    return (fused ? (d3 ? 2 * narr : narr) * rs : 0) + 2 * real + round_up((int)ktab, 256) + round_up((int)kdtab, 256) +
           parts + 2 * sizeof(RunDesc) + 1024;
}

// Column tile width of a 3-D mixed run: the widest up to the 2-D default whose column
// tile (L x CT) and m-pass tile (M x CT) fit the kernels' shared memory; 0 if none.
static int tile_width_3d(int L, int M) {
    for (int c = mixed_col_tile_width(L); c >= 1; c /= 2) {
        int cand[4];
        const int n = mixed_col_tile_candidates(L, cand);
        bool ok = false;
        for (int i = 0; i < n; ++i) ok = ok || cand[i] == c;
        if (ok && M * c <= 4096) return c;
    }
    return 0;
}

// Column tile widths of a precision's fused kernels (default and autotuner candidates).
static int tile_default(int L, int prec) {
    return prec == PFC_PRECISION_MIXED ? mixed_col_tile_width(L) : col_tile_width(L);
}
static int tile_candidates(int L, int prec, int *out) {
    return prec == PFC_PRECISION_MIXED ? mixed_col_tile_candidates(L, out) : col_tile_candidates(L, out);
}

}  // namespace pfc

// Device bytes a run reserves: its own allocation, plus for the FP32 path the shared
// coefficient table (counted in full, as if not shared), plus for the FP64 paths the
// 22 complex-double and 6 real working arrays.
extern "C" int pfc_run_bytes(const pfc_run_params *p, double *bytes) {
    using namespace pfc;
    if (!p || !bytes) return set_error(PFC_E_INVALID, "null argument");
    if (!is_supported_len(p->L) || !is_supported_len(p->M) || p->N < 1)
        return set_error(PFC_E_INVALID, "unsupported grid");
    const bool fused = fused_path(p->precision);
    const bool d3 = fused && p->N > 1;
    // the widest tile the autotuner may choose (the most padding)
    int cand[4];
    const int nc = tile_candidates(p->L, p->precision, cand);
    int ct = nc ? cand[nc - 1] : tile_default(p->L, p->precision);
    if (d3) ct = tile_width_3d(p->L, p->M);
    if (d3 && (ct == 0 || !mixed_row_len_ok(p->N) || p->precision != PFC_PRECISION_MIXED))
        return set_error(PFC_E_INVALID, "3-D grid not taken by the fused paths");
    double b = (double)run_state_bytes(p->L, p->M, p->N, p->precision, ct);
    const double P = (double)p->L * p->M * p->N;
    if (d3) b += (double)p->L * p->M * round_up(p->N / 2 + 1, ct) * kcoef_point_bytes(p->precision);
    else if (fused) b += (double)p->L * round_up(p->M / 2 + 1, ct) * kcoef_point_bytes(p->precision);
    else b += P * (22.0 * 16.0 + 6.0 * 8.0);
    *bytes = b;
    return PFC_OK;
}

using namespace pfc;

// ---------------------------------------------------------------------------
// Run objects
// ---------------------------------------------------------------------------
struct GrainHost {
    float center_x, center_y, center_z;
    float cth;
    double cother;
};
static_assert(sizeof(GrainHost) == 24, "grain layout");

int pfc_run_init_state(pfc_run *r);

extern "C" const char *pfc_last_error(void) { return g_last_error.c_str(); }

extern "C" int pfc_default_params(int model, pfc_run_params *p) {
    if (!p) return set_error(PFC_E_INVALID, "null params");
    std::memset(p, 0, sizeof(*p));
    p->model = model;
    p->L = 256;
    p->M = 256;
    p->N = 1;
    p->seed = 20200604u;
    p->dt = 0.05f;
    p->dx = 0.125f;
    p->con0 = 0.2f;
    p->axx = 0.0f;
    p->precision = PFC_PRECISION_MIXED;
    p->device = 0;
    if (model == PFC_MODEL_CVD) {
        p->u0 = 0.01f;
        p->sig = 0.03f;
        p->grainx = p->grainy = p->grainz = 1;
    } else if (model == PFC_MODEL_MISFIT) {
        p->u0 = 0.05f;
        p->sig = 0.05f;
        p->grainx = 16;
        p->grainy = 16;
        p->grainz = 1;
    } else {
        return set_error(PFC_E_INVALID, "unknown model");
    }
    return PFC_OK;
}

static void free_run(pfc_run *r) {
    if (!r) return;
    release_kcoef(r);
    if (r->dev_mem) cudaFree(r->dev_mem);
    if (r->h_nonfinite) cudaFreeHost((void *)r->h_nonfinite);
    if (r->d_eslots) cudaFree(r->d_eslots);
    if (r->f64) fp64_destroy(r->f64);
    delete r;
}

static int tile_width_for(int device, int L, int M, int prec, int *width, int *stage);

// Create a run; ct_force > 0 fixes the column tile width of an FP32 run (the
// autotuner's trial runs), 0 takes the grid's tuned width.
static int run_create(const pfc_run_params *p, int ct_force, int stage_force, pfc_run **out) {
    if (!p || !out) return set_error(PFC_E_INVALID, "null argument");
    *out = nullptr;
    if (p->model != PFC_MODEL_MISFIT && p->model != PFC_MODEL_CVD) return set_error(PFC_E_INVALID, "unknown model");
    if (!is_supported_len(p->L) || !is_supported_len(p->M))
        return set_error(PFC_E_INVALID, "L and M must be powers of two in [32, 2048]");
    if (p->N < 1 || p->N > 2048 || (p->N & (p->N - 1)) != 0) return set_error(PFC_E_INVALID, "N must be a power of two <= 2048");
    if (p->precision != PFC_PRECISION_FP32 && p->precision != PFC_PRECISION_FP64 &&
        p->precision != PFC_PRECISION_FP64_PURE && p->precision != PFC_PRECISION_MIXED)
        return set_error(PFC_E_INVALID, "unknown precision");
    const bool fused = fused_path(p->precision);
    const bool d3 = fused && p->N != 1;
    if (d3 && p->precision != PFC_PRECISION_MIXED)
        return set_error(PFC_E_INVALID, "the FP32 path takes 2-D grids (N = 1); 3-D runs use the mixed or FP64 precisions");
    if (p->N != 1 && p->model == PFC_MODEL_MISFIT) return set_error(PFC_E_INVALID, "Misfit runs are 2-D (N = 1)");
    if (d3 && !mixed_row_len_ok(p->N))
        return set_error(PFC_E_INVALID, "3-D mixed-precision runs take N a power of two in [8, 2048]");
    if (d3 && tile_width_3d(p->L, p->M) == 0)
        return set_error(PFC_E_INVALID, "3-D grid not supported by the mixed kernels (L * M too unbalanced); use fp64");
    if (!(p->dt > 0.0f) || !(p->dx > 0.0f)) return set_error(PFC_E_INVALID, "dt and dx must be > 0");
    if (p->model == PFC_MODEL_MISFIT &&
        (p->grainx <= 0 || p->grainy <= 0 || p->grainz <= 0 || p->grainx > p->L || p->grainy > p->M || p->grainz > p->N))
        return set_error(PFC_E_INVALID, "grain counts must be in [1, grid extent]");
    if (!(p->axx >= 0.0f)) return set_error(PFC_E_INVALID, "axx must be >= 0");
    Context *ctx = nullptr;
    int rc = get_context(p->device, &ctx);
    if (rc != PFC_OK) return rc;
    PFC_CUDA_TRY(cudaSetDevice(p->device));
    int ct = tile_default(p->L, p->precision), stage = COL_STAGE_BULK;
    if (d3) {
        ct = tile_width_3d(p->L, p->M);
        stage = COL_STAGE_BULK;  // 1 % faster than cp.async at 256 x 256 x 64
    } else if (fused) {
        if (ct_force > 0) {
            ct = ct_force;
            stage = stage_force;
        } else {
            rc = tile_width_for(p->device, p->L, p->M, p->precision, &ct, &stage);
            if (rc != PFC_OK) return rc;
        }
    }

    pfc_run *r = new pfc_run();
    r->p = *p;
    r->ctx = ctx;
    r->stream = ctx->stream;
    r->L = p->L;
    r->M = p->M;
    r->N = p->N;
    r->P = (long)p->L * p->M * p->N;
    r->d3 = d3;
    r->Hp = d3 ? round_up(p->N / 2 + 1, ct) : round_up(p->M / 2 + 1, ct);
    r->rows = d3 ? p->L * p->M : p->L;
    r->rowlen = d3 ? p->N : p->M;
    model_coefs(p->model, &r->k);
    const ModelCoefs &k = r->k;
    r->c2a = c2_params(p->sig, k.gaa1, k.gaa2, k.ka1, k.ka2, k.sigMa1, k.sigMa2);
    r->c2b = c2_params(p->sig, k.gab1, k.gab2, k.kb1, k.kb2, k.sigMb1, k.sigMb2);
    kref_table(p->L, p->dx, r->krefl);
    kref_table(p->M, p->dx, r->krefm);
    kref_table(p->N, p->dx, r->krefn);
    r->b0 = (p->dx > 0.0f && p->dt > 0.0f && p->axx >= 0.0f) ? (float)std::sqrt(p->axx / p->dx / p->dx / p->dx / p->dt)
                                                              : 0.0f;

    // device memory: 8 row-space arrays + 2 real fields + k tables + partials + result
    const size_t rs = (size_t)r->rows * r->Hp * sizeof(float2);
    const size_t real = (size_t)r->P * sizeof(float);
    const int nrow = fused ? analysis_partials(r->rows, r->rowlen, p->precision)
                           : analysis_partials(r->L, r->M, PFC_PRECISION_FP32);
    // mixed path: the checkpoint column kernel's (energy, 0) pair per spectral column (the
    // energy's gradient term summed in k-space; km in 2-D, kn*M + km in 3-D, so that the
    // count and the order do not depend on the tile width) follows the analysis partials
    const int gtiles = p->precision != PFC_PRECISION_MIXED ? 0 : (d3 ? (p->N / 2 + 1) * p->M : p->M / 2 + 1);
    const int nparts = nrow + gtiles;
    r->nparts = nparts;
    const size_t ktab = (size_t)(r->L + r->M + r->N + 1) * sizeof(float);
    const size_t kdtab = p->precision == PFC_PRECISION_MIXED ? (size_t)(r->L + r->M + r->N) * sizeof(double) : 0;
    const size_t parts = (size_t)(2 * nparts + 4096) * sizeof(double);
    const size_t bytes = run_state_bytes(r->L, r->M, r->N, p->precision, ct);
    cudaError_t e = cudaMalloc(&r->dev_mem, bytes);
    if (e != cudaSuccess) {
        free_run(r);
        return set_error(PFC_E_NOMEM, std::string("cudaMalloc run state: ") + cudaGetErrorString(e));
    }
    cudaMemsetAsync(r->dev_mem, 0, bytes, r->stream);
    char *m = (char *)r->dev_mem;
    RunDesc &d = r->desc;
    std::memset(&d, 0, sizeof(d));
    RunDesc &dc = r->desc_col;
    std::memset(&dc, 0, sizeof(dc));
    if (fused) {
        // gx, gy (the last two) on the FP32 path only, as in run_state_bytes; the mixed
        // path's stay null
        const int narr = p->precision == PFC_PRECISION_MIXED ? 6 : 8;
        float2 **arrs[8] = {&d.psi, &d.con, &d.ca, &d.cb, &d.inn, &d.inc, &d.gx, &d.gy};
        for (int i = 0; i < narr; ++i) {
            *arrs[i] = (float2 *)m;
            m += rs;
        }
        if (d3) {  // the layout-B arrays of the column view
            float2 **b[8] = {&dc.psi, &dc.con, &dc.ca, &dc.cb, &dc.inn, &dc.inc, &dc.gx, &dc.gy};
            for (int i = 0; i < narr; ++i) {
                *b[i] = (float2 *)m;
                m += rs;
            }
        }
    }
    d.psi_real = (float *)m;
    m += real;
    d.con_real = (float *)m;
    m += real;
    float *kt = (float *)m;
    m += round_up((int)ktab, 256);
    d.krefl = kt;
    d.krefm = kt + r->L;
    r->d_krefn = kt + r->L + r->M;
    d.step_ctr = (int *)(kt + r->L + r->M + r->N);
    if (kdtab) {
        // pure-FP64 k-vectors (the oracle's pure mode of MIS:455-462)
        double *kd = (double *)m;
        m += round_up((int)kdtab, 256);
        // entry i = s(i) * dk, s(i) the signed index, dk = 2 pi / (n dx): the product the
        // column kernel forms for l without a load
        std::vector<double> h(r->L + r->M + r->N);
        d.dkl = 2.0 * PI_REF / ((double)r->L * p->dx);
        d.dkm = 2.0 * PI_REF / ((double)r->M * p->dx);
        d.dkn = 2.0 * PI_REF / ((double)r->N * p->dx);
        for (int l = 0; l < r->L; ++l) h[l] = (double)(l <= r->L / 2 ? l : l - r->L) * d.dkl;
        for (int mm = 0; mm < r->M; ++mm) h[r->L + mm] = (double)(mm <= r->M / 2 ? mm : mm - r->M) * d.dkm;
        for (int n = 0; n < r->N; ++n) h[r->L + r->M + n] = (double)(n <= r->N / 2 ? n : n - r->N) * d.dkn;
        r->kd_host = h;
        cudaMemcpyAsync(kd, r->kd_host.data(), kdtab, cudaMemcpyHostToDevice, r->stream);
        d.kdl = kd;
        d.kdm = kd + r->L;
        d.kdn = kd + r->L + r->M;
    }
    d.partials = (double *)m;
    d.gpart_off = nrow;
    // alpha / (P S^2): S = 1/L (2-D), 1/(L*M) (the 3-D column view)
    d.gscale = (double)r->k.para_alpha * (d3 ? (double)r->L * (double)r->M / (double)r->N : (double)r->L / (double)r->M);
    r->d_scratch = (double *)m + 2 * nparts;
    m += parts;
    r->d_desc = (RunDesc *)m;
    r->d_desc_col = r->d_desc + 1;
    cudaMemcpyAsync(kt, r->krefl.data(), r->L * sizeof(float), cudaMemcpyHostToDevice, r->stream);
    cudaMemcpyAsync(kt + r->L, r->krefm.data(), r->M * sizeof(float), cudaMemcpyHostToDevice, r->stream);
    cudaMemcpyAsync(kt + r->L + r->M, r->krefn.data(), r->N * sizeof(float), cudaMemcpyHostToDevice, r->stream);
    d.L = r->rows;  // the row view: L rows of M in 2-D, L*M rows of N in 3-D
    d.M = r->rowlen;
    d.N = d3 ? 1 : r->N;
    d.Hp = r->Hp;
    d.col_scale = 1.0 / (double)r->L;
    d.CT = ct;
    d.stage = stage;
    d.lct = 0;
    while ((1 << d.lct) < d.CT) ++d.lct;
    d.T = r->Hp / d.CT;
    d.model = p->model;
    d.dt = p->dt;
    d.k = r->k;
    d.c2a = r->c2a;
    d.c2b = r->c2b;
    // noise (MIS:490-491, 983-1014): amplitude dt * b0 in float, as the reference's product
    d.noise_amp = (p->model == PFC_MODEL_MISFIT && r->b0 != 0.0f) ? p->dt * r->b0 : 0.0f;
    d.noise_key = noise_key(p->seed);
    d.noise_amp_d = (p->model == PFC_MODEL_MISFIT && r->b0 != 0.0f) ? (double)p->dt * (double)r->b0 : 0.0;
    d.mn_dt = (double)r->k.dynamic_mn * (double)p->dt;
    d.mc_dt = (double)r->k.dynamic_mc * (double)p->dt;
    if (fused) {
        int *hf = nullptr;
        cudaError_t ce = cudaHostAlloc(reinterpret_cast<void **>(&hf), sizeof(int), cudaHostAllocMapped);
        if (ce == cudaSuccess) {
            *hf = 0;
            r->h_nonfinite = hf;
            ce = cudaHostGetDevicePointer(reinterpret_cast<void **>(&d.nonfinite), hf, 0);
        }
        if (ce != cudaSuccess) {
            free_run(r);
            return cuda_error(ce, "run status word");
        }
    }
    if (d3) {
        // the column view: layout-B arrays, (n-tile, km) tiles of L rows, 1/(L*M) scaling
        const RunDesc keep = dc;  // its layout-B array pointers
        dc = d;
        dc.psi = keep.psi;
        dc.con = keep.con;
        dc.ca = keep.ca;
        dc.cb = keep.cb;
        dc.inn = keep.inn;
        dc.inc = keep.inc;
        dc.gx = keep.gx;
        dc.gy = keep.gy;
        dc.L = r->L;
        dc.M = r->M;
        dc.N = r->N;
        dc.T = (r->Hp / ct) * r->M;
        dc.col3d = 1;
        dc.col_scale = 1.0 / ((double)r->L * (double)r->M);
    }
    if (fused) {
        cudaError_t ce = cudaMemcpyAsync(r->d_desc, &d, sizeof(RunDesc), cudaMemcpyHostToDevice, r->stream);
        if (ce == cudaSuccess && d3)
            ce = cudaMemcpyAsync(r->d_desc_col, &dc, sizeof(RunDesc), cudaMemcpyHostToDevice, r->stream);
        if (ce != cudaSuccess) {
            free_run(r);
            return cuda_error(ce, "descriptor upload");
        }
        rc = acquire_kcoef(r);
        if (rc != PFC_OK) {
            free_run(r);
            return rc;
        }
    }

    if (!fused) {
        rc = fp64_create(r);
        if (rc != PFC_OK) {
            free_run(r);
            return rc;
        }
    }
    rc = pfc_run_init_state(r);
    if (rc != PFC_OK) {
        free_run(r);
        return rc;
    }
    *out = r;
    return PFC_OK;
}

extern "C" int pfc_run_create(const pfc_run_params *p, pfc_run **out) { return run_create(p, 0, 0, out); }

// ---------------------------------------------------------------------------
// Autotuner: the column tile width of fused-path runs (FP32 or mixed precision) of an
// L x M grid, and how the column kernel stages its input tiles.  A run's row-space
// layout and its column kernel's tile both follow the width; every column's transform
// is the same arithmetic whatever the width or the staging, so the choice changes
// speed, not results.  On the first run of a grid and precision on a device, each
// candidate width (the default, a quarter, half and twice it, where the tile fits:
// col_tile_candidates, mixed_col_tile_candidates) runs a batch of Misfit runs of at
// least 8 M points in all (4 to 16 runs) with each staging method: 3 warm-up steps,
// then 8 steps of the row and column sweeps timed with CUDA events.  The fastest pair
// is kept for the rest of the process.  PFC_AUTOTUNE=0 in the environment keeps the
// default width with bulk-copy staging; pfc_set_tile_width and pfc_set_col_staging fix
// them.
// ---------------------------------------------------------------------------
struct TileChoice {
    int width = 0;
    int stage = COL_STAGE_BULK;
    int n = 0;
    int cand[4] = {0, 0, 0, 0};
    float ms[4][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};  // [candidate][staging]
    // fastest staging of a candidate width
    int best_stage(int w) const {
        for (int i = 0; i < n; ++i)
            if (cand[i] == w) return ms[i][COL_STAGE_ASYNC] < ms[i][COL_STAGE_BULK] ? COL_STAGE_ASYNC : COL_STAGE_BULK;
        return COL_STAGE_BULK;
    }
};
static std::mutex g_tile_mu;
// (device, L, M, precision) of 2-D grids; a 3-D run takes tile_width_3d(L, M) and never
// consults it
static std::map<std::tuple<int, int, int, int>, TileChoice> g_tile;

// Device time of 8 steps of a trial batch with tile width ct, for each staging method
// (ms[COL_STAGE_ASYNC], ms[COL_STAGE_BULK]).  The batch holds at least 8 M points (8 runs
// at 1024^2, 4 to 16 runs): with fewer, the wide tiles' column kernel (one CTA per SM)
// has too few items per CTA, and the trial would rank the widths differently from the
// batches it tunes for.
static int time_tile_width(int device, int L, int M, int prec, int ct, float ms[2]) {
    const long pts = (long)L * M;
    const int nruns = (int)std::max(4L, std::min(16L, (8L << 20) / pts));
    std::vector<pfc_run *> runs;
    int rc = PFC_OK;
    for (int i = 0; i < nruns && rc == PFC_OK; ++i) {
        pfc_run_params p;
        pfc_default_params(PFC_MODEL_MISFIT, &p);
        p.L = L;
        p.M = M;
        p.device = device;
        p.precision = prec;
        p.seed = 1000u + (uint32_t)i;
        pfc_run *r = nullptr;
        rc = run_create(&p, ct, COL_STAGE_BULK, &r);
        if (rc == PFC_OK) runs.push_back(r);
    }
    RunDesc *d = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == PFC_OK) {
        const int n = (int)runs.size();
        std::vector<RunDesc> h;
        for (auto *r : runs) h.push_back(r->desc);
        cudaStream_t st = runs[0]->stream;
        const TwiddleSet &tw = runs[0]->ctx->tw;
        auto step = [&](int stage) {
            cudaError_t x = launch_row_step(d, n, L, M, prec, tw, st);
            if (x == cudaSuccess) x = launch_col_step(d, n, L, M, ct, stage, COL_STEP, prec, tw, st);
            return x;
        };
        cudaError_t ce = cudaMalloc(&d, h.size() * sizeof(RunDesc));
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(d, h.data(), h.size() * sizeof(RunDesc), cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
        if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
        for (int stage = COL_STAGE_ASYNC; stage <= COL_STAGE_BULK && ce == cudaSuccess; ++stage) {
            for (int i = 0; i < 3 && ce == cudaSuccess; ++i) ce = step(stage);
            if (ce == cudaSuccess) ce = cudaEventRecord(e0, st);
            for (int i = 0; i < 8 && ce == cudaSuccess; ++i) ce = step(stage);
            if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
            if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms[stage], e0, e1);
        }
        if (ce == cudaErrorMemoryAllocation) rc = set_error(PFC_E_NOMEM, "tile width trial: out of memory");
        else if (ce != cudaSuccess) rc = cuda_error(ce, "tile width trial");
        if (rc == PFC_OK) rc = fault_status(runs[0]->ctx);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (d) cudaFree(d);
    for (auto *r : runs) pfc_run_destroy(r);
    return rc;
}

static int tile_width_for(int device, int L, int M, int prec, int *width, int *stage) {
    std::lock_guard<std::mutex> lk(g_tile_mu);
    const auto key = std::make_tuple(device, L, M, prec);
    auto it = g_tile.find(key);
    if (it != g_tile.end()) {
        *width = it->second.width;
        *stage = it->second.stage;
        return PFC_OK;
    }
    TileChoice c;
    c.width = tile_default(L, prec);
    int cand[4];
    const int nc = tile_candidates(L, prec, cand);
    const char *env = std::getenv("PFC_AUTOTUNE");
    if (!(env && env[0] == '0')) {
        float best = 0.f;
        for (int i = 0; i < nc; ++i) {
            float ms[2] = {0.f, 0.f};
            const int rc = time_tile_width(device, L, M, prec, cand[i], ms);
            if (rc == PFC_E_NOMEM) {  // no room for trial runs: keep the defaults
                c = TileChoice{};
                c.width = tile_default(L, prec);
                break;
            }
            if (rc != PFC_OK) return rc;
            c.cand[c.n] = cand[i];
            c.ms[c.n][0] = ms[0];
            c.ms[c.n++][1] = ms[1];
            for (int s = COL_STAGE_ASYNC; s <= COL_STAGE_BULK; ++s)
                if ((i == 0 && s == COL_STAGE_ASYNC) || ms[s] < best) {
                    best = ms[s];
                    c.width = cand[i];
                    c.stage = s;
                }
        }
    }
    g_tile[key] = c;
    *width = c.width;
    *stage = c.stage;
    return PFC_OK;
}

static int check_tile_args(int L, int M, int prec) {
    if (!is_supported_len(L) || !is_supported_len(M)) return set_error(PFC_E_INVALID, "unsupported grid");
    if (!fused_path(prec)) return set_error(PFC_E_INVALID, "tile widths belong to the fused (mixed, FP32) paths");
    return PFC_OK;
}

extern "C" int pfc_tile_width(int device, int L, int M, int precision, int *width, int *candidates, float *trial_ms,
                              int *ntrials) {
    if (!width) return set_error(PFC_E_INVALID, "null argument");
    int rc = check_tile_args(L, M, precision);
    if (rc != PFC_OK) return rc;
    Context *ctx = nullptr;
    rc = get_context(device, &ctx);
    if (rc != PFC_OK) return rc;
    PFC_CUDA_TRY(cudaSetDevice(device));
    int stage = 0;
    rc = tile_width_for(device, L, M, precision, width, &stage);
    if (rc != PFC_OK) return rc;
    std::lock_guard<std::mutex> lk(g_tile_mu);
    const TileChoice &c = g_tile[std::make_tuple(device, L, M, precision)];
    if (ntrials) *ntrials = c.n;
    for (int i = 0; i < c.n; ++i) {
        if (candidates) candidates[i] = c.cand[i];
        if (trial_ms) trial_ms[i] = std::min(c.ms[i][0], c.ms[i][1]);
    }
    return PFC_OK;
}

extern "C" int pfc_col_staging(int device, int L, int M, int precision, int *stage, float *ms_async, float *ms_bulk,
                               int *ntrials) {
    if (!stage) return set_error(PFC_E_INVALID, "null argument");
    int rc = check_tile_args(L, M, precision);
    if (rc != PFC_OK) return rc;
    Context *ctx = nullptr;
    rc = get_context(device, &ctx);
    if (rc != PFC_OK) return rc;
    PFC_CUDA_TRY(cudaSetDevice(device));
    int width = 0;
    rc = tile_width_for(device, L, M, precision, &width, stage);
    if (rc != PFC_OK) return rc;
    std::lock_guard<std::mutex> lk(g_tile_mu);
    const TileChoice &c = g_tile[std::make_tuple(device, L, M, precision)];
    if (ntrials) *ntrials = c.n;
    for (int i = 0; i < c.n; ++i) {
        if (ms_async) ms_async[i] = c.ms[i][COL_STAGE_ASYNC];
        if (ms_bulk) ms_bulk[i] = c.ms[i][COL_STAGE_BULK];
    }
    return PFC_OK;
}

extern "C" int pfc_set_col_staging(int device, int L, int M, int precision, int stage) {
    int rc = check_tile_args(L, M, precision);
    if (rc != PFC_OK) return rc;
    if (stage != COL_STAGE_ASYNC && stage != COL_STAGE_BULK) return set_error(PFC_E_INVALID, "unknown staging");
    std::lock_guard<std::mutex> lk(g_tile_mu);
    const auto key = std::make_tuple(device, L, M, precision);
    auto it = g_tile.find(key);
    if (it == g_tile.end()) {
        TileChoice c;
        c.width = tile_default(L, precision);
        it = g_tile.emplace(key, c).first;
    }
    it->second.stage = stage;  // a trial record, if any, is kept
    return PFC_OK;
}

extern "C" int pfc_selftest_tile_stage(int device, int issue, int n, double limit_ms, int *timed_out, int *match,
                                       double *ms) {
    if (!timed_out || !match || !ms) return set_error(PFC_E_INVALID, "null argument");
    if (n < 2 || n > 8192 || (n & 1) || !(limit_ms > 0.0) || limit_ms > 10000.0)
        return set_error(PFC_E_INVALID, "n must be even in [2, 8192] and limit_ms in (0, 10000]");
    Context *c = nullptr;
    int rc = get_context(device, &c);
    if (rc != PFC_OK) return rc;
    PFC_CUDA_TRY(cudaSetDevice(device));
    std::vector<float2> h(n), back(n, make_float2(0.f, 0.f));
    for (int i = 0; i < n; ++i) h[i] = make_float2((float)i + 0.25f, -(float)(3 * i) - 0.5f);
    float2 *d = nullptr;
    int *f = nullptr, *fd = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&d, 2 * sizeof(float2) * n);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&f), sizeof(int), cudaHostAllocMapped);
    if (e == cudaSuccess) {
        *(volatile int *)f = 0;
        e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&fd), f, 0);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + n, 0, sizeof(float2) * n, c->stream);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
    if (e == cudaSuccess)
        e = launch_stage_selftest(d, d + n, n, issue ? 1 : 0, (unsigned long long)(limit_ms * 1e6), fd, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(back.data(), d + n, sizeof(float2) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    if (e == cudaSuccess) {
        *timed_out = *(volatile int *)f != 0 ? 1 : 0;
        *match = std::memcmp(back.data(), h.data(), sizeof(float2) * n) == 0 ? 1 : 0;
        *ms = t;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (f) cudaFreeHost(f);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return cuda_error(e, "pfc_selftest_tile_stage");
    return PFC_OK;
}

extern "C" int pfc_selftest_log(int device, const double *x, double *y, int n) {
    if (!x || !y) return set_error(PFC_E_INVALID, "null argument");
    if (n < 1 || n > (1 << 24)) return set_error(PFC_E_INVALID, "n must be in [1, 2^24]");
    Context *c = nullptr;
    int rc = get_context(device, &c);
    if (rc != PFC_OK) return rc;
    PFC_CUDA_TRY(cudaSetDevice(device));
    double *d = nullptr;
    cudaError_t e = cudaMalloc(&d, 2 * sizeof(double) * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_log_selftest(d, d + n, n, c->tw.logt, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(y, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return cuda_error(e, "pfc_selftest_log");
    return PFC_OK;
}

extern "C" int pfc_set_tile_width(int device, int L, int M, int precision, int width) {
    int rc = check_tile_args(L, M, precision);
    if (rc != PFC_OK) return rc;
    int cand[4];
    const int nc = tile_candidates(L, precision, cand);
    bool ok = false;
    for (int i = 0; i < nc; ++i) ok = ok || cand[i] == width;
    if (!ok) return set_error(PFC_E_INVALID, "tile width not available for this grid");
    std::lock_guard<std::mutex> lk(g_tile_mu);
    TileChoice &c = g_tile[std::make_tuple(device, L, M, precision)];
    c.width = width;  // a trial record, if any, is kept
    c.stage = c.best_stage(width);
    return PFC_OK;
}

// Initial condition into d.psi_real / d.con_real (FP32, exact reference values).
static int init_real_fields(pfc_run *r) {
    const pfc_run_params &p = r->p;
    const ModelCoefs &k = r->k;
    RunDesc &d = r->desc;
    if (p.model == PFC_MODEL_MISFIT) {
        // INITIAL_dis (MIS:610-682)
        const int dnx = p.L / p.grainx, dny = p.M / p.grainy, dnz = p.N / p.grainz;
        std::vector<GrainHost> grains;
        for (int iii = 0; iii < p.grainx; iii++)
            for (int jjj = 0; jjj < p.grainy; jjj++)
                for (int kkk = 0; kkk < p.grainz; kkk++) {
                    GrainHost g;
                    g.center_x = (float)(dnx * iii + dnx / 2);
                    g.center_y = (float)(dny * jjj + dny / 2);
                    g.center_z = (float)(dnz * kkk + dnz / 2);
                    const unsigned int center_sum =
                        (unsigned int)((dnx * iii + dnx / 2) + (dny * jjj + dny / 2) + (dnz * kkk + dnz / 2));
                    uint64_t st = (uint64_t)(p.seed ^ (center_sum * 2654435761u));
                    const double v1 = 80.0 * (rng_u01(st) - 0.5);
                    (void)rng_u01(st);
                    const float theta = (float)(v1 * PI_REF / 180);
                    g.cth = cosf(theta);
                    g.cother = std::cos(PI_REF / 2 - (double)theta - (double)(iii + jjj + kkk) * PI_REF);
                    grains.push_back(g);
                }
        const float kk = (1 - p.con0) * k.ka0 + p.con0 * k.kb0;
        const int ext = p.L + p.M + 4;
        const int xmin = -ext, ntab = 2 * ext + 1;
        std::vector<float> costab(ntab);
        for (int i = 0; i < ntab; ++i) {
            const int X = xmin + i;
            costab[i] = cosf(kk * (float)X * p.dx);
        }
        const double limx = (double)((float)p.L * p.dx / (float)p.grainx) / 2. - 0.2;
        const double limy = (double)((float)p.M * p.dx / (float)p.grainy) / 2. - 0.2;
        const size_t gbytes = grains.size() * sizeof(GrainHost), tbytes = costab.size() * sizeof(float);
        char *tmp = nullptr;
        PFC_CUDA_TRY(cudaMalloc(&tmp, gbytes + tbytes + 256));
        PFC_CUDA_TRY(cudaMemcpyAsync(tmp, grains.data(), gbytes, cudaMemcpyHostToDevice, r->stream));
        PFC_CUDA_TRY(cudaMemcpyAsync(tmp + round_up((int)gbytes, 256), costab.data(), tbytes, cudaMemcpyHostToDevice,
                                     r->stream));
        const float A1 = 0.1427f, A2 = 0.106f;
        PFC_CUDA_TRY(launch_init_misfit(d.psi_real, d.con_real, p.L, p.M, p.N, p.u0, p.con0, p.dx, tmp,
                                        (int)grains.size(), limx, limy, (const float *)(tmp + round_up((int)gbytes, 256)),
                                        xmin, ntab, 2 * A1, 4 * A2, r->stream));
        PFC_CUDA_TRY(cudaStreamSynchronize(r->stream));
        cudaFree(tmp);
    } else {
        // INITIAL_C2 (CVD:587-642), rotation w3 = 0
        const float w3 = (float)(0. * PI_REF / 180);
        const float cw = cosf(w3), sw = sinf(w3);
        std::vector<float> tab(2 * (p.L + p.M));
        for (int pass = 0; pass < 2; ++pass) {
            const float kx = pass == 0 ? k.ka0 : k.kb0;
            float *tl = tab.data() + pass * (p.L + p.M);
            float *tm = tl + p.L;
            for (int l = 0; l < p.L; ++l) {
                const float x = (float)(0 - p.L / 2 + l) * p.dx;
                tl[l] = cosf(kx * x * cw + kx * 0.0f * sw);
            }
            for (int mm = 0; mm < p.M; ++mm) {
                const float y = (float)(mm - p.M / 2) * p.dx;
                tm[mm] = cosf(-0.0f * kx * sw + kx * y * cw);
            }
        }
        float *tmp = nullptr;
        PFC_CUDA_TRY(cudaMalloc(&tmp, tab.size() * sizeof(float)));
        PFC_CUDA_TRY(cudaMemcpyAsync(tmp, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, r->stream));
        const float A1 = 0.15f, A2 = 0.106f;
        PFC_CUDA_TRY(launch_init_cvd(d.psi_real, d.con_real, p.L, p.M, p.N, p.u0, p.con0, tmp, 2 * A1, 4 * A2, r->stream));
        PFC_CUDA_TRY(cudaStreamSynchronize(r->stream));
        cudaFree(tmp);
    }
    return PFC_OK;
}

// m-pass arguments of a 3-D run for the arrays `which` (0 psi, 1 con, 2 c2a, 3 c2b, 4 inn,
// 5 inc): forward reads layout A (the row view's arrays) and writes layout B (the column
// view's), inverse the other way.
static MPassArgs mpass_args(const pfc_run *r, std::initializer_list<int> which, bool forward) {
    const RunDesc &a = r->desc, &b = r->desc_col;
    float2 *A[6] = {a.psi, a.con, a.ca, a.cb, a.inn, a.inc};
    float2 *B[6] = {b.psi, b.con, b.ca, b.cb, b.inn, b.inc};
    MPassArgs m{};
    for (int w : which) {
        m.src[m.narr] = forward ? A[w] : B[w];
        m.dst[m.narr] = forward ? B[w] : A[w];
        ++m.narr;
    }
    m.L = r->L;
    m.M = r->M;
    m.Tn = r->Hp / r->desc.CT;
    m.CT = r->desc.CT;
    return m;
}

// Means of the real fields (FP64), then row space and the c2a/c2b arrays.
static int fp32_from_real(pfc_run *r, bool means_from_device) {
    RunDesc &d = r->desc;
    if (means_from_device) {
        const int blocks = 256;
        PFC_CUDA_TRY(launch_sum_f32(d.psi_real, r->P, r->d_scratch, blocks, r->d_scratch + blocks, r->stream));
        PFC_CUDA_TRY(launch_sum_f32(d.con_real, r->P, r->d_scratch, blocks, r->d_scratch + blocks + 1, r->stream));
        double sums[2];
        PFC_CUDA_TRY(cudaMemcpyAsync(sums, r->d_scratch + blocks, sizeof(sums), cudaMemcpyDeviceToHost, r->stream));
        PFC_CUDA_TRY(cudaStreamSynchronize(r->stream));
        r->psi_mean = sums[0] / (double)r->P;
        r->con_mean = sums[1] / (double)r->P;
    }
    d.psi_mean = r->psi_mean;
    d.con_mean = r->con_mean;
    d.psi_mean_f = (float)r->psi_mean;
    d.con_mean_f = (float)r->con_mean;
    PFC_CUDA_TRY(cudaMemcpyAsync(r->d_desc, &d, sizeof(RunDesc), cudaMemcpyHostToDevice, r->stream));
    // the row kernel of step t advances the counter to t before the column kernel reads it
    r->step_ctr_init = r->t - 1;
    PFC_CUDA_TRY(cudaMemcpyAsync(d.step_ctr, &r->step_ctr_init, sizeof(int), cudaMemcpyHostToDevice, r->stream));
    const int prec = r->p.precision;
    PFC_CUDA_TRY(launch_row_forward(r->d_desc, 1, r->rows, r->rowlen, prec, r->ctx->tw, r->stream));
    if (r->d3) {
        RunDesc &dc = r->desc_col;
        dc.psi_mean = d.psi_mean;
        dc.con_mean = d.con_mean;
        dc.psi_mean_f = d.psi_mean_f;
        dc.con_mean_f = d.con_mean_f;
        PFC_CUDA_TRY(cudaMemcpyAsync(r->d_desc_col, &dc, sizeof(RunDesc), cudaMemcpyHostToDevice, r->stream));
        // psi to layout B, c2a / c2b from it (the column kernel's set-up mode), back to layout A
        PFC_CUDA_TRY(launch_mpass(mpass_args(r, {0}, true), true, r->ctx->tw, r->stream));
        PFC_CUDA_TRY(launch_col_step_mixed_tiles(r->d_desc_col, 1, r->L, dc.T, dc.CT, dc.stage, COL_PREPARE,
                                                 r->ctx->tw, r->stream));
        PFC_CUDA_TRY(launch_mpass(mpass_args(r, {2, 3}, false), false, r->ctx->tw, r->stream));
    } else {
        PFC_CUDA_TRY(launch_col_step(r->d_desc, 1, r->L, r->M, r->desc.CT, r->desc.stage, COL_PREPARE, prec,
                                     r->ctx->tw, r->stream));
    }
    PFC_SYNC_CHECKED(r->ctx, r->stream);
    r->fields_valid = true;
    r->energy_valid = false;
    return PFC_OK;
}

int pfc_run_init_state(pfc_run *r) {
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    int rc = init_real_fields(r);
    if (rc != PFC_OK) return rc;
    r->t = 0;
    if (!fused_path(r->p.precision)) return fp64_init_from_real(r, true);
    return fp32_from_real(r, true);
}

extern "C" int pfc_run_destroy(pfc_run *r) {
    if (!r) return PFC_OK;
    cudaSetDevice(r->p.device);
    cudaStreamSynchronize(r->stream);
    free_run(r);
    return PFC_OK;
}

// nsteps fused steps; with analysis, the last ends with the checkpoint column mode and
// the analysis row kernel, whose (energy sum, mass sum) go to red_out (the run's scratch
// when null).
// row_done: the first step's row work (inn, inc) was done by the analysis that ended the
// previous call; next_row (mixed path, with analysis): the closing analysis also does the
// next step's row work, so that the next call passes row_done.
static int fused_advance(pfc_run *r, int nsteps, int analysis, double *red_out = nullptr, bool row_done = false,
                         bool next_row = false) {
    const int prec = r->p.precision;
    for (int i = 0; i < nsteps; ++i) {
        const bool last = i == nsteps - 1;
        const int mode = (last && analysis) ? COL_STEP_CHECKPOINT : COL_STEP;
        if (i > 0 || !row_done)
            PFC_CUDA_TRY(launch_row_step(r->d_desc, 1, r->rows, r->rowlen, prec, r->ctx->tw, r->stream));
        if (r->d3) {
            const RunDesc &dc = r->desc_col;
            PFC_CUDA_TRY(launch_mpass(mpass_args(r, {0, 1, 4, 5}, true), true, r->ctx->tw, r->stream));
            PFC_CUDA_TRY(launch_col_step_mixed_tiles(r->d_desc_col, 1, r->L, dc.T, dc.CT, dc.stage, mode,
                                                     r->ctx->tw, r->stream));
            // (the checkpoint mode's gradient term is a k-space sum: no gx, gy to carry back)
            PFC_CUDA_TRY(launch_mpass(mpass_args(r, {0, 1, 2, 3}, false), false, r->ctx->tw, r->stream));
        } else {
            PFC_CUDA_TRY(launch_col_step(r->d_desc, 1, r->L, r->M, r->desc.CT, r->desc.stage, mode, prec,
                                         r->ctx->tw, r->stream));
        }
    }
    r->t += nsteps;
    r->fields_valid = false;
    r->energy_valid = false;
    if (analysis) {
        if (next_row)
            PFC_CUDA_TRY(launch_row_analysis_step_mixed(r->d_desc, 1, r->rows, r->rowlen, r->ctx->tw, r->stream));
        else
            PFC_CUDA_TRY(launch_row_analysis(r->d_desc, 1, r->rows, r->rowlen, prec, r->ctx->tw, r->stream));
        PFC_CUDA_TRY(launch_reduce_fixed(r->desc.partials, r->nparts, 2, 2, red_out ? red_out : r->d_scratch,
                                         r->stream));
        r->fields_valid = true;
        r->energy_valid = true;
    }
    return PFC_OK;
}

extern "C" int pfc_run_advance(pfc_run *r, int nsteps, int analysis) {
    if (!r || nsteps < 0) return set_error(PFC_E_INVALID, "bad run or step count");
    if (nsteps == 0) return PFC_OK;
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    if (!fused_path(r->p.precision)) return fp64_advance(r, nsteps);
    return fused_advance(r, nsteps, analysis);
}

extern "C" int pfc_run_advance_energies(pfc_run *r, int nsteps, double *e_over_p, double *mass_over_p) {
    if (!r || nsteps < 0 || (nsteps > 0 && (!e_over_p || !mass_over_p)))
        return set_error(PFC_E_INVALID, "bad run, step count or output arrays");
    if (nsteps == 0) return PFC_OK;
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    if (!fused_path(r->p.precision)) {  // the FP64 path computes the energy with every step
        for (int i = 0; i < nsteps; ++i) {
            int rc = fp64_advance(r, 1);
            if (rc == PFC_OK) rc = fp64_energy(r, e_over_p + i, mass_over_p + i);
            if (rc != PFC_OK) return rc;
        }
        return PFC_OK;
    }
    if (r->eslots_cap < nsteps) {
        PFC_CUDA_TRY(cudaStreamSynchronize(r->stream));
        if (r->d_eslots) cudaFree(r->d_eslots);
        r->d_eslots = nullptr;
        r->eslots_cap = 0;
        cudaError_t e = cudaMalloc(&r->d_eslots, sizeof(double) * 2 * (size_t)nsteps);
        if (e != cudaSuccess) {
            r->d_eslots = nullptr;
            return set_error(PFC_E_NOMEM, std::string("cudaMalloc energy slots: ") + cudaGetErrorString(e));
        }
        r->eslots_cap = nsteps;
    }
    // each step as pfc_run_advance(r, 1, 1), its sums in its own slot.  On the mixed path
    // the analysis of step i (but the last) also does step i + 1's row work: the same
    // operations as the row kernel's, so the same bits, with one launch and one read of
    // the row-space arrays fewer per step.
    const bool fuse = r->p.precision == PFC_PRECISION_MIXED;
    for (int i = 0; i < nsteps; ++i) {
        const int rc = fused_advance(r, 1, 1, r->d_eslots + 2 * i, fuse && i > 0, fuse && i + 1 < nsteps);
        if (rc != PFC_OK) return rc;
    }
    PFC_CUDA_TRY(cudaMemcpyAsync(r->d_scratch, r->d_eslots + 2 * (nsteps - 1), 2 * sizeof(double),
                                 cudaMemcpyDeviceToDevice, r->stream));  // pfc_run_energy's last step
    std::vector<double> h(2 * (size_t)nsteps);
    PFC_CUDA_TRY(cudaMemcpyAsync(h.data(), r->d_eslots, h.size() * sizeof(double), cudaMemcpyDeviceToHost, r->stream));
    PFC_SYNC_CHECKED(r->ctx, r->stream);
    for (int i = 0; i < nsteps; ++i) {
        e_over_p[i] = h[2 * i] / r->L / r->M / r->N;
        mass_over_p[i] = h[2 * i + 1] / r->L / r->M / r->N;
    }
    if (*r->h_nonfinite != 0)  // the values are written all the same; the flag stays set for pfc_run_nonfinite
        return set_error(PFC_E_NONFINITE, "non-finite fields (a NaN or Inf nonlinear term)");
    return PFC_OK;
}

extern "C" int pfc_run_advance_timed(pfc_run *r, int nsteps, float *ms) {
    if (!r || !ms || nsteps < 0) return set_error(PFC_E_INVALID, "bad argument");
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    cudaEvent_t e0, e1;
    PFC_CUDA_TRY(cudaEventCreate(&e0));
    PFC_CUDA_TRY(cudaEventCreate(&e1));
    int rc = PFC_OK;
    cudaError_t e = cudaStreamSynchronize(r->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e0, r->stream);
    if (e == cudaSuccess) rc = pfc_run_advance(r, nsteps, 0);
    if (e == cudaSuccess && rc == PFC_OK) e = cudaEventRecord(e1, r->stream);
    if (e == cudaSuccess && rc == PFC_OK) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess && rc == PFC_OK) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != PFC_OK) return rc;
    if (e != cudaSuccess) return cuda_error(e, "pfc_run_advance_timed");
    return fault_status(r->ctx);
}

extern "C" int pfc_run_steps(const pfc_run *r, int *steps) {
    if (!r || !steps) return set_error(PFC_E_INVALID, "null argument");
    *steps = r->t;
    return PFC_OK;
}

// Make d.psi_real / d.con_real hold the current state.
static int materialize(pfc_run *r) {
    if (!fused_path(r->p.precision)) return fp64_materialize(r);
    if (r->fields_valid) return PFC_OK;
    PFC_CUDA_TRY(launch_row_analysis(r->d_desc, 1, r->rows, r->rowlen, r->p.precision, r->ctx->tw, r->stream));
    r->fields_valid = true;
    return PFC_OK;
}

extern "C" int pfc_run_get_fields_f32(pfc_run *r, float *phi, float *con) {
    if (!r) return set_error(PFC_E_INVALID, "null run");
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    int rc = materialize(r);
    if (rc != PFC_OK) return rc;
    if (phi) PFC_CUDA_TRY(cudaMemcpyAsync(phi, r->desc.psi_real, r->P * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    if (con) PFC_CUDA_TRY(cudaMemcpyAsync(con, r->desc.con_real, r->P * sizeof(float), cudaMemcpyDeviceToHost, r->stream));
    PFC_SYNC_CHECKED(r->ctx, r->stream);
    return PFC_OK;
}

extern "C" int pfc_run_get_fields(pfc_run *r, double *phi, double *con) {
    if (!r) return set_error(PFC_E_INVALID, "null run");
    if (!fused_path(r->p.precision)) return fp64_get_fields(r, phi, con);
    std::vector<float> a(phi ? r->P : 0), b(con ? r->P : 0);
    int rc = pfc_run_get_fields_f32(r, phi ? a.data() : nullptr, con ? b.data() : nullptr);
    if (rc != PFC_OK) return rc;
    for (long i = 0; phi && i < r->P; ++i) phi[i] = a[i];
    for (long i = 0; con && i < r->P; ++i) con[i] = b[i];
    return PFC_OK;
}

// FP64 host fields -> FP32 copies and the FP64 sums.  The fields are cut into 16 fixed
// chunks, each summed with four accumulators, and the chunk sums are added in chunk
// order, so the result does not depend on how many host threads share the chunks.
static void convert_fields(const double *phi, const double *con, long P, float *a, float *b, double &sa,
                           double &sb) {
    constexpr int CH = 16;
    double ps[CH], cs[CH];
    auto work = [&](int c) {
        const long lo = P * c / CH, hi = P * (c + 1) / CH;
        double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0, c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
        long i = lo;
        for (; i + 4 <= hi; i += 4) {
            a[i] = (float)phi[i];
            a[i + 1] = (float)phi[i + 1];
            a[i + 2] = (float)phi[i + 2];
            a[i + 3] = (float)phi[i + 3];
            b[i] = (float)con[i];
            b[i + 1] = (float)con[i + 1];
            b[i + 2] = (float)con[i + 2];
            b[i + 3] = (float)con[i + 3];
            p0 += phi[i];
            p1 += phi[i + 1];
            p2 += phi[i + 2];
            p3 += phi[i + 3];
            c0 += con[i];
            c1 += con[i + 1];
            c2 += con[i + 2];
            c3 += con[i + 3];
        }
        for (; i < hi; ++i) {
            a[i] = (float)phi[i];
            b[i] = (float)con[i];
            p0 += phi[i];
            c0 += con[i];
        }
        ps[c] = (p0 + p1) + (p2 + p3);
        cs[c] = (c0 + c1) + (c2 + c3);
    };
    const unsigned hc = std::thread::hardware_concurrency();
    const int nt = P >= (1L << 18) ? (int)std::min(8u, hc ? hc : 1u) : 1;
    if (nt <= 1) {
        for (int c = 0; c < CH; ++c) work(c);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&work, t, nt] {
                for (int c = t; c < CH; c += nt) work(c);
            });
        for (auto &x : th) x.join();
    }
    sa = 0.0;
    sb = 0.0;
    for (int c = 0; c < CH; ++c) {
        sa += ps[c];
        sb += cs[c];
    }
}

extern "C" int pfc_run_set_fields(pfc_run *r, const double *phi, const double *con) {
    if (!r || !phi || !con) return set_error(PFC_E_INVALID, "null argument");
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    if (!fused_path(r->p.precision)) return fp64_set_fields(r, phi, con);
    // converted into the context's pinned staging buffer and uploaded from there; the
    // buffer is held until fp32_from_real has synchronised the stream
    Context *ctx = r->ctx;
    std::lock_guard<std::mutex> lk(ctx->stage_mu);
    if (ctx->stage_floats < 2 * (size_t)r->P) {
        if (ctx->stage) cudaFreeHost(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_floats = 0;
        PFC_CUDA_TRY(cudaMallocHost(&ctx->stage, 2 * (size_t)r->P * sizeof(float)));
        ctx->stage_floats = 2 * (size_t)r->P;
    }
    float *a = ctx->stage, *b = ctx->stage + r->P;
    double sa = 0.0, sb = 0.0;
    convert_fields(phi, con, r->P, a, b, sa, sb);
    r->psi_mean = sa / (double)r->P;
    r->con_mean = sb / (double)r->P;
    PFC_CUDA_TRY(cudaMemcpyAsync(r->desc.psi_real, a, r->P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    PFC_CUDA_TRY(cudaMemcpyAsync(r->desc.con_real, b, r->P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    return fp32_from_real(r, false);
}

// FP32 host fields: one cudaMemcpyAsync per field straight into the run's real-field
// arrays (asynchronous when the host arrays are pinned), the FP64 means summed on the
// device, then the row-space state built as for pfc_run_set_fields.
extern "C" int pfc_run_set_fields_f32(pfc_run *r, const float *phi, const float *con) {
    if (!r || !phi || !con) return set_error(PFC_E_INVALID, "null argument");
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    if (!fused_path(r->p.precision)) {
        std::vector<double> a(phi, phi + r->P), b(con, con + r->P);
        return fp64_set_fields(r, a.data(), b.data());
    }
    PFC_CUDA_TRY(cudaMemcpyAsync(r->desc.psi_real, phi, r->P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    PFC_CUDA_TRY(cudaMemcpyAsync(r->desc.con_real, con, r->P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    return fp32_from_real(r, true);
}

extern "C" int pfc_run_energy(pfc_run *r, double *e_over_p, double *mass_over_p) {
    if (!r) return set_error(PFC_E_INVALID, "null run");
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    if (!fused_path(r->p.precision)) return fp64_energy(r, e_over_p, mass_over_p);
    if (!r->energy_valid) return set_error(PFC_E_STATE, "energy is available after pfc_run_advance(..., analysis=1)");
    double s[2];
    PFC_CUDA_TRY(cudaMemcpyAsync(s, r->d_scratch, sizeof(s), cudaMemcpyDeviceToHost, r->stream));
    PFC_SYNC_CHECKED(r->ctx, r->stream);
    if (e_over_p) *e_over_p = s[0] / r->L / r->M / r->N;
    if (mass_over_p) *mass_over_p = s[1] / r->L / r->M / r->N;
    return PFC_OK;
}

extern "C" int pfc_run_nonfinite(pfc_run *r, int *flag) {
    if (!r || !flag) return set_error(PFC_E_INVALID, "null argument");
    if (!fused_path(r->p.precision)) return set_error(PFC_E_INVALID, "the check belongs to the fused paths");
    PFC_CUDA_TRY(cudaSetDevice(r->p.device));
    PFC_SYNC_CHECKED(r->ctx, r->stream);
    *flag = *r->h_nonfinite != 0 ? 1 : 0;
    *r->h_nonfinite = 0;
    return PFC_OK;
}

extern "C" int pfc_run_means(const pfc_run *r, double *phi_mean, double *con_mean) {
    if (!r) return set_error(PFC_E_INVALID, "null run");
    if (phi_mean) *phi_mean = r->psi_mean;
    if (con_mean) *con_mean = r->con_mean;
    return PFC_OK;
}

// ---------------------------------------------------------------------------
// Batches: runs grouped by grid size, one launch per size class per sweep,
// captured once into a CUDA graph per step count.
// ---------------------------------------------------------------------------
struct SizeClass {
    int L, M, CT, stage, prec;
    std::vector<pfc_run *> runs;
    RunDesc *d_descs = nullptr;
};

struct pfc_batch {
    std::vector<SizeClass> classes;
    cudaStream_t stream = nullptr;
    int device = 0;
    Context *ctx = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
};

extern "C" int pfc_batch_create(pfc_run *const *runs, int nruns, pfc_batch **out) {
    if (!runs || nruns <= 0 || !out) return set_error(PFC_E_INVALID, "empty batch");
    *out = nullptr;
    const int dev = runs[0]->p.device;
    for (int i = 0; i < nruns; ++i) {
        if (!runs[i]) return set_error(PFC_E_INVALID, "null run in batch");
        if (!fused_path(runs[i]->p.precision) || runs[i]->d3)
            return set_error(PFC_E_INVALID, "batches hold 2-D fused-path (mixed, FP32) runs only");
        if (runs[i]->p.device != dev) return set_error(PFC_E_INVALID, "batch runs must share one device");
    }
    PFC_CUDA_TRY(cudaSetDevice(dev));
    pfc_batch *b = new pfc_batch();
    b->device = dev;
    b->ctx = runs[0]->ctx;
    b->stream = runs[0]->stream;
    for (int i = 0; i < nruns; ++i) {
        SizeClass *sc = nullptr;
        for (auto &c : b->classes)
            if (c.L == runs[i]->L && c.M == runs[i]->M && c.CT == runs[i]->desc.CT && c.stage == runs[i]->desc.stage &&
                c.prec == runs[i]->p.precision)
                sc = &c;
        if (!sc) {
            b->classes.push_back(SizeClass{runs[i]->L, runs[i]->M, runs[i]->desc.CT, runs[i]->desc.stage,
                                           runs[i]->p.precision, {}, nullptr});
            sc = &b->classes.back();
        }
        sc->runs.push_back(runs[i]);
    }
    for (auto &c : b->classes) {
        std::vector<RunDesc> h;
        for (auto *r : c.runs) h.push_back(r->desc);
        cudaError_t e = cudaMalloc(&c.d_descs, h.size() * sizeof(RunDesc));
        if (e != cudaSuccess) {
            pfc_batch_destroy(b);
            return cuda_error(e, "cudaMalloc batch descriptors");
        }
        cudaMemcpy(c.d_descs, h.data(), h.size() * sizeof(RunDesc), cudaMemcpyHostToDevice);
    }
    *out = b;
    return PFC_OK;
}

extern "C" int pfc_batch_destroy(pfc_batch *b) {
    if (!b) return PFC_OK;
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto &c : b->classes)
        if (c.d_descs) cudaFree(c.d_descs);
    delete b;
    return PFC_OK;
}

static int batch_enqueue(pfc_batch *b, int nsteps) {
    for (int i = 0; i < nsteps; ++i) {
        for (auto &c : b->classes)
            PFC_CUDA_TRY(launch_row_step(c.d_descs, (int)c.runs.size(), c.L, c.M, c.prec, b->ctx->tw, b->stream));
        for (auto &c : b->classes)
            PFC_CUDA_TRY(
                launch_col_step(c.d_descs, (int)c.runs.size(), c.L, c.M, c.CT, c.stage, COL_STEP, c.prec,
                                b->ctx->tw, b->stream));
    }
    return PFC_OK;
}

// Event-timed advance on the batch's stream: *ms = device time of the nsteps.
extern "C" int pfc_batch_advance_timed(pfc_batch *b, int nsteps, float *ms) {
    if (!b || !ms) return set_error(PFC_E_INVALID, "null argument");
    PFC_CUDA_TRY(cudaSetDevice(b->device));
    cudaEvent_t e0, e1;
    PFC_CUDA_TRY(cudaEventCreate(&e0));
    PFC_CUDA_TRY(cudaEventCreate(&e1));
    int rc = PFC_OK;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
    if (e == cudaSuccess) rc = pfc_batch_advance(b, nsteps);
    if (e == cudaSuccess && rc == PFC_OK) e = cudaEventRecord(e1, b->stream);
    if (e == cudaSuccess && rc == PFC_OK) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess && rc == PFC_OK) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != PFC_OK) return rc;
    if (e != cudaSuccess) return cuda_error(e, "pfc_batch_advance_timed");
    return fault_status(b->ctx);
}

// Per-kernel device times: reps steps, each row-kernel and column-kernel launch
// (all size classes) bracketed by events; averages in milliseconds per launch set.
extern "C" int pfc_batch_kernel_times(pfc_batch *b, int reps, double *row_ms, double *col_ms) {
    if (!b || reps <= 0 || !row_ms || !col_ms) return set_error(PFC_E_INVALID, "bad argument");
    PFC_CUDA_TRY(cudaSetDevice(b->device));
    std::vector<cudaEvent_t> ev(3 * reps);
    for (auto &x : ev) PFC_CUDA_TRY(cudaEventCreate(&x));
    PFC_CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < reps; ++i) {
        PFC_CUDA_TRY(cudaEventRecord(ev[3 * i], b->stream));
        for (auto &c : b->classes)
            PFC_CUDA_TRY(launch_row_step(c.d_descs, (int)c.runs.size(), c.L, c.M, c.prec, b->ctx->tw, b->stream));
        PFC_CUDA_TRY(cudaEventRecord(ev[3 * i + 1], b->stream));
        for (auto &c : b->classes)
            PFC_CUDA_TRY(
                launch_col_step(c.d_descs, (int)c.runs.size(), c.L, c.M, c.CT, c.stage, COL_STEP, c.prec,
                                b->ctx->tw, b->stream));
        PFC_CUDA_TRY(cudaEventRecord(ev[3 * i + 2], b->stream));
    }
    PFC_SYNC_CHECKED(b->ctx, b->stream);
    double rs = 0.0, cs = 0.0;
    for (int i = 0; i < reps; ++i) {
        float a = 0.f, c = 0.f;
        PFC_CUDA_TRY(cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]));
        PFC_CUDA_TRY(cudaEventElapsedTime(&c, ev[3 * i + 1], ev[3 * i + 2]));
        rs += a;
        cs += c;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    for (auto &c : b->classes)
        for (auto *r : c.runs) {
            r->t += reps;
            r->fields_valid = false;
            r->energy_valid = false;
        }
    *row_ms = rs / reps;
    *col_ms = cs / reps;
    return PFC_OK;
}

extern "C" int pfc_batch_advance(pfc_batch *b, int nsteps) {
    if (!b || nsteps < 0) return set_error(PFC_E_INVALID, "bad batch or step count");
    if (nsteps == 0) return PFC_OK;
    PFC_CUDA_TRY(cudaSetDevice(b->device));
    // one graph covers `chunk` steps; replay it and enqueue the remainder directly
    const int chunk = nsteps < 16 ? nsteps : 16;
    if (!b->graph || b->graph_steps != chunk) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        // kernel attribute setup (max dynamic shared memory) happens outside the capture
        for (auto &c : b->classes) PFC_CUDA_TRY(prepare_size(c.L, c.M, c.CT, c.stage, c.prec));
        int rc = PFC_OK;
        cudaGraph_t g = nullptr;
        PFC_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = batch_enqueue(b, chunk);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc != PFC_OK) return rc;
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
        b->graph_steps = chunk;
    }
    int done = 0;
    while (nsteps - done >= chunk) {
        PFC_CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
        done += chunk;
    }
    int rc = batch_enqueue(b, nsteps - done);
    if (rc != PFC_OK) return rc;
    for (auto &c : b->classes)
        for (auto *r : c.runs) {
            r->t += nsteps;
            r->fields_valid = false;
            r->energy_valid = false;
        }
    return PFC_OK;
}
