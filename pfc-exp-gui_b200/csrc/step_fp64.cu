// step_fp64.cu -- plain FP64 path: the reference step operation by operation on the GPU.
//
// One kernel per reference routine and one 3-D complex-double DFT per fftw_execute,
// in the order of src/experiment/misfit_uniform_time_seed_fftw_early.cpp:479-501
// (Misfit) and src/experiment/cvd.cpp:400-422 (CVD), with the reference's float
// locals (Rhat, cmix, k-vectors, C2 tables, energy terms) rounded exactly where the
// reference rounds them.  Compiled with --fmad=false so that no multiply-add is
// contracted.  This is the FP64 oracle on the device and the "plain FP64" baseline
// the fused FP32 path is measured against; it is not tuned beyond coalesced access.
//
// The noise term (Gauss + p5, MIS:490-491) is omitted when b0 == 0: it is then a
// signed zero.  With axx > 0 (Misfit) the reference's own sequential generator runs on
// the host each step (gauss_host: polar Box-Muller on one splitmix64 stream per step,
// MIS:951-981), so the noise field is the reference's value for value; it is uploaded,
// transformed (p5) and added in the update as MAINEQUATIONC2_NOI does (MIS:983-1014).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "fft_core.cuh"
#include "pfc_engine.h"

namespace pfc {

struct Fp64State {
    double2 *phi, *con, *phiHat, *conHat, *in1, *in2, *in3, *inn, *inc, *outn, *outc;
    double2 *c2adenp, *c2bdenp, *c2aden, *c2bden, *gra1, *gra2, *gra3, *grao1, *grao2, *grao3, *grac;
    float *C2AHat, *C2BHat;     // reference-exact tables (float, MIS:425-427)
    double *C2Ad, *C2Bd;        // pure-FP64 tables
    double *kd;                 // pure-FP64 k-vectors, lengths L, M, N
    double *partials;           // energy partial sums
    double2 *nois, *noisf;      // noise field and its transform (Misfit with b0 != 0)
    std::vector<float> host_noise;
    int exact;                  // 1: reference float roundings, 0: pure FP64
    void *mem;
};

static constexpr double PI_REF = 3.1415926;
static constexpr int EBLOCKS = 512;

// ---------------------------------------------------------------------------
// Generic axis FFT: length-N transforms along one axis of a complex-double array.
// Sequence q: contiguous axis -> data[q*N + e]; strided axis with stride S ->
// data[(q/S)*N*S + e*S + q%S].  NB sequences per CTA, 16 values per thread.
// ---------------------------------------------------------------------------
template <int N> struct AxisCfg {
    static constexpr int NB = (4096 / N) > 64 ? 64 : (4096 / N);
    static constexpr int NT = (NB * N / 16) < 32 ? 32 : ((NB * N / 16) > 256 ? 256 : NB * N / 16);
};

template <int N, bool FWD>
__global__ void __launch_bounds__(AxisCfg<N>::NT) k_fft_axis(double2 *__restrict__ data, long stride, long nseq,
                                                              const double2 *__restrict__ tw) {
    constexpr int NB = AxisCfg<N>::NB, NT = AxisCfg<N>::NT;
    extern __shared__ double2 sd[];
    const long q0 = (long)blockIdx.x * NB;
    if (stride == 1) {
        for (int idx = threadIdx.x; idx < NB * N; idx += NT) {
            const int b = idx / N, e = idx % N;
            const long q = q0 + b;
            sd[spad(e * NB + b)] = q < nseq ? data[q * N + e] : make_double2(0.0, 0.0);
        }
    } else {
        for (int idx = threadIdx.x; idx < NB * N; idx += NT) {
            const int b = idx % NB, e = idx / NB;
            const long q = q0 + b;
            sd[spad(idx)] = q < nseq ? data[(q / stride) * N * stride + (long)e * stride + q % stride] : make_double2(0.0, 0.0);
        }
    }
    __syncthreads();
    fft_smem<N, NB, NT, FWD>(sd, tw);
    if (stride == 1) {
        for (int idx = threadIdx.x; idx < NB * N; idx += NT) {
            const int b = idx / N, e = idx % N;
            const long q = q0 + b;
            if (q < nseq) data[q * N + e] = sd[spad(e * NB + b)];
        }
    } else {
        for (int idx = threadIdx.x; idx < NB * N; idx += NT) {
            const int b = idx % NB, e = idx / NB;
            const long q = q0 + b;
            if (q < nseq) data[(q / stride) * N * stride + (long)e * stride + q % stride] = sd[spad(idx)];
        }
    }
}

template <int N>
static cudaError_t axis_impl(double2 *data, long stride, long nseq, bool fwd, const TwiddleSet &tw, int lg,
                             cudaStream_t st) {
    constexpr int NB = AxisCfg<N>::NB, NT = AxisCfg<N>::NT;
    const size_t smem = sizeof(double2) * padded_len<NB * N>::value;
    static unsigned mask = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(mask & (1u << dev))) {
        cudaFuncSetAttribute(k_fft_axis<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_fft_axis<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        mask |= 1u << dev;
    }
    const long blocks = (nseq + NB - 1) / NB;
    if (fwd)
        k_fft_axis<N, true><<<(unsigned)blocks, NT, smem, st>>>(data, stride, nseq, tw.f64[lg]);
    else
        k_fft_axis<N, false><<<(unsigned)blocks, NT, smem, st>>>(data, stride, nseq, tw.f64[lg]);
    return cudaGetLastError();
}

static cudaError_t fft_axis(double2 *data, int n, long stride, long nseq, bool fwd, const TwiddleSet &tw,
                            cudaStream_t st) {
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    switch (n) {
        case 1: return cudaSuccess;
        case 2: return axis_impl<2>(data, stride, nseq, fwd, tw, lg, st);
        case 4: return axis_impl<4>(data, stride, nseq, fwd, tw, lg, st);
        case 8: return axis_impl<8>(data, stride, nseq, fwd, tw, lg, st);
        case 16: return axis_impl<16>(data, stride, nseq, fwd, tw, lg, st);
        case 32: return axis_impl<32>(data, stride, nseq, fwd, tw, lg, st);
        case 64: return axis_impl<64>(data, stride, nseq, fwd, tw, lg, st);
        case 128: return axis_impl<128>(data, stride, nseq, fwd, tw, lg, st);
        case 256: return axis_impl<256>(data, stride, nseq, fwd, tw, lg, st);
        case 512: return axis_impl<512>(data, stride, nseq, fwd, tw, lg, st);
        case 1024: return axis_impl<1024>(data, stride, nseq, fwd, tw, lg, st);
        case 2048: return axis_impl<2048>(data, stride, nseq, fwd, tw, lg, st);
        default: return cudaErrorInvalidValue;
    }
}

// 3-D DFT in FFTW layout (n2 fastest), FFTW sign convention, unnormalised.
static cudaError_t fft3d(const pfc_run *r, const double2 *in, double2 *out, bool fwd) {
    const long P = r->P;
    cudaError_t e;
    if (in != out && (e = cudaMemcpyAsync(out, in, P * sizeof(double2), cudaMemcpyDeviceToDevice, r->stream)) != cudaSuccess)
        return e;
    const TwiddleSet &tw = r->ctx->tw;
    const int L = r->L, M = r->M, N = r->N;
    if ((e = fft_axis(out, N, 1, (long)L * M, fwd, tw, r->stream)) != cudaSuccess) return e;
    if ((e = fft_axis(out, M, N, (long)L * N, fwd, tw, r->stream)) != cudaSuccess) return e;
    return fft_axis(out, L, (long)M * N, (long)M * N, fwd, tw, r->stream);
}

// ---------------------------------------------------------------------------
// Pointwise kernels (one per reference routine).
// ---------------------------------------------------------------------------
#define GRID_LOOP(i, P) for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (P); i += (long)gridDim.x * blockDim.x)

// UPDATEINN3 (MIS:773-784) and UPDATEINFMIX (MIS:786-798)
__global__ void k64_inn3_infmix(const double2 *phi, const double2 *con, double2 *in1, double2 *in2, long P, float niu,
                                float ksi, float w, float c0) {
    GRID_LOOP(i, P) {
        const double ph = phi[i].x, c = con[i].x;
        in1[i] = make_double2(-(double)niu * (ph * ph) / 2.0 + (double)ksi * pow(ph, 3.0) / 3.0, 0.0);
        in2[i] = make_double2((double)w * (c * log(c / (double)c0) + (1.0 - c) * log((1.0 - c) / (1.0 - (double)c0))), 0.0);
    }
}

// UPDATEINFCMIX first half (MIS:803-813)
__global__ void k64_c2mult(const double2 *phiHat, const float *C2A, const float *C2B, const double *C2Ad,
                           const double *C2Bd, double2 *pa, double2 *pb, long P, int exact) {
    GRID_LOOP(i, P) {
        const double a = exact ? (double)C2A[i] : C2Ad[i], b = exact ? (double)C2B[i] : C2Bd[i];
        pa[i] = make_double2(a * phiHat[i].x, a * phiHat[i].y);
        pb[i] = make_double2(b * phiHat[i].x, b * phiHat[i].y);
    }
}

// UPDATEINFCMIX second half (MIS:818-831)
__global__ void k64_infcmix_post(double2 *ca, double2 *cb, const double2 *con, double2 *in3, long P, int LMN) {
    GRID_LOOP(i, P) {
        const double2 a = make_double2(ca[i].x / LMN, ca[i].y / LMN);
        const double2 b = make_double2(cb[i].x / LMN, cb[i].y / LMN);
        ca[i] = a;
        cb[i] = b;
        const double c = con[i].x, omc = 1.0 - c;
        in3[i] = make_double2(-(1.0 - 3.0 * (c * c) + 2.0 * pow(c, 3.0)) * a.x -
                                  (1.0 - 3.0 * (omc * omc) + 2.0 * pow(omc, 3.0)) * b.x,
                              0.0);
    }
}

// UPDATEINC2MIX (MIS:835-848) and UPDATEINC2MIXC (MIS:851-874)
__global__ void k64_inc2mix(const double2 *in1, const double2 *in2, const double2 *in3, const double2 *phi,
                            const double2 *con, const double2 *ca, const double2 *cb, double2 *inn, double2 *inc,
                            long P, float w, float c0, int exact) {
    GRID_LOOP(i, P) {
        inn[i] = make_double2(in1[i].x + in2[i].x + in3[i].x, 0.0);
        const double ph = phi[i].x, c = con[i].x, a = ca[i].x, b = cb[i].x;
        const double m1 = (double)w * (ph + 1.0) * log(c / (double)c0);
        const double m2 = (double)w * (ph + 1.0) * log((1.0 - c) / (1.0 - (double)c0));
        const double m3 = 3.0 * ph * (a - b) * (c * c);
        const double m4 = 3.0 * ph * (-1.0 * a + b) * c;
        if (exact) {
            const float f1 = (float)m1, f2 = (float)m2, f3 = (float)m3, f4 = (float)m4;
            inc[i] = make_double2((double)(__fsub_rn(__fsub_rn(__fsub_rn(f1, f2), f3), f4)), 0.0);
        } else {
            inc[i] = make_double2(m1 - m2 - m3 - m4, 0.0);
        }
    }
}

// MAINEQUATIONC2MIX / MAINEQUATIONC2_NOI (MIS:928-1014, CVD:865-886).  noisf != null
// adds the noise term dt*b0 * xi^ * |k| * mask * lowpass (MIS:1002-1003): the masks
// detrx = (l == 0), detrxn = (l == L/2), detry = (m == 0), detryn = (m == M/2) keep the
// real part (weight sqrt(|0.5 + 0.5 (detrx + detrxn)(detry + detryn)|)) and the
// imaginary part (sqrt(|0.5 - 0.5 (...)(...)|)) of the transformed white noise.
__global__ void k64_main_eq(double2 *phiHat, double2 *conHat, const double2 *outn, const double2 *outc,
                            const float *kl, const float *km, const float *kn, const double *kd, int L, int M, int N,
                            float mn, float mc, float alpha, float dt, int exact, const double2 *noisf, float b0) {
    const long P = (long)L * M * N;
    GRID_LOOP(i, P) {
        const int n = (int)(i % N), m = (int)((i / N) % M), l = (int)(i / ((long)N * M));
        const double dm = (double)((l == 0) + (l == L / 2)) * (double)((m == 0) + (m == M / 2));
        if (exact) {
            const float ks = __fadd_rn(__fadd_rn(__fmul_rn(kl[l], kl[l]), __fmul_rn(km[m], km[m])), __fmul_rn(kn[n], kn[n]));
            const float an = __fmul_rn(__fmul_rn(mn, dt), ks);
            double nre = 0.0, nim = 0.0;
            if (noisf) {
                const double sk = (double)__fsqrt_rn(ks);
                const double lp = 0.5 - 0.5 * tanh((sk - 2.0 * PI_REF) / 0.1);
                const double db = (double)__fmul_rn(dt, b0);  // dt * b0 in float, as the reference forms it
                nre = db * noisf[i].x * sk * sqrt(fabs(0.5 + 0.5 * dm)) * lp;
                nim = db * noisf[i].y * sk * sqrt(fabs(0.5 - 0.5 * dm)) * lp;
            }
            const float R1 = (float)(phiHat[i].x - (double)an * outn[i].x + nre);
            const float R2 = (float)(phiHat[i].y - (double)an * outn[i].y + nim);
            phiHat[i] = make_double2((double)R1 / (1.0 + (double)an), (double)R2 / (1.0 + (double)an));
            const float ac = __fmul_rn(__fmul_rn(mc, dt), ks);
            const float R3 = (float)(conHat[i].x - (double)ac * outc[i].x);
            const float R4 = (float)(conHat[i].y - (double)ac * outc[i].y);
            const float dc = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(mc, dt), alpha), ks), ks);
            conHat[i] = make_double2((double)R3 / (1.0 + (double)dc), (double)R4 / (1.0 + (double)dc));
        } else {
            // pure FP64: k-vectors in double
            const double ks = kd[l] * kd[l] + kd[L + m] * kd[L + m] + kd[L + M + n] * kd[L + M + n];
            const double an = (double)mn * dt * ks, ac = (double)mc * dt * ks, dc = (double)mc * dt * alpha * ks * ks;
            double nre = 0.0, nim = 0.0;
            if (noisf) {
                const double sk = sqrt(ks);
                const double lp = 0.5 - 0.5 * tanh((sk - 2.0 * PI_REF) / 0.1);
                nre = (double)dt * (double)b0 * noisf[i].x * sk * sqrt(fabs(0.5 + 0.5 * dm)) * lp;
                nim = (double)dt * (double)b0 * noisf[i].y * sk * sqrt(fabs(0.5 - 0.5 * dm)) * lp;
            }
            phiHat[i] = make_double2((phiHat[i].x - an * outn[i].x + nre) / (1.0 + an),
                                     (phiHat[i].y - an * outn[i].y + nim) / (1.0 + an));
            conHat[i] = make_double2((conHat[i].x - ac * outc[i].x) / (1.0 + dc), (conHat[i].y - ac * outc[i].y) / (1.0 + dc));
        }
    }
}

// UPDATEINC2GRA first half (MIS:880-896)
__global__ void k64_gra_pre(const double2 *conHat, const float *kl, const float *km, const float *kn, const double *kd,
                            double2 *g1, double2 *g2, double2 *g3, int L, int M, int N, int exact) {
    const long P = (long)L * M * N;
    GRID_LOOP(i, P) {
        const int n = (int)(i % N), m = (int)((i / N) % M), l = (int)(i / ((long)N * M));
        const double2 c = conHat[i];
        const double a = exact ? (double)kl[l] : kd[l];
        const double b = exact ? (double)km[m] : kd[L + m];
        const double d = exact ? (double)kn[n] : kd[L + M + n];
        g1[i] = make_double2(1.0 * a * c.y, -1.0 * a * c.x);
        g2[i] = make_double2(1.0 * b * c.y, -1.0 * b * c.x);
        g3[i] = make_double2(1.0 * d * c.y, -1.0 * d * c.x);
    }
}

// UPDATEINC2GRA second half (MIS:902-921), including the grao2-twice term of MIS:915
__global__ void k64_gra_post(double2 *o1, double2 *o2, double2 *o3, double2 *grac, int L, int M, int N) {
    const long P = (long)L * M * N;
    GRID_LOOP(i, P) {
        const double2 a = make_double2(o1[i].x / L / M / N, o1[i].y / L / M / N);
        const double2 b = make_double2(o2[i].x / L / M / N, o2[i].y / L / M / N);
        const double2 c = make_double2(o3[i].x / L / M / N, o3[i].y / L / M / N);
        o1[i] = a;
        o2[i] = b;
        o3[i] = c;
        grac[i] = make_double2(a.x * a.x + b.x * b.x + b.x * b.x, 0.0);
    }
}

// UPDATECOEF (MIS:686-697)
__global__ void k64_coef(double2 *phi, double2 *con, long P, int LMN) {
    GRID_LOOP(i, P) {
        phi[i] = make_double2(phi[i].x / LMN, 0.0);
        con[i] = make_double2(con[i].x / LMN, 0.0);
    }
}

// ENERGYC2 (MIS:1043-1092): per-block partial sums in index order.
__global__ void k64_energy(const double2 *phi, const double2 *con, const double2 *in3, const double2 *grac, long P,
                           float niu, float ksi, float w, float c0, float alpha, int exact, double *partials) {
    __shared__ double red[2][32];
    double se = 0.0, sm = 0.0;
    const long per = (P + gridDim.x - 1) / gridDim.x;
    const long b0 = blockIdx.x * per, b1 = b0 + per < P ? b0 + per : P;
    for (long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double ph = phi[i].x, c = con[i].x;
        const double eid = (ph * ph) / 2.0 - (double)niu * pow(ph, 3.0) / 6.0 + (double)ksi * pow(ph, 4.0) / 12.0;
        const double emix = (ph + 1.0) * (double)w * (c * log(c / (double)c0) + (1.0 - c) * log((1.0 - c) / (1.0 - (double)c0)));
        const double eex = 0.5 * ph * in3[i].x + (double)alpha * grac[i].x;
        if (exact)
            se += (double)__fadd_rn(__fadd_rn((float)eid, (float)emix), (float)eex);
        else
            se += eid + emix + eex;
        sm += ph;
    }
    for (int off = 16; off > 0; off >>= 1) {
        se += __shfl_down_sync(0xffffffffu, se, off);
        sm += __shfl_down_sync(0xffffffffu, sm, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = se;
        red[1][threadIdx.x >> 5] = sm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            a += red[0][i];
            b += red[1][i];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

__global__ void k64_from_real(const float *psi, const float *con, double2 *phi, double2 *cn, long P, double con_im) {
    GRID_LOOP(i, P) {
        phi[i] = make_double2((double)psi[i], 0.0);
        cn[i] = make_double2((double)con[i], con_im);
    }
}

__global__ void k64_to_real(const double2 *phi, const double2 *cn, float *psi, float *con, double *dphi, double *dcon,
                            long P) {
    GRID_LOOP(i, P) {
        psi[i] = (float)phi[i].x;
        con[i] = (float)cn[i].x;
        if (dphi) dphi[i] = phi[i].x;
        if (dcon) dcon[i] = cn[i].x;
    }
}

__global__ void k64_sum_fixed(const double *partials, int count, double *out) {
    if (threadIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int i = 0; i < count; ++i) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    out[0] = a;
    out[1] = b;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static unsigned grid_for(long P) {
    long b = (P + 255) / 256;
    return (unsigned)(b > 148 * 32 ? 148 * 32 : b);
}

#define TRY(expr)                                            \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return cuda_error(_e, #expr); \
    } while (0)

// Gauss (MIS:951-981): the reference's noise field of loop index `timestep`, value for
// value: one splitmix64 stream (pfc_common.h:165-176) keyed by the base seed, the rank
// (0 in one process) and the step, polar Box-Muller with rejection, f * v1 per point.
// Sequential by construction (each point's draws depend on the rejections before it).
static void gauss_host(uint32_t seed, int timestep, std::vector<float> &out) {
    uint64_t st = (uint64_t)seed;
    st ^= (uint64_t)((unsigned int)(0 + 1)) * 2654435761ULL;
    st ^= (uint64_t)((unsigned int)timestep) * 374761393ULL;
    auto u01 = [&st]() {
        uint64_t z = (st += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    for (size_t i = 0; i < out.size(); ++i) {
        float v1 = 0.0f, v2 = 0.0f, r2 = 2.0f;
        while (r2 >= 1.0f || r2 <= 0.0f) {
            v1 = (float)(2.0 * u01() - 1.0);
            v2 = (float)(2.0 * u01() - 1.0);
            r2 = v1 * v1 + v2 * v2;
        }
        const float f = (float)std::sqrt(-2. * logf(r2) / r2);
        out[i] = f * v1;
    }
}

// real noise values (float, staged in the first half of the noisf buffer) -> complex doubles
__global__ void k64_widen_noise(const float *in, double2 *out, long P) {
    GRID_LOOP(i, P) out[i] = make_double2((double)in[i], 0.0);
}

int fp64_create(pfc_run *r) {
    Fp64State *s = new Fp64State();  // value-initialised: every pointer null
    const size_t cz = (size_t)r->P * sizeof(double2);
    const size_t fz = ((size_t)r->P * sizeof(float) + 255) / 256 * 256;
    const size_t dz = ((size_t)r->P * sizeof(double) + 255) / 256 * 256;
    const size_t kz = ((size_t)(r->L + r->M + r->N) * sizeof(double) + 255) / 256 * 256;
    const bool noise = r->p.model == PFC_MODEL_MISFIT && r->b0 != 0.0f;
    const size_t bytes = (22 + (noise ? 2 : 0)) * cz + 2 * fz + 2 * dz + kz + (2 * EBLOCKS + 16) * sizeof(double);
    cudaError_t e = cudaMalloc(&s->mem, bytes);
    if (e != cudaSuccess) {
        delete s;
        return set_error(PFC_E_NOMEM, std::string("cudaMalloc FP64 state: ") + cudaGetErrorString(e));
    }
    cudaMemsetAsync(s->mem, 0, bytes, r->stream);
    char *m = (char *)s->mem;
    double2 **arrs[] = {&s->phi,     &s->con,     &s->phiHat, &s->conHat, &s->in1,  &s->in2,   &s->in3,   &s->inn,
                        &s->inc,     &s->outn,    &s->outc,   &s->c2adenp, &s->c2bdenp, &s->c2aden, &s->c2bden, &s->gra1,
                        &s->gra2,    &s->gra3,    &s->grao1,  &s->grao2,  &s->grao3, &s->grac};
    for (auto a : arrs) {
        *a = (double2 *)m;
        m += cz;
    }
    s->C2AHat = (float *)m;
    m += fz;
    s->C2BHat = (float *)m;
    m += fz;
    s->C2Ad = (double *)m;
    m += dz;
    s->C2Bd = (double *)m;
    m += dz;
    s->kd = (double *)m;
    m += kz;
    s->partials = (double *)m;
    m += (2 * EBLOCKS + 16) * sizeof(double);
    if (noise) {
        s->nois = (double2 *)m;
        m += cz;
        s->noisf = (double2 *)m;
        s->host_noise.resize(r->P);
    }
    s->exact = r->p.precision == PFC_PRECISION_FP64 ? 1 : 0;
    r->f64 = s;
    // C2AK / C2BK tables (MIS:700-750) evaluated on the host exactly as the reference does
    const int L = r->L, M = r->M, N = r->N;
    const float sig = r->p.sig;
    const ModelCoefs &k = r->k;
    std::vector<float> ta(r->P), tb(r->P);
    std::vector<double> tad(r->P), tbd(r->P), kd(L + M + N);
    // pure-FP64 k-vectors: same formula as MIS:455-462 with double system length
    for (int l = 0; l < L; ++l) kd[l] = (double)(l <= L / 2 ? l : l - L) * 2.0 * PI_REF / ((double)L * (double)r->p.dx);
    for (int mm = 0; mm < M; ++mm) kd[L + mm] = (double)(mm <= M / 2 ? mm : mm - M) * 2.0 * PI_REF / ((double)M * (double)r->p.dx);
    for (int n = 0; n < N; ++n) kd[L + M + n] = (double)(n <= N / 2 ? n : n - N) * 2.0 * PI_REF / ((double)N * (double)r->p.dx);
    for (int pass = 0; pass < 2; ++pass) {
        const float g1 = pass ? k.gab1 : k.gaa1, g2 = pass ? k.gab2 : k.gaa2;
        const float k1 = pass ? k.kb1 : k.ka1, k2 = pass ? k.kb2 : k.ka2;
        const float s1 = pass ? k.sigMb1 : k.sigMa1, s2 = pass ? k.sigMb2 : k.sigMa2;
        const float kc = c2_kc(sig, g1, g2, k1, k2, s1, s2);
        std::vector<float> &t = pass ? tb : ta;
        std::vector<double> &td = pass ? tbd : tad;
        const double q1 = (double)sig / s1, q2 = (double)sig / s2;
        const double dbb1 = 1. / (2. * g1 * g1), dbb2 = 1. / (2. * g2 * g2);
        const double dD = dbb1 * k1 - dbb2 * k2, dE = q1 * q1 - q2 * q2 + dbb1 * k1 * k1 - dbb2 * k2 * k2;
        double dkc = (dD + std::sqrt(dD * dD - (dbb1 - dbb2) * dE)) / (dbb1 - dbb2);
        if (g1 == g2) dkc = (q2 * q2 - q1 * q1 + dbb1 * ((double)k2 * k2 - (double)k1 * k1)) / (2 * dbb1 * ((double)k2 - k1));
        for (int l = 0; l < L; l++)
            for (int mm = 0; mm < M; mm++)
                for (int n = 0; n < N; n++) {
                    const float ks = r->krefl[l] * r->krefl[l] + r->krefm[mm] * r->krefm[mm] + r->krefn[n] * r->krefn[n];
                    const float sq = std::sqrt(ks);
                    float v = 0.0f;
                    if (sq <= kc) v = (float)(std::exp(-std::pow(sig / s1, 2)) * std::exp(-std::pow(sq - k1, 2) / (2 * g1 * g1)));
                    if (sq > kc) v = (float)(std::exp(-std::pow(sig / s2, 2)) * std::exp(-std::pow(sq - k2, 2) / (2 * g2 * g2)));
                    t[n + (long)N * (mm + (long)M * l)] = v;
                    const double kk = kd[l] * kd[l] + kd[L + mm] * kd[L + mm] + kd[L + M + n] * kd[L + M + n];
                    const double sd = std::sqrt(kk);
                    td[n + (long)N * (mm + (long)M * l)] =
                        sd <= dkc ? std::exp(-q1 * q1) * std::exp(-(sd - k1) * (sd - k1) / (2.0 * g1 * g1))
                                  : std::exp(-q2 * q2) * std::exp(-(sd - k2) * (sd - k2) / (2.0 * g2 * g2));
                }
    }
    TRY(cudaMemcpyAsync(s->C2AHat, ta.data(), r->P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaMemcpyAsync(s->C2BHat, tb.data(), r->P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaMemcpyAsync(s->C2Ad, tad.data(), r->P * sizeof(double), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaMemcpyAsync(s->C2Bd, tbd.data(), r->P * sizeof(double), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaMemcpyAsync(s->kd, kd.data(), kd.size() * sizeof(double), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaStreamSynchronize(r->stream));
    return PFC_OK;
}

void fp64_destroy(Fp64State *s) {
    if (!s) return;
    if (s->mem) cudaFree(s->mem);
    delete s;
}

int fp64_init_from_real(pfc_run *r, bool) {
    Fp64State *s = r->f64;
    // INITIAL_dis / INITIAL_C2 set con's imaginary part to 1e-10 (MIS:627, CVD:601)
    k64_from_real<<<grid_for(r->P), 256, 0, r->stream>>>(r->desc.psi_real, r->desc.con_real, s->phi, s->con, r->P, 1.0E-10);
    TRY(cudaGetLastError());
    TRY(cudaStreamSynchronize(r->stream));
    r->psi_mean = 0.0;
    r->con_mean = 0.0;
    r->fields_valid = true;
    r->energy_valid = false;
    return PFC_OK;
}

// UPDATEINFCMIX (MIS:801-833)
static int infcmix(pfc_run *r) {
    Fp64State *s = r->f64;
    const long P = r->P;
    k64_c2mult<<<grid_for(P), 256, 0, r->stream>>>(s->phiHat, s->C2AHat, s->C2BHat, s->C2Ad, s->C2Bd, s->c2adenp,
                                                   s->c2bdenp, P, s->exact);
    TRY(cudaGetLastError());
    TRY(fft3d(r, s->c2adenp, s->c2aden, false));  // p10
    TRY(fft3d(r, s->c2bdenp, s->c2bden, false));  // p11
    k64_infcmix_post<<<grid_for(P), 256, 0, r->stream>>>(s->c2aden, s->c2bden, s->con, s->in3, P, r->L * r->M * r->N);
    TRY(cudaGetLastError());
    return PFC_OK;
}

int fp64_advance(pfc_run *r, int nsteps) {
    Fp64State *s = r->f64;
    const long P = r->P;
    const ModelCoefs &k = r->k;
    const int exact = s->exact;
    const float *kl = r->desc.krefl, *km = r->desc.krefm, *kn = r->d_krefn;
    for (int it = 0; it < nsteps; ++it) {
        k64_inn3_infmix<<<grid_for(P), 256, 0, r->stream>>>(s->phi, s->con, s->in1, s->in2, P, k.niu, k.ksi, k.para_w,
                                                            k.para_c0);
        TRY(cudaGetLastError());
        TRY(fft3d(r, s->phi, s->phiHat, true));  // p1
        int rc = infcmix(r);
        if (rc != PFC_OK) return rc;
        k64_inc2mix<<<grid_for(P), 256, 0, r->stream>>>(s->in1, s->in2, s->in3, s->phi, s->con, s->c2aden, s->c2bden,
                                                        s->inn, s->inc, P, k.para_w, k.para_c0, exact);
        TRY(cudaGetLastError());
        TRY(fft3d(r, s->inn, s->outn, true));   // p8
        TRY(fft3d(r, s->inc, s->outc, true));   // p9
        TRY(fft3d(r, s->con, s->conHat, true)); // p6
        if (s->nois) {
            // Gauss (MIS:951-981) for this step's loop index, then p5
            gauss_host(r->p.seed, r->t + it, s->host_noise);
            TRY(cudaMemcpyAsync(s->noisf, s->host_noise.data(), P * sizeof(float), cudaMemcpyHostToDevice, r->stream));
            k64_widen_noise<<<grid_for(P), 256, 0, r->stream>>>((const float *)s->noisf, s->nois, P);
            TRY(cudaGetLastError());
            TRY(fft3d(r, s->nois, s->noisf, true));  // p5
        }
        k64_main_eq<<<grid_for(P), 256, 0, r->stream>>>(s->phiHat, s->conHat, s->outn, s->outc, kl, km, kn, s->kd, r->L, r->M,
                                                        r->N, k.dynamic_mn, k.dynamic_mc, k.para_alpha, r->p.dt, exact,
                                                        s->nois ? s->noisf : nullptr, r->b0);
        TRY(cudaGetLastError());
        k64_gra_pre<<<grid_for(P), 256, 0, r->stream>>>(s->conHat, kl, km, kn, s->kd, s->gra1, s->gra2, s->gra3, r->L, r->M,
                                                        r->N, exact);
        TRY(cudaGetLastError());
        TRY(fft3d(r, s->gra1, s->grao1, false));  // pe12
        TRY(fft3d(r, s->gra2, s->grao2, false));  // pe13
        TRY(fft3d(r, s->gra3, s->grao3, false));  // pe14
        k64_gra_post<<<grid_for(P), 256, 0, r->stream>>>(s->grao1, s->grao2, s->grao3, s->grac, r->L, r->M, r->N);
        TRY(cudaGetLastError());
        TRY(fft3d(r, s->phiHat, s->phi, false));  // p2
        TRY(fft3d(r, s->conHat, s->con, false));  // p7
        k64_coef<<<grid_for(P), 256, 0, r->stream>>>(s->phi, s->con, P, r->L * r->M * r->N);
        TRY(cudaGetLastError());
        rc = infcmix(r);
        if (rc != PFC_OK) return rc;
    }
    r->t += nsteps;
    r->fields_valid = false;
    r->energy_valid = true;
    return PFC_OK;
}

int fp64_materialize(pfc_run *r) {
    if (r->fields_valid) return PFC_OK;
    k64_to_real<<<grid_for(r->P), 256, 0, r->stream>>>(r->f64->phi, r->f64->con, r->desc.psi_real, r->desc.con_real,
                                                       nullptr, nullptr, r->P);
    TRY(cudaGetLastError());
    r->fields_valid = true;
    return PFC_OK;
}

int fp64_get_fields(pfc_run *r, double *phi, double *con) {
    TRY(cudaSetDevice(r->p.device));
    double *tmp = nullptr;
    TRY(cudaMalloc(&tmp, 2 * r->P * sizeof(double)));
    k64_to_real<<<grid_for(r->P), 256, 0, r->stream>>>(r->f64->phi, r->f64->con, r->desc.psi_real, r->desc.con_real,
                                                       tmp, tmp + r->P, r->P);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && phi) e = cudaMemcpyAsync(phi, tmp, r->P * sizeof(double), cudaMemcpyDeviceToHost, r->stream);
    if (e == cudaSuccess && con) e = cudaMemcpyAsync(con, tmp + r->P, r->P * sizeof(double), cudaMemcpyDeviceToHost, r->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_error(e, "fp64_get_fields");
    r->fields_valid = true;
    return PFC_OK;
}

int fp64_set_fields(pfc_run *r, const double *phi, const double *con) {
    std::vector<double2> a(r->P), b(r->P);
    for (long i = 0; i < r->P; ++i) {
        a[i] = make_double2(phi[i], 0.0);
        b[i] = make_double2(con[i], 0.0);
    }
    TRY(cudaMemcpyAsync(r->f64->phi, a.data(), r->P * sizeof(double2), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaMemcpyAsync(r->f64->con, b.data(), r->P * sizeof(double2), cudaMemcpyHostToDevice, r->stream));
    TRY(cudaStreamSynchronize(r->stream));
    r->fields_valid = false;
    r->energy_valid = false;
    return PFC_OK;
}

int fp64_energy(pfc_run *r, double *e_over_p, double *mass_over_p) {
    if (!r->energy_valid) return set_error(PFC_E_STATE, "energy is available after at least one step");
    Fp64State *s = r->f64;
    const ModelCoefs &k = r->k;
    k64_energy<<<EBLOCKS, 256, 0, r->stream>>>(s->phi, s->con, s->in3, s->grac, r->P, k.niu, k.ksi, k.para_w, k.para_c0,
                                               k.para_alpha, s->exact, s->partials);
    TRY(cudaGetLastError());
    k64_sum_fixed<<<1, 32, 0, r->stream>>>(s->partials, EBLOCKS, s->partials + 2 * EBLOCKS);
    TRY(cudaGetLastError());
    double out[2];
    TRY(cudaMemcpyAsync(out, s->partials + 2 * EBLOCKS, sizeof(out), cudaMemcpyDeviceToHost, r->stream));
    TRY(cudaStreamSynchronize(r->stream));
    if (e_over_p) *e_over_p = out[0] / r->L / r->M / r->N;
    if (mass_over_p) *mass_over_p = out[1] / r->L / r->M / r->N;
    return PFC_OK;
}

}  // namespace pfc

// ---------------------------------------------------------------------------
// pfc_dft3d: the 3-D complex-double DFT of the reference's FFTW calls
// (fftw_plan_dft_3d + fftw_execute, MIS:438-452), on the GPU, host buffers.
// ---------------------------------------------------------------------------
extern "C" int pfc_dft3d(const double *in, double *out, int n0, int n1, int n2, int sign) {
    using namespace pfc;
    if (!in || !out) return set_error(PFC_E_INVALID, "null buffer");
    const int dims[3] = {n0, n1, n2};
    for (int d : dims)
        if (d < 1 || d > 2048 || (d & (d - 1)) != 0) return set_error(PFC_E_INVALID, "extents must be powers of two <= 2048");
    if (sign != -1 && sign != 1) return set_error(PFC_E_INVALID, "sign must be -1 (forward) or +1 (backward)");
    int dev = 0;
    cudaGetDevice(&dev);
    Context *ctx = nullptr;
    int rc = get_context(dev, &ctx);
    if (rc != PFC_OK) return rc;
    const long P = (long)n0 * n1 * n2;
    double2 *d = nullptr;
    TRY(cudaMalloc(&d, P * sizeof(double2)));
    cudaError_t e = cudaMemcpyAsync(d, in, P * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream);
    const bool fwd = sign == -1;
    if (e == cudaSuccess) e = fft_axis(d, n2, 1, (long)n0 * n1, fwd, ctx->tw, ctx->stream);
    if (e == cudaSuccess) e = fft_axis(d, n1, n2, (long)n0 * n2, fwd, ctx->tw, ctx->stream);
    if (e == cudaSuccess) e = fft_axis(d, n0, (long)n1 * n2, (long)n1 * n2, fwd, ctx->tw, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, P * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_error(e, "pfc_dft3d");
    return PFC_OK;
}
