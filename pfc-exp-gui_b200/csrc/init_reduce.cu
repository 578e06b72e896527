// init_reduce.cu -- initial conditions and FP64 reductions.
//
// Compiled with --fmad=false: every float/double multiply and add here is rounded
// separately, as in the reference's x86-64 build, so the initial fields match the
// reference bit for bit.
//
// INITIAL_dis (src/experiment/misfit_uniform_time_seed_fftw_early.cpp:610-682) and
// INITIAL_C2 (src/experiment/cvd.cpp:587-642) evaluate cosf() of float arguments.
// The arguments only take a small set of values (an integer lattice index times a
// constant), so the host evaluates them once with the C library, exactly as the
// reference does, and the kernels look them up.  Everything else (grain boxes,
// the rotated lattice index X, Y with its double arithmetic and truncation to int)
// is computed per point on the device.
#include <cuda_runtime.h>
#include <stdint.h>

#include "pfc_internal.h"

namespace pfc {

struct GrainDev {
    float center_x, center_y, center_z;
    float cth;      // cosf(theta)
    double cother;  // cos(pi/2 - theta - (iii+jjj+kkk) pi)
};

// INITIAL_dis: phi = u0 and con = con0 everywhere, then the grain pattern for m < min(M, 160).
__global__ void k_init_misfit(float *__restrict__ psi, float *__restrict__ con, int L, int M, int N,
                              float u0, float con0, float dx, const GrainDev *__restrict__ grains, int ngrains,
                              double limx, double limy, const float *__restrict__ costab, int xmin, int ntab,
                              float A1x2, float A2x4) {
    const long P = (long)L * M * N;
    const int seed_m_max = M < 160 ? M : 160;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x) {
        const int n = (int)(i % N);
        const int m = (int)((i / N) % M);
        const int l = (int)(i / ((long)N * M));
        float v = u0;
        if (m < seed_m_max) {
            for (int g = ngrains - 1; g >= 0; --g) {
                const GrainDev gr = grains[g];
                const float xx = __fmul_rn(__fadd_rn(__fsub_rn(0.0f, gr.center_x), (float)l), dx);
                const float yy = __fmul_rn(__fsub_rn((float)m, gr.center_y), dx);
                const float zz = __fmul_rn(__fsub_rn((float)n, gr.center_z), dx);
                if ((double)fabsf(xx) < limx && (double)fabsf(yy) < limy && (double)fabsf(zz) < 4.3) {
                    const int X = (int)__dadd_rn((double)__fmul_rn((float)l, gr.cth), __dmul_rn((double)m, gr.cother));
                    const int Y = (int)__dsub_rn((double)__fmul_rn((float)m, gr.cth), __dmul_rn((double)l, gr.cother));
                    int ix = X - xmin, iy = Y - xmin;
                    ix = ix < 0 ? 0 : (ix >= ntab ? ntab - 1 : ix);
                    iy = iy < 0 ? 0 : (iy >= ntab ? ntab - 1 : iy);
                    const float cx = costab[ix], cy = costab[iy];
                    v = __fadd_rn(__fadd_rn(__fmul_rn(A1x2, __fadd_rn(cx, cy)), __fmul_rn(__fmul_rn(A2x4, cx), cy)), u0);
                    break;
                }
            }
        }
        psi[i] = v;
        con[i] = con0;
    }
}

// INITIAL_C2: A lattice for m < M/2, B lattice above (rotation angle w3 = 0).
__global__ void k_init_cvd(float *__restrict__ psi, float *__restrict__ con, int L, int M, int N, float u0,
                           float con0, const float *__restrict__ tab, float A1x2, float A2x4) {
    // tab layout: [cosA_l (L)] [cosA_m (M)] [cosB_l (L)] [cosB_m (M)]
    const long P = (long)L * M * N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x) {
        const int m = (int)((i / N) % M);
        const int l = (int)(i / ((long)N * M));
        const bool A = m < M / 2;
        const float c1 = A ? tab[l] : tab[L + M + l];
        const float c2 = A ? tab[L + m] : tab[2 * L + M + m];
        psi[i] = __fadd_rn(__fadd_rn(__fmul_rn(A1x2, __fadd_rn(c1, c2)), __fmul_rn(__fmul_rn(A2x4, c1), c2)), u0);
        con[i] = A ? con0 : __fsub_rn(1.0f, con0);
    }
}

// Sum of a float field in double: per-block partials, then one block adds them in
// a fixed order (deterministic).
__global__ void k_sum_partials(const float *__restrict__ a, long n, double *__restrict__ partials) {
    __shared__ double red[32];
    double acc = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        acc += (double)a[i];
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        partials[blockIdx.x] = s;
    }
}

// out[j] = sum_i partials[i * stride + j] for j < width (width <= stride), the additions in
// index order, one thread per j.  The CTA stages the partials chunk by chunk into shared
// memory with coalesced loads, so the ordered sum waits on shared-memory reads rather
// than on one global load per term.
constexpr int REDUCE_NT = 256, REDUCE_CHUNK = 4096;  // threads; doubles staged at a time
__device__ __forceinline__ void ordered_sums(const double *__restrict__ partials, int count, int stride, int width,
                                             double *__restrict__ out) {
    __shared__ double buf[REDUCE_CHUNK];
    const long total = (long)count * stride;
    const int rows = REDUCE_CHUNK / stride;  // whole rows of `stride` doubles per chunk
    double s = 0.0;
    for (long base = 0; base < total; base += (long)rows * stride) {
        const int n = (int)(total - base < (long)rows * stride ? total - base : (long)rows * stride);
        __syncthreads();  // the previous chunk's sums are done
        for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = partials[base + i];
        __syncthreads();
        if (threadIdx.x < width)
            for (int i = threadIdx.x; i < n; i += stride) s += buf[i];
    }
    if (threadIdx.x < width) out[threadIdx.x] = s;
}

__global__ void __launch_bounds__(REDUCE_NT) k_reduce_fixed(const double *__restrict__ partials, int count, int stride,
                                                            int width, double *__restrict__ out) {
    ordered_sums(partials, count, stride, width, out);
}

// out[j] = sum_i partials[i * stride + j] for j < width <= 2, by a tree of fixed shape: thread
// t of the REDUCE_NT threads sums rows t, t + REDUCE_NT, ... in index order, then the 32
// lanes of each warp by shuffles (halving offsets) and the warps' sums in warp order.  The
// result does not depend on scheduling, and a run's sums are the same alone and in a batch
// (k_reduce_runs calls the same function); the rows are read in parallel.
__device__ __forceinline__ void tree_sums(const double *__restrict__ partials, int count, int stride, int width,
                                          double *__restrict__ out) {
    __shared__ double red[2][REDUCE_NT / 32];
    double acc[2] = {0.0, 0.0};
    // a thread adds partials tid, tid + NT, tid + 2 NT, ... in that order; eight of them are
    // loaded ahead of their additions, so that the loads overlap
    constexpr int U = 8;
    int i = threadIdx.x;
    for (; i + (U - 1) * REDUCE_NT < count; i += U * REDUCE_NT) {
        double v[U][2];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int j = 0; j < 2; ++j) v[u][j] = j < width ? partials[(long)(i + u * REDUCE_NT) * stride + j] : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (j < width) acc[j] += v[u][j];
    }
    for (; i < count; i += REDUCE_NT)
#pragma unroll
        for (int j = 0; j < 2; ++j)
            if (j < width) acc[j] += partials[(long)i * stride + j];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        double v = acc[j];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[j][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < width) {
        double t = 0.0;
        for (int w = 0; w < REDUCE_NT / 32; ++w) t += red[threadIdx.x][w];
        out[threadIdx.x] = t;
    }
}

__global__ void __launch_bounds__(REDUCE_NT) k_reduce_tree(const double *__restrict__ partials, int count, int stride,
                                                           int width, double *__restrict__ out) {
    tree_sums(partials, count, stride, width, out);
}

cudaError_t launch_init_misfit(float *psi, float *con, int L, int M, int N, float u0, float con0, float dx,
                               const void *grains, int ngrains, double limx, double limy, const float *costab,
                               int xmin, int ntab, float A1x2, float A2x4, cudaStream_t s) {
    const long P = (long)L * M * N;
    int blocks = (int)((P + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_init_misfit<<<blocks, 256, 0, s>>>(psi, con, L, M, N, u0, con0, dx, (const GrainDev *)grains, ngrains, limx,
                                         limy, costab, xmin, ntab, A1x2, A2x4);
    return cudaGetLastError();
}

cudaError_t launch_init_cvd(float *psi, float *con, int L, int M, int N, float u0, float con0, const float *tab,
                            float A1x2, float A2x4, cudaStream_t s) {
    const long P = (long)L * M * N;
    int blocks = (int)((P + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_init_cvd<<<blocks, 256, 0, s>>>(psi, con, L, M, N, u0, con0, tab, A1x2, A2x4);
    return cudaGetLastError();
}

// Deterministic FP64 sum of n floats.  scratch must hold `blocks` doubles.
cudaError_t launch_sum_f32(const float *a, long n, double *scratch, int blocks, double *out, cudaStream_t s) {
    k_sum_partials<<<blocks, 256, 0, s>>>(a, n, scratch);
    k_reduce_fixed<<<1, REDUCE_NT, 0, s>>>(scratch, blocks, 1, 1, out);
    return cudaGetLastError();
}

// Sums of the analysis partials (energy, mass): the fixed-shape tree of tree_sums.
cudaError_t launch_reduce_fixed(const double *partials, int count, int stride, int width, double *out,
                                cudaStream_t s) {
    if (stride < 1 || width > stride || width > 2) return cudaErrorInvalidValue;
    k_reduce_tree<<<1, REDUCE_NT, 0, s>>>(partials, count, stride, width, out);
    return cudaGetLastError();
}

// k_reduce_fixed(partials, count, 2, 2, ...) for run blockIdx.x of a batch.
__global__ void __launch_bounds__(REDUCE_NT) k_reduce_runs(const RunDesc *__restrict__ runs, int count, int slot) {
    const RunDesc &d = runs[blockIdx.x];
    tree_sums(d.partials, count, 2, 2, d.ehist + 2 * slot);
}

cudaError_t launch_reduce_runs(const RunDesc *d_runs, int nruns, int nparts, int slot, cudaStream_t s) {
    if (nruns <= 0) return cudaSuccess;
    k_reduce_runs<<<nruns, REDUCE_NT, 0, s>>>(d_runs, nparts, slot);
    return cudaGetLastError();
}

}  // namespace pfc
