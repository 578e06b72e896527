// analysis.cu -- checkpoint analysis kernels: peak finders, elastic3D, cryst_order.
//
// Compiled with --fmad=false.  The peak tests, sub-pixel fits and neighbour
// distances use exactly the reference's sequence of separately rounded float and
// double operations, so atom indices, positions, neighbour counts and strains are
// bit-identical to the reference given the same field.  Only the spherical
// harmonics of cryst_order call transcendental functions (cosf, sinf, acos, atan)
// whose last bits may differ from the C library's.
//
// Atoms are emitted in the reference's loop order by an ordered stream compaction:
// count per block, exclusive scan of the block counts, then each block re-evaluates
// its points and writes its atoms at (block offset + rank within the block).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "pfc_b200.h"
#include "pfc_engine.h"

namespace pfc {

static constexpr double PI_REF = 3.1415926;
static constexpr int CBLK = 256;         // threads per compaction block
static constexpr int CPT = 4;            // points per thread
static constexpr int CSPAN = CBLK * CPT; // points per compaction block

// ---------------------------------------------------------------------------
// Misfit peak finder (MIS:3261-3556).  Emission index o = m*L + p (loops n, m, l
// with l fastest); p is the field row (buffer row p+1, edge-replicated halo).
// ---------------------------------------------------------------------------
struct MisfitPeak {
    const float *phi, *con;
    int L, M;
    float dx, con0;
    __device__ __forceinline__ double at(int p, int m) const { return (double)phi[(long)p * M + m]; }
    __device__ __forceinline__ static double nb(double v) { return isfinite(v) ? v : -INFINITY; }
    __device__ bool test(long o) const {
        const int p = (int)(o % L), m = (int)(o / L);
        const double center = at(p, m);
        if (!isfinite(center) || center <= -0.07) return false;
        const int pf = p > 0 ? p - 1 : 0, pb = p < L - 1 ? p + 1 : L - 1;
        const int mf = m > 0 ? m - 1 : M - 1, mb = m < M - 1 ? m + 1 : 0;
        const double v[8] = {nb(at(pf, m)),  nb(at(pb, m)),  nb(at(p, mf)),  nb(at(p, mb)),
                             nb(at(pb, mb)), nb(at(pf, mb)), nb(at(pb, mf)), nb(at(pf, mf))};
        bool ge_all = true, gt_any = false;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (center < v[q]) ge_all = false;
            if (center > v[q]) gt_any = true;
        }
        return ge_all && gt_any;
    }
    __device__ void record(long o, double *out) const {
        const int p = (int)(o % L), m = (int)(o / L);
        const int pf = p > 0 ? p - 1 : 0, pb = p < L - 1 ? p + 1 : L - 1;
        const int mf = m > 0 ? m - 1 : M - 1, mb = m < M - 1 ? m + 1 : 0;
        const double xtemp = (double)__fmul_rn((float)(p + 2), dx);
        const double ytemp = (double)__fmul_rn((float)(m + 1), dx);
        const double ztemp = (double)__fmul_rn(1.0f, dx);
        const double z0 = at(p, m), z1 = at(pb, m), z3 = at(pf, m), z4 = at(p, mb), z2 = at(p, mf);
        double delta_x = 0.0, delta_y = 0.0, phi_local = z0;
        if (isfinite(z1) && isfinite(z3) && isfinite(z4) && isfinite(z2)) {
            const double dx_d = (double)dx;
            const double inv2dx = 0.5 / dx_d;
            const double invdx2 = 1.0 / (dx_d * dx_d);
            const double a1 = (z1 - z3) * inv2dx;
            const double a2 = (z4 - z2) * inv2dx;
            const double a3 = 0.5 * (z1 + z3 - 2.0 * z0) * invdx2;
            const double a4 = 0.5 * (z2 + z4 - 2.0 * z0) * invdx2;
            const double eps = 1e-12;
            if (isfinite(a3) && fabs(a3) > eps) delta_x = -a1 / (2.0 * a3);
            if (isfinite(a4) && fabs(a4) > eps) delta_y = -a2 / (2.0 * a4);
            const double h = 0.5 * dx_d;
            delta_x = delta_x < -h ? -h : (h < delta_x ? h : delta_x);
            delta_y = delta_y < -h ? -h : (h < delta_y ? h : delta_y);
            double phi_interp = z0;
            if (isfinite(a3) && fabs(a3) > eps && isfinite(a1)) phi_interp -= 0.25 * a1 * a1 / a3;
            if (isfinite(a4) && fabs(a4) > eps && isfinite(a2)) phi_interp -= 0.25 * a2 * a2 / a4;
            if (isfinite(phi_interp)) phi_local = phi_interp;
        }
        const float c = con[(long)p * M + m];
        out[0] = xtemp + delta_x;
        out[1] = ytemp + delta_y;
        out[2] = ztemp;
        out[3] = phi_local;
        out[4] = (double)(isfinite(c) ? c : con0);
    }
    static constexpr int REC = 5;
};

// ---------------------------------------------------------------------------
// Elastic peak finder (ELA:2802-2921).  Emission index o = natural index
// n + N*(m + M*p); buffer row l = p + 1 with edge-replicated halo rows.
// ---------------------------------------------------------------------------
struct ElasticPeak {
    const float *phi;
    const float *phic_ptr;  // device scalar: phimax - phimax * 0.40f
    int L, M, N;
    float dx;
    // value of the reference's buffer at flat index idx of buf[M*N*(L+2)]
    __device__ __forceinline__ float buf(long idx) const {
        const long slab = (long)M * N;
        long row = idx / slab - 1;
        row = row < 0 ? 0 : (row > L - 1 ? L - 1 : row);
        return phi[row * slab + idx % slab];
    }
    __device__ bool test(long o) const {
        const float phic = *phic_ptr;
        const int n = (int)(o % N), m = (int)((o / N) % M), p = (int)(o / ((long)N * M));
        const int l = p + 1;
        const float center = phi[o];
        if (!(center > phic)) return false;
        const long total = (long)M * N * (L + 2);
        for (int lx = -1; lx < 2; lx++)
            for (int ly = -1; ly < 2; ly++)
                for (int lz = -1; lz < 2; lz++) {
                    const int ix = l + lx;
                    int jy = m + ly, kz = n + lz;
                    if (jy > (M - 1)) jy = jy - M + 1;
                    if (kz > (N - 1)) kz = kz - N + 1;
                    if (jy < 0) jy = jy + M - 1;
                    if (kz < 0) kz = kz + N - 1;
                    const long idx = kz + (long)N * (jy + (long)M * ix);
                    // the reference reads one element outside its buffer at the first and
                    // last buffer position (ELA:2879); such a read never rejects here
                    if (idx < 0 || idx >= total) continue;
                    if (buf(idx) > center) return false;
                }
        return true;
    }
    __device__ void record(long o, double *out) const {
        const int n = (int)(o % N), m = (int)((o / N) % M), p = (int)(o / ((long)N * M));
        const int l = p + 1;
        const int lf = l - 1, lb = l + 1;
        int mf = m - 1, mb = m + 1, nf = n - 1, nbb = n + 1;
        if (mf < 0) mf = M - 1;
        if (mb > M - 1) mb = 0;
        if (nf < 0) nf = N - 1;
        if (nbb > N - 1) nbb = 0;
        auto B = [&](int nn, int mm, int ll) { return (double)buf(nn + (long)N * (mm + (long)M * ll)); };
        const double xtemp = (double)l, ytemp = (double)m, ztemp = (double)n;
        const double z0 = B(n, m, l), z1 = B(n, m, lb), z3 = B(n, m, lf), z4 = B(n, mb, l), z2 = B(n, mf, l);
        const double z5 = B(nbb, m, l), z6 = B(nf, m, l);
        const double dxd = (double)dx, dx2 = (double)__fmul_rn(dx, dx);
        const double a0 = z0;
        const double a1 = 0.5 * (z1 - z3) / dxd + 10e-8;
        const double a2 = 0.5 * (z4 - z2) / dxd + 10e-8;
        const double a3 = 0.5 * (z1 + z3 - 2. * z0) / dx2 + 10e-8;
        const double a4 = 0.5 * (z2 + z4 - 2. * z0) / dx2 + 10e-8;
        const double a5 = 0.5 * (z5 - z6) / dxd + 10e-8;
        const double a6 = 0.5 * (z5 + z6 - 2. * z0) / dx2 + 10e-8;
        out[0] = (xtemp + 1) * dxd + (-a1 / (2. * a3));
        out[1] = (ytemp + 1) * dxd + (-a2 / (2. * a4));
        out[2] = (ztemp + 1) * dxd + (-a5 / (2. * a6));
        out[3] = a0 - 0.25 * a1 * a1 / a3 - 0.25 * a2 * a2 / a4 - 0.25 * a5 * a5 / a6;
    }
    static constexpr int REC = 4;
};

// ---------------------------------------------------------------------------
// Ordered compaction
// ---------------------------------------------------------------------------
template <typename F> __global__ void k_count(F f, long n, int *__restrict__ block_counts) {
    __shared__ int red[CBLK / 32];
    const long base = (long)blockIdx.x * CSPAN + (long)threadIdx.x * CPT;
    int c = 0;
#pragma unroll
    for (int q = 0; q < CPT; ++q)
        if (base + q < n && f.test(base + q)) ++c;
    for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < CBLK / 32; ++w) s += red[w];
        block_counts[blockIdx.x] = s;
    }
}

// Exclusive scan of nb block counts in one block; total in offsets[nb].
__global__ void k_scan(const int *__restrict__ counts, int nb, int *__restrict__ offsets) {
    __shared__ int part[1024];
    const int t = threadIdx.x, T = blockDim.x;
    const int per = (nb + T - 1) / T, b0 = t * per, b1 = b0 + per < nb ? b0 + per : nb;
    int s = 0;
    for (int i = b0; i < b1; ++i) s += counts[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        int acc = 0;
        for (int i = 0; i < T; ++i) {
            const int v = part[i];
            part[i] = acc;
            acc += v;
        }
        offsets[nb] = acc;
    }
    __syncthreads();
    int acc = part[t];
    for (int i = b0; i < b1; ++i) {
        offsets[i] = acc;
        acc += counts[i];
    }
}

template <typename F>
__global__ void k_emit(F f, long n, const int *__restrict__ offsets, double *__restrict__ out, int cap) {
    __shared__ int warp_tot[CBLK / 32];
    const long base = (long)blockIdx.x * CSPAN + (long)threadIdx.x * CPT;
    bool hit[CPT];
    int c = 0;
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
        hit[q] = base + q < n && f.test(base + q);
        c += hit[q];
    }
    // exclusive prefix of c over the block in thread order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = c;
    for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += v;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    int woff = 0;
    for (int w = 0; w < warp; ++w) woff += warp_tot[w];
    int rank = offsets[blockIdx.x] + woff + incl - c;
#pragma unroll
    for (int q = 0; q < CPT; ++q)
        if (hit[q]) {
            if (rank < cap) f.record(base + q, out + (long)F::REC * rank);
            ++rank;
        }
}

// Scratch for one compaction over n points.
struct CompactScratch {
    int *counts = nullptr;
    int nb = 0;
};

template <typename F>
static int compact(F f, long n, double *d_out, int cap, int *count, cudaStream_t st) {
    const int nb = (int)((n + CSPAN - 1) / CSPAN);
    int *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, sizeof(int) * (2 * (size_t)nb + 2), st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync compaction");
    k_count<<<nb, CBLK, 0, st>>>(f, n, buf);
    k_scan<<<1, 1024, 0, st>>>(buf, nb, buf + nb);
    k_emit<<<nb, CBLK, 0, st>>>(f, n, buf + nb, d_out, cap);
    int total = 0;
    e = cudaMemcpyAsync(&total, buf + 2 * nb, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return cuda_error(e, "peak compaction");
    *count = total;
    return PFC_OK;
}

// Global-maximum fallback of MIS:3310-3330 and 3449-3464: the last finite maximum
// in l-major order; one thread, rarely used (fields without any local maximum).
__global__ void k_misfit_fallback(const float *phi, const float *con, int L, int M, float dx, float con0,
                                  double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double gmax = -INFINITY;
    int gm = 0, gl = 1;
    for (int p = 0; p < L; ++p)
        for (int m = 0; m < M; ++m) {
            const double v = (double)phi[(long)p * M + m];
            if (!isfinite(v)) continue;
            gmax = gmax < v ? v : gmax;
            if (v >= gmax) {
                gm = m;
                gl = p + 1;
            }
        }
    const double dxd = (double)dx;
    out[0] = (double)(0 + gl + 1) * dxd;
    out[1] = (double)(gm + 1) * dxd;
    out[2] = dxd;
    out[3] = isfinite(gmax) ? gmax : 0.0;
    const float c = con[(long)(gl - 1) * M + gm];
    out[4] = (double)(isfinite(c) ? c : con0);
}

__global__ void k_phic(const float *phi, long n, float *phic) {
    __shared__ float red[32];
    float m = 0.0f;  // phimax starts at 0 (ELA:2809)
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        const float v = phi[i];
        if (v > m) m = v;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float o = __shfl_down_sync(0xffffffffu, m, off);
        if (o > m) m = o;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (red[w] > s) s = red[w];
        phic[0] = __fsub_rn(s, __fmul_rn(s, 0.40f));
    }
}

int phimax_misfit_dev(const float *d_phi, const float *d_con, int L, int M, float dx, float con0, double *d_out,
                      int cap, int *count, int *raw_count, cudaStream_t st) {
    MisfitPeak f{d_phi, d_con, L, M, dx, con0};
    int rc = compact(f, (long)L * M, d_out, cap, count, st);
    if (rc != PFC_OK) return rc;
    if (raw_count) *raw_count = *count;
    if (*count == 0) {
        if (cap > 0) k_misfit_fallback<<<1, 32, 0, st>>>(d_phi, d_con, L, M, dx, con0, d_out);
        *count = 1;
    }
    return PFC_OK;
}

int phimax_elastic_dev(const float *d_phi, int L, int M, int N, float dx, double *d_out, int cap, int *count,
                       cudaStream_t st) {
    float *phic = nullptr;
    cudaError_t e = cudaMallocAsync(&phic, sizeof(float), st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync phic");
    k_phic<<<1, 1024, 0, st>>>(d_phi, (long)L * M * N, phic);
    ElasticPeak f{d_phi, phic, L, M, N, dx};
    int rc = compact(f, (long)L * M * N, d_out, cap, count, st);
    cudaFreeAsync(phic, st);
    return rc;
}

// ---------------------------------------------------------------------------
// Neighbour search shared by elastic3D and cryst_order (ELA:3048-3090, 3652-3722):
// float minimum-image distances computed from double positions.
// ---------------------------------------------------------------------------
struct PairGeom {
    float r3[9];
    float drx, dry, drz, rr;
};

__device__ __forceinline__ float min3f(float a, float b, float c) {
    const float aa = fabsf(a), bb = fabsf(b), cc = fabsf(c);
    return ((aa < bb ? aa : bb) < cc) ? (aa < bb ? aa : bb) : cc;
}

__device__ __forceinline__ void pair_geom(double xi, double yi, double zi, double xj, double yj, double zj, float fx,
                                          float fy, float fz, PairGeom &g) {
    g.r3[0] = (float)(xi - xj);
    g.r3[1] = (float)(yi - yj);
    g.r3[2] = (float)(zi - zj);
    g.r3[3] = __fadd_rn(g.r3[0], fx);
    g.r3[4] = __fadd_rn(g.r3[1], fy);
    g.r3[5] = __fadd_rn(g.r3[2], fz);
    g.r3[6] = __fsub_rn(g.r3[0], fx);
    g.r3[7] = __fsub_rn(g.r3[1], fy);
    g.r3[8] = __fsub_rn(g.r3[2], fz);
    g.drx = min3f(fabsf(g.r3[0]), fabsf(g.r3[3]), fabsf(g.r3[6]));
    g.dry = min3f(fabsf(g.r3[1]), fabsf(g.r3[4]), fabsf(g.r3[7]));
    g.drz = min3f(fabsf(g.r3[2]), fabsf(g.r3[5]), fabsf(g.r3[8]));
    g.rr = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(g.drx, g.drx), __fmul_rn(g.dry, g.dry)), __fmul_rn(g.drz, g.drz)));
}

// Image position of the neighbour (rjx, rjy, rjz of ELA:3676-3684): the last of the
// three images whose |offset| is within 1e-3 of the minimum.
__device__ __forceinline__ void neighbour_pos(const PairGeom &g, double xi, double yi, double zi, float &rjx,
                                              float &rjy, float &rjz) {
    for (int ii = 0; ii < 7; ii += 3)
        if (fabsf(__fsub_rn(fabsf(g.r3[ii]), g.drx)) < 1e-3) rjx = (float)(xi - (double)g.r3[ii]);
    for (int ii = 1; ii < 8; ii += 3)
        if (fabsf(__fsub_rn(fabsf(g.r3[ii]), g.dry)) < 1e-3) rjy = (float)(yi - (double)g.r3[ii]);
    for (int ii = 2; ii < 9; ii += 3)
        if (fabsf(__fsub_rn(fabsf(g.r3[ii]), g.drz)) < 1e-3) rjz = (float)(zi - (double)g.r3[ii]);
}

// One warp per atom i; lanes scan j in ascending chunks of 32 and the first 16
// qualifying neighbours (in ascending j) are kept, as in ELA:3674.
__global__ void k_elastic3d(const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z,
                            int n, float fx, float fy, float fz, float benchel, double *__restrict__ strain,
                            uint32_t *__restrict__ nbout) {
    __shared__ double contrib[8][16][3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * 8 + warp;
    if (i >= n) return;
    const double xi = x[i], yi = y[i], zi = z[i];
    unsigned Nb = 0;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        bool ok = false;
        PairGeom g;
        if (j < n && j != i) {
            pair_geom(xi, yi, zi, x[j], y[j], z[j], fx, fy, fz, g);
            ok = g.rr < benchel && (double)g.rr > 0.7;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const unsigned slot = Nb + __popc(bal & ((1u << lane) - 1u));
            if (slot < 16) {
                float rjx = 0.f, rjy = 0.f, rjz = 0.f;
                neighbour_pos(g, xi, yi, zi, rjx, rjy, rjz);
                const double rij = (double)g.rr;
                const double cn = ((double)rjx - xi) / rij, sn = ((double)rjy - yi) / rij, tn = ((double)rjz - zi) / rij;
                double sx = 0.0, sy = 0.0, sz = 0.0;  // the reference's uninitialised term is 0 here
                if (rij < 1.3) {
                    sx = 1.0 * (rij - 1) * cn;
                    sy = 1.0 * (rij - 1) * sn;
                    sz = 1.0 * (rij - 1) * tn;
                }
                contrib[warp][slot][0] = sx;
                contrib[warp][slot][1] = sy;
                contrib[warp][slot][2] = sz;
            }
        }
        Nb += __popc(bal);
    }
    __syncwarp();
    if (lane == 0) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        const unsigned k = Nb < 16 ? Nb : 16;
        for (unsigned s = 0; s < k; ++s) {
            sx = sx + contrib[warp][s][0];
            sy = sy + contrib[warp][s][1];
            sz = sz + contrib[warp][s][2];
        }
        strain[i] = sqrt(sx * sx + sy * sy + sz * sz);
        nbout[i] = Nb;
    }
}

// cryst_order neighbour list: r < 1.2, first 16 in ascending j, angles of ELA:3096-3104.
__global__ void k_cryst_neighbours(const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ z, int n, float fx, float fy, float fz,
                                   uint32_t *__restrict__ nbcount, int *__restrict__ nbidx, double *__restrict__ theta,
                                   double *__restrict__ fai) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * 8 + warp;
    if (i >= n) return;
    const double xi = x[i], yi = y[i], zi = z[i];
    unsigned Nb = 0;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        bool ok = false;
        PairGeom g;
        if (j < n && j != i) {
            pair_geom(xi, yi, zi, x[j], y[j], z[j], fx, fy, fz, g);
            ok = g.rr < 1.2f;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const unsigned slot = Nb + __popc(bal & ((1u << lane) - 1u));
            if (slot < 16) {
                float rjx = 0.f, rjy = 0.f, rjz = 0.f;
                neighbour_pos(g, xi, yi, zi, rjx, rjy, rjz);
                const double rij = (double)g.rr;
                const double CoX = rjx, CoY = rjy, CoZ = rjz;
                const long k = (long)16 * i + slot;
                theta[k] = acos((CoZ - zi) / (rij + 1.e-4));
                double f = atan((CoY - yi) / (CoX - xi + 1.e-4));
                if ((CoX - xi) < 0.) f = f + PI_REF;
                fai[k] = f;
                nbidx[k] = j;
            }
        }
        Nb += __popc(bal);
    }
    if (lane == 0) nbcount[i] = Nb;
}

// Spherical harmonics in float (pfc_common.h:274-343).
__device__ __forceinline__ float lg_poly(int l, float x) {
    float plm2 = 1, plm1 = x, pl = 0;
    if (l == 0) return 1;
    if (l == 1) return x;
    for (int i = 2; i <= l; i++) {
        pl = __fdiv_rn(__fsub_rn(__fmul_rn(__fmul_rn((float)(2 * i - 1), x), plm1), __fmul_rn((float)(i - 1), plm2)), (float)i);
        plm2 = plm1;
        plm1 = pl;
    }
    return pl;
}
__device__ __forceinline__ float plgndr(int l, int m, float x) {
    float pll = 0, pmm = 1.0f, pmmp1;
    if (m < 0) m = -m;
    if (m == 0) return lg_poly(l, x);
    const float somx2 = (float)sqrt((1.0 - x) * (1.0 + x));
    float fact = 1.0f;
    for (int i = 1; i <= m; i++) {
        pmm = __fmul_rn(pmm, __fmul_rn(-fact, somx2));
        fact = (float)(fact + 2.0);
    }
    if (l == m) return pmm;
    pmmp1 = __fmul_rn(__fmul_rn(x, (float)(2 * m + 1)), pmm);
    if (l == (m + 1)) return pmmp1;
    for (int ll = m + 2; ll <= l; ll++) {
        pll = __fdiv_rn(__fsub_rn(__fmul_rn(__fmul_rn(x, (float)(2 * ll - 1)), pmmp1), __fmul_rn((float)(ll + m - 1), pmm)),
                        (float)(ll - m));
        pmm = pmmp1;
        pmmp1 = pll;
    }
    return pll;
}
__device__ __forceinline__ int facto(int h) {
    int g = 1;
    for (int i = 1; i <= h; i++) g = g * i;
    return g;
}
__device__ __forceinline__ float ylm_norm(int l, int m, int sign_exp) {
    return (float)(pow(-1.0, (double)sign_exp) * sqrt((2 * l + 1) / 4. / PI_REF) *
                   (double)__fsqrt_rn(__fdiv_rn((float)facto(l - m), (float)facto(l + m))));
}
__device__ __forceinline__ float ylm_r(int l, int m, float theta, float fai) {
    if (m < 0) m = -m;
    const float fnorm = ylm_norm(l, m, m);
    return __fmul_rn(__fmul_rn(fnorm, plgndr(l, m, cosf(theta))), cosf(__fmul_rn((float)m, fai)));
}
__device__ __forceinline__ float ylm_c(int l, int m, float theta, float fai) {
    float fnorm, comp;
    if (m < 0) {
        m = -m;
        fnorm = ylm_norm(l, m, m + m);
        comp = -sinf(__fmul_rn((float)m, fai));
    } else {
        fnorm = ylm_norm(l, m, m);
        comp = sinf(__fmul_rn((float)m, fai));
    }
    return __fmul_rn(__fmul_rn(fnorm, plgndr(l, m, cosf(theta))), comp);
}

// qlmb[i][m] (ELA:3166-3177): average of Y_6m over the neighbours of i.
__global__ void k_qlmb(int n, const uint32_t *__restrict__ nbcount, const double *__restrict__ theta,
                       const double *__restrict__ fai, double2 *__restrict__ qlmb) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)n * 13) return;
    const int i = (int)(t / 13), m = (int)(t % 13) - 6;
    const unsigned Nb = nbcount[i];
    double re = 0.0, im = 0.0;
    if (Nb > 0 && Nb <= 16) {
        for (unsigned j = 0; j < Nb; ++j) {
            const float th = (float)theta[16L * i + j], fa = (float)fai[16L * i + j];
            re += (double)ylm_r(6, m, th, fa);
            im += (double)ylm_c(6, m, th, fa);
        }
        re = re / (double)(float)Nb;
        im = im / (double)(float)Nb;
    }
    qlmb[t] = make_double2(re, im);
}

// qlmbar and the per-atom sums of ELA:3181-3223 and 3264-3317 (two passes with l = 6
// accumulating into one sum).
__global__ void k_q46(int n, const uint32_t *__restrict__ nbcount, const int *__restrict__ nbidx,
                      const double2 *__restrict__ qlmb, double *__restrict__ q4, double *__restrict__ q6) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned Nb = nbcount[i];
    double t[13];
    for (int mm = 0; mm < 13; ++mm) {
        double br = 0.0, bi = 0.0;
        if (Nb > 0 && Nb <= 16) {
            for (unsigned j = 0; j < Nb; ++j) {
                const int jj = nbidx[16L * i + j];
                br += qlmb[13L * jj + mm].x;
                bi += qlmb[13L * jj + mm].y;
            }
            br = (qlmb[13L * i + mm].x + br) / (double)(float)(Nb + 1);
            bi = (qlmb[13L * i + mm].y + bi) / (double)(float)(Nb + 1);
        }
        t[mm] = br * br + bi * bi;
    }
    const double xishu = 4 * PI_REF / (double)(float)(2 * 6 + 1);
    double s = 0.0;
    for (int mm = 0; mm < 13; ++mm) s += t[mm];
    q4[i] = sqrt(xishu * s);
    for (int mm = 0; mm < 13; ++mm) s += t[mm];
    q6[i] = sqrt(xishu * s);
}

int elastic3d_dev(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                  float benchel, double *strain, uint32_t *nb, cudaStream_t st) {
    if (n <= 0) return PFC_OK;
    const float fx = (float)L * dx, fy = (float)M * dx, fz = (float)N * dx;
    k_elastic3d<<<(n + 7) / 8, 256, 0, st>>>(x, y, z, n, fx, fy, fz, benchel, strain, nb);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFC_OK : cuda_error(e, "k_elastic3d");
}

int cryst_order_dev(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                    double *q4, double *q6, cudaStream_t st) {
    if (n <= 0) return PFC_OK;
    const float fx = (float)L * dx, fy = (float)M * dx, fz = (float)N * dx;
    char *mem = nullptr;
    const size_t bytes = (size_t)n * (4 + 16 * 4 + 16 * 8 * 2 + 13 * 16) + 1024;
    cudaError_t e = cudaMallocAsync(&mem, bytes, st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync cryst_order");
    cudaMemsetAsync(mem, 0, bytes, st);
    double *theta = (double *)mem;
    double *fai = theta + 16L * n;
    double2 *qlmb = (double2 *)(fai + 16L * n);
    int *nbidx = (int *)(qlmb + 13L * n);
    uint32_t *nbc = (uint32_t *)(nbidx + 16L * n);
    k_cryst_neighbours<<<(n + 7) / 8, 256, 0, st>>>(x, y, z, n, fx, fy, fz, nbc, nbidx, theta, fai);
    k_qlmb<<<(unsigned)((13L * n + 255) / 256), 256, 0, st>>>(n, nbc, theta, fai, qlmb);
    k_q46<<<(n + 127) / 128, 128, 0, st>>>(n, nbc, nbidx, qlmb, q4, q6);
    e = cudaGetLastError();
    cudaFreeAsync(mem, st);
    return e == cudaSuccess ? PFC_OK : cuda_error(e, "cryst_order kernels");
}

// ---------------------------------------------------------------------------
// CVD checkpoint analysis (CVD:1067-1520): the atompositionCFGC2 peak finder, the GR
// pair-distance histogram and Q6_GLO.  All float arithmetic is the reference's (this
// file is compiled without FMA contraction).
// ---------------------------------------------------------------------------

// Peak finder of CVD:1112-1165 on a single rank: buffer planes 0 and L+1 are copies
// of the first and last plane (the MPI_Sendrecv stub, pfc_common.h:101-110); a point
// >= phic is an atom when it is >= its neighbours at flat buffer offsets +-N*M, +-N
// and +-1 (no wrap: at the ends of a row the neighbour is in the adjacent row).
// Emission index o = natural index n + N*(m + M*p), buffer plane p + 1.
struct CvdPeak {
    const float *phi;
    const float *stats;  // device [phic, phimax]
    int L, M, N;
    float dx;
    __device__ __forceinline__ float buf(long idx) const {
        const long slab = (long)M * N;
        long row = idx / slab - 1;
        row = row < 0 ? 0 : (row > L - 1 ? L - 1 : row);
        return phi[row * slab + idx % slab];
    }
    __device__ bool test(long o) const {
        const long slab = (long)M * N, idx = o + slab;
        const float v = phi[o];
        if (!(v >= stats[0])) return false;
        if (!(v >= buf(idx - slab) && v >= buf(idx + slab))) return false;
        if (!(v >= buf(idx - N) && v >= buf(idx + N))) return false;
        return v >= buf(idx - 1) && v >= buf(idx + 1);
    }
    // (pc_x, pc_y, pc_z, pc_phi) of CVD:1152-1155: fractional y, z and x positions
    __device__ void record(long o, double *out) const {
        const int n = (int)(o % N), m = (int)((o / N) % M), p = (int)(o / ((long)N * M));
        const float fx = __fmul_rn((float)L, dx), fy = __fmul_rn((float)M, dx), fz = __fmul_rn((float)N, dx);
        out[0] = (double)__fdiv_rn(__fmul_rn((float)(m + 1), dx), fy);
        out[1] = (double)__fdiv_rn(__fmul_rn((float)(n + 1), dx), fz);
        out[2] = (double)__fdiv_rn(__fmul_rn((float)(p + 1), dx), fx);
        out[3] = (double)phi[o];
    }
    static constexpr int REC = 4;
};

// phimax starts at phimm = -1 (CVD:58, 1077); phic = u0 + (phimax - u0) * phi_rat.
__global__ void k_cvd_stats(const float *phi, long n, float u0, float *stats) {
    __shared__ float red[32];
    float m = -1.0f;
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        const float v = phi[i];
        if (v > m) m = v;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float o = __shfl_down_sync(0xffffffffu, m, off);
        if (o > m) m = o;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = -1.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (red[w] > s) s = red[w];
        stats[0] = __fadd_rn(u0, __fmul_rn(__fsub_rn(s, u0), 0.618f));
        stats[1] = s;
    }
}

// Pair geometry of GR and Q6_GLO (CVD:1297-1310): float differences of the records
// scaled by the frame of each slot, minimum image, rr = sqrt(...) + 1e-6 added in
// double and stored to float.
struct CvdPair {
    float r3[9];
    float drx, dry, drz, rr;
};
__device__ __forceinline__ void cvd_pair(float xi, float yi, float zi, float xj, float yj, float zj, float fx, float fy,
                                         float fz, CvdPair &g) {
    g.r3[0] = __fmul_rn(__fsub_rn(xi, xj), fx);
    g.r3[1] = __fmul_rn(__fsub_rn(yi, yj), fy);
    g.r3[2] = __fmul_rn(__fsub_rn(zi, zj), fz);
    g.r3[3] = __fadd_rn(g.r3[0], fx);
    g.r3[4] = __fadd_rn(g.r3[1], fy);
    g.r3[5] = __fadd_rn(g.r3[2], fz);
    g.r3[6] = __fsub_rn(g.r3[0], fx);
    g.r3[7] = __fsub_rn(g.r3[1], fy);
    g.r3[8] = __fsub_rn(g.r3[2], fz);
    g.drx = min3f(g.r3[0], g.r3[3], g.r3[6]);
    g.dry = min3f(g.r3[1], g.r3[4], g.r3[7]);
    g.drz = min3f(g.r3[2], g.r3[5], g.r3[8]);
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(g.drx, g.drx), __fmul_rn(g.dry, g.dry)), __fmul_rn(g.drz, g.drz));
    g.rr = __double2float_rn(__dadd_rn((double)__fsqrt_rn(s), 1e-6));
}

// GR histogram (CVD:1293-1311): pairs i < j over upper-triangle tiles of 256 x 256
// records; counts go to a shared-memory histogram, then to the global one (integer
// additions, so the result does not depend on the order).
constexpr int GR_TILE = 256;
__global__ void k_cvd_gr(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z, int n,
                         int tiles, float fx, float fy, float fz, float delr, int maxbin, double rmin,
                         unsigned *__restrict__ hist) {
    extern __shared__ unsigned sh[];
    float *jx = reinterpret_cast<float *>(sh + maxbin), *jy = jx + GR_TILE, *jz = jy + GR_TILE;
    int bi = 0, rem = blockIdx.x;
    while (rem >= tiles - bi) {
        rem -= tiles - bi;
        ++bi;
    }
    const int bj = bi + rem;
    for (int b = threadIdx.x; b < maxbin; b += blockDim.x) sh[b] = 0u;
    const int j0 = bj * GR_TILE;
    for (int t = threadIdx.x; t < GR_TILE; t += blockDim.x) {
        const int j = j0 + t;
        jx[t] = j < n ? x[j] : 0.f;
        jy[t] = j < n ? y[j] : 0.f;
        jz[t] = j < n ? z[j] : 0.f;
    }
    __syncthreads();
    const int i = bi * GR_TILE + threadIdx.x;
    if (i < n) {
        const float xi = x[i], yi = y[i], zi = z[i];
        const int jend = min(GR_TILE, n - j0);
        for (int t = 0; t < jend; ++t) {
            if (j0 + t <= i) continue;
            CvdPair g;
            cvd_pair(xi, yi, zi, jx[t], jy[t], jz[t], fx, fy, fz, g);
            const unsigned bin = (unsigned)(int)__fdiv_rn(g.rr, delr);
            if ((double)g.rr > rmin && bin < (unsigned)maxbin) atomicAdd(&sh[bin], 2u);
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < maxbin; b += blockDim.x)
        if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// Q6_GLO neighbour lists (CVD:1376-1419): one warp per record i scans j in ascending
// chunks of 32; every j != i with rr in [rlo, rhi] counts, the first 24 are kept.
constexpr int Q6_CN = 24;
__global__ void k_cvd_q6_neighbours(const float *__restrict__ x, const float *__restrict__ y,
                                    const float *__restrict__ z, int n, float fx, float fy, float fz, double rlo,
                                    double rhi, unsigned *__restrict__ nbcount, int *__restrict__ nbidx) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * 8 + warp;
    if (i >= n) return;
    const float xi = x[i], yi = y[i], zi = z[i];
    unsigned Nb = 0;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        bool ok = false;
        if (j < n && j != i) {
            CvdPair g;
            cvd_pair(xi, yi, zi, x[j], y[j], z[j], fx, fy, fz, g);
            ok = (double)g.rr <= rhi && (double)g.rr >= rlo;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const unsigned slot = Nb + __popc(bal & ((1u << lane) - 1u));
            if (slot < Q6_CN) nbidx[(long)Q6_CN * i + slot] = j;
        }
        Nb += __popc(bal);
    }
    if (lane == 0) nbcount[i] = Nb;
}

// Per record i (CVD:1435-1482): neighbour angles theta, fai and, for m = -6..6, the
// neighbour average of Y_6m (qre, qim) and the float sum over m of |qlmb|^2 that gives
// the local Q6.  Records with no neighbour or more than 24 contribute zeros.
__global__ void k_cvd_q6_atoms(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                               int n, float fx, float fy, float fz, const unsigned *__restrict__ nbcount,
                               const int *__restrict__ nbidx, double2 *__restrict__ qlmb, float *__restrict__ ql) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned Nb = nbcount[i];
    const bool use = Nb > 0 && Nb <= (unsigned)Q6_CN;
    float th[Q6_CN], fa[Q6_CN];
    const float xi = x[i], yi = y[i], zi = z[i];
    if (use) {
        for (unsigned k = 0; k < Nb; ++k) {
            const int j = nbidx[(long)Q6_CN * i + k];
            CvdPair g;
            cvd_pair(xi, yi, zi, x[j], y[j], z[j], fx, fy, fz, g);
            // CoX/CoY/CoZ (CVD:1403-1412): the last image whose |offset| is within 1e-5
            float rjx = 0.f, rjy = 0.f, rjz = 0.f;
            for (int ii = 0; ii < 7; ii += 3)
                if ((double)__fsub_rn(fabsf(g.r3[ii]), g.drx) < 1e-5) rjx = __fsub_rn(__fmul_rn(xi, fx), g.r3[ii]);
            for (int ii = 1; ii < 8; ii += 3)
                if ((double)__fsub_rn(fabsf(g.r3[ii]), g.dry) < 1e-5) rjy = __fsub_rn(__fmul_rn(yi, fy), g.r3[ii]);
            for (int ii = 2; ii < 9; ii += 3)
                if ((double)__fsub_rn(fabsf(g.r3[ii]), g.drz) < 1e-5) rjz = __fsub_rn(__fmul_rn(zi, fz), g.r3[ii]);
            th[k] = acosf(__fdiv_rn(__fsub_rn(rjz, __fmul_rn(zi, fz)), g.rr));
            const float dyv = __fsub_rn(rjy, __fmul_rn(yi, fy));
            fa[k] = dyv == 0.f ? 0.f : atanf(__fdiv_rn(dyv, __fsub_rn(rjx, __fmul_rn(xi, fx))));
        }
    }
    float acc = 0.f;
    for (int mm = 0; mm < 13; ++mm) {
        double re = 0.0, im = 0.0;
        if (use) {
            for (unsigned k = 0; k < Nb; ++k) {
                re += (double)ylm_r(6, mm - 6, th[k], fa[k]);
                im += (double)ylm_c(6, mm - 6, th[k], fa[k]);
            }
            re = re / (double)(float)Nb;
            im = im / (double)(float)Nb;
        }
        qlmb[13L * i + mm] = make_double2(re, im);
        acc = __double2float_rn(__dadd_rn((double)acc, __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im))));
    }
    const float xishu = __double2float_rn(4 * PI_REF / (double)(float)13);
    ql[i] = __fsqrt_rn(__fmul_rn(xishu, acc));
}

// Global Q6 (CVD:1484-1497): for each m one thread adds the records in order, with
// the reference's float accumulators; then the 13 terms are summed in m order.
__global__ void k_cvd_q6_global(int n, const unsigned *__restrict__ nbcount, const double2 *__restrict__ qlmb,
                                float *__restrict__ out) {
    __shared__ float term[13];
    const int mm = threadIdx.x;
    if (mm < 13) {
        float qr = 0.f, qc = 0.f, sum = 0.f;
        for (int i = 0; i < n; ++i) {
            const double2 q = qlmb[13L * i + mm];
            const double nb = (double)nbcount[i];
            qr = __double2float_rn(__dadd_rn((double)qr, __dmul_rn(nb, q.x)));
            qc = __double2float_rn(__dadd_rn((double)qc, __dmul_rn(nb, q.y)));
            sum = __fadd_rn(sum, (float)nbcount[i]);
        }
        qr = __fdiv_rn(qr, sum);
        qc = __fdiv_rn(qc, sum);
        term[mm] = __fadd_rn(__fmul_rn(qr, qr), __fmul_rn(qc, qc));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float qm = 0.f;
        for (int k = 0; k < 13; ++k) qm = __fadd_rn(qm, term[k]);
        const float xishu = __double2float_rn(4 * PI_REF / (double)(float)13);
        out[0] = __fsqrt_rn(__fmul_rn(xishu, qm));
    }
}

int cvd_atoms_dev(const float *d_phi, int L, int M, int N, float dx, float u0, double *d_out, int cap, int *count,
                  float *stats_host, cudaStream_t st) {
    float *stats = nullptr;
    cudaError_t e = cudaMallocAsync(&stats, 2 * sizeof(float), st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync CVD stats");
    const long P = (long)L * M * N;
    k_cvd_stats<<<1, 1024, 0, st>>>(d_phi, P, u0, stats);
    CvdPeak f{d_phi, stats, L, M, N, dx};
    int rc = compact(f, P, d_out, cap, count, st);
    if (rc == PFC_OK) {
        e = cudaMemcpyAsync(stats_host, stats, 2 * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_error(e, "CVD stats copy");
    }
    cudaFreeAsync(stats, st);
    return rc;
}

// x, y, z: device records; hist: device [maxbin], zeroed here.
int cvd_gr_dev(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, unsigned *hist,
               int maxbin, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(unsigned) * (size_t)maxbin, st);
    if (e != cudaSuccess) return cuda_error(e, "GR histogram clear");
    if (n < 2) return PFC_OK;
    const float fx = (float)L * dx, fy = (float)M * dx, fz = (float)N * dx;
    const float delr = (float)(1.0f / 25.);
    const int tiles = (n + GR_TILE - 1) / GR_TILE;
    const long blocks = (long)tiles * (tiles + 1) / 2;
    const size_t smem = sizeof(unsigned) * (size_t)maxbin + 3 * GR_TILE * sizeof(float);
    static unsigned attr_mask = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (smem > 48 * 1024 && !(attr_mask & (1u << dev))) {
        e = cudaFuncSetAttribute(k_cvd_gr, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return cuda_error(e, "GR shared memory");
        attr_mask |= 1u << dev;
    }
    if (smem > 200 * 1024) return set_error(PFC_E_INVALID, "GR histogram too large for shared memory");
    k_cvd_gr<<<(unsigned)blocks, GR_TILE, smem, st>>>(x, y, z, n, tiles, fx, fy, fz, delr, maxbin,
                                                     (double)1.0f / sqrt(2.) * 0.5, hist);
    e = cudaGetLastError();
    return e == cudaSuccess ? PFC_OK : cuda_error(e, "k_cvd_gr");
}

// x, y, z: device records; nb, ql: device [n]; *ql_global_host receives the global Q6.
int cvd_q6_dev(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, unsigned *nb,
               float *ql, float *ql_global_host, cudaStream_t st) {
    if (n <= 0) return PFC_OK;
    const float fx = (float)L * dx, fy = (float)M * dx, fz = (float)N * dx;
    char *mem = nullptr;
    const size_t bytes = (size_t)n * (Q6_CN * sizeof(int) + 13 * sizeof(double2)) + 256;
    cudaError_t e = cudaMallocAsync(&mem, bytes, st);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync Q6");
    double2 *qlmb = (double2 *)mem;
    int *nbidx = (int *)(qlmb + 13L * n);
    float *glob = (float *)(nbidx + (long)Q6_CN * n);
    const double rhi = (double)1.0f * sqrt(3.) / 2. * 1.2 + 1e-3, rlo = (double)1.0f * sqrt(3.) / 2. * 0.9 - 1e-3;
    k_cvd_q6_neighbours<<<(n + 7) / 8, 256, 0, st>>>(x, y, z, n, fx, fy, fz, rlo, rhi, nb, nbidx);
    k_cvd_q6_atoms<<<(n + 127) / 128, 128, 0, st>>>(x, y, z, n, fx, fy, fz, nb, nbidx, qlmb, ql);
    k_cvd_q6_global<<<1, 32, 0, st>>>(n, nb, qlmb, glob);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(ql_global_host, glob, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(mem, st);
    return e == cudaSuccess ? PFC_OK : cuda_error(e, "Q6 kernels");
}

}  // namespace pfc

using namespace pfc;

// ---------------------------------------------------------------------------
// C ABI (host buffers in, host buffers out)
// ---------------------------------------------------------------------------
namespace {
// A device buffer of one host-array call, taken from the device's default memory pool in
// stream order and returned to it the same way (the pool keeps freed memory, so repeated
// calls do not map and unmap device memory; get_context sets that).
struct DevBuf {
    void *p = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t alloc(size_t bytes, cudaStream_t s) {
        st = s;
        return cudaMallocAsync(&p, bytes, s);
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, st);
    }
};
int host_ctx(cudaStream_t *st) {
    int dev = 0;
    cudaGetDevice(&dev);
    Context *c = nullptr;
    int rc = get_context(dev, &c);
    if (rc != PFC_OK) return rc;
    *st = c->stream;
    return PFC_OK;
}
}  // namespace

#define ATRY(expr)                                           \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return cuda_error(_e, #expr); \
    } while (0)

extern "C" int pfc_phimax_misfit(const float *phi, const float *con, int L, int M, float dx, float con0, double *out5,
                                 int cap, int *count) {
    if (!phi || !con || !count || L <= 0 || M <= 0 || cap < 0 || (cap > 0 && !out5))
        return set_error(PFC_E_INVALID, "bad arguments to pfc_phimax_misfit");
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    const long P = (long)L * M;
    DevBuf f, o;
    ATRY(f.alloc(2 * P * sizeof(float), st));
    ATRY(o.alloc((size_t)(cap > 0 ? cap : 1) * 5 * sizeof(double), st));
    float *dphi = (float *)f.p, *dcon = dphi + P;
    ATRY(cudaMemcpyAsync(dphi, phi, P * sizeof(float), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(dcon, con, P * sizeof(float), cudaMemcpyHostToDevice, st));
    rc = phimax_misfit_dev(dphi, dcon, L, M, dx, con0, (double *)o.p, cap, count, nullptr, st);
    if (rc != PFC_OK) return rc;
    const int k = *count < cap ? *count : cap;
    if (k > 0) ATRY(cudaMemcpyAsync(out5, o.p, (size_t)k * 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    return PFC_OK;
}

extern "C" int pfc_phimax_elastic(const float *phi, int L, int M, int N, float dx, double *out4, int cap, int *count) {
    if (!phi || !count || L <= 0 || M <= 0 || N <= 0 || cap < 0 || (cap > 0 && !out4))
        return set_error(PFC_E_INVALID, "bad arguments to pfc_phimax_elastic");
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    const long P = (long)L * M * N;
    DevBuf f, o;
    ATRY(f.alloc(P * sizeof(float), st));
    ATRY(o.alloc((size_t)(cap > 0 ? cap : 1) * 4 * sizeof(double), st));
    ATRY(cudaMemcpyAsync(f.p, phi, P * sizeof(float), cudaMemcpyHostToDevice, st));
    rc = phimax_elastic_dev((const float *)f.p, L, M, N, dx, (double *)o.p, cap, count, st);
    if (rc != PFC_OK) return rc;
    const int k = *count < cap ? *count : cap;
    if (k > 0) ATRY(cudaMemcpyAsync(out4, o.p, (size_t)k * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    return PFC_OK;
}

extern "C" int pfc_cvd_atoms(const float *phi, int L, int M, int N, float dx, float u0, float *out4, int cap,
                             int *count, float *phic, float *phimax) {
    if (!phi || !count || L <= 0 || M <= 0 || N <= 0 || cap < 1 || !out4)
        return set_error(PFC_E_INVALID, "bad arguments to pfc_cvd_atoms");
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    const long P = (long)L * M * N;
    DevBuf f, o;
    ATRY(f.alloc(P * sizeof(float), st));
    ATRY(o.alloc((size_t)cap * 4 * sizeof(double), st));
    ATRY(cudaMemcpyAsync(f.p, phi, P * sizeof(float), cudaMemcpyHostToDevice, st));
    float stats[2];
    rc = cvd_atoms_dev((const float *)f.p, L, M, N, dx, u0, (double *)o.p, cap, count, stats, st);
    if (rc != PFC_OK) return rc;
    if (phic) *phic = stats[0];
    if (phimax) *phimax = stats[1];
    const int k = *count < cap ? *count : cap;
    std::vector<double> rec((size_t)k * 4);
    if (k > 0) ATRY(cudaMemcpyAsync(rec.data(), o.p, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < rec.size(); ++i) out4[i] = (float)rec[i];  // the records hold float values
    if (*count == 0) {  // the reference's "no atoms" record (CVD:1169)
        out4[0] = out4[1] = out4[2] = -1.0f;
        out4[3] = 0.0f;
        *count = 1;
    }
    return PFC_OK;
}

static int upload_records(const float *x, const float *y, const float *z, int n, DevBuf &b, cudaStream_t st) {
    ATRY(b.alloc((size_t)3 * n * sizeof(float) + 16, st));
    float *d = (float *)b.p;
    ATRY(cudaMemcpyAsync(d, x, n * sizeof(float), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(d + n, y, n * sizeof(float), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(d + 2 * n, z, n * sizeof(float), cudaMemcpyHostToDevice, st));
    return PFC_OK;
}

extern "C" int pfc_cvd_gr_hist(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx,
                               uint32_t *hist, int cap, int *maxbin) {
    if (!x || !y || !z || n < 0 || !hist || !maxbin || L <= 0 || M <= 0 || N <= 0 || !(dx > 0.0f))
        return set_error(PFC_E_INVALID, "bad arguments to pfc_cvd_gr_hist");
    const float delr = (float)(1.0f / 25.);
    const int mb = (int)(((float)L * dx) / delr);
    if (mb > cap) return set_error(PFC_E_INVALID, "histogram capacity below maxbin");
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    DevBuf r, h;
    rc = upload_records(x, y, z, n > 0 ? n : 1, r, st);
    if (rc != PFC_OK) return rc;
    ATRY(h.alloc(sizeof(unsigned) * (size_t)(mb > 0 ? mb : 1), st));
    const float *d = (const float *)r.p;
    const int nn = n > 0 ? n : 1;
    rc = cvd_gr_dev(d, d + nn, d + 2 * nn, n, L, M, N, dx, (unsigned *)h.p, mb, st);
    if (rc != PFC_OK) return rc;
    if (mb > 0) ATRY(cudaMemcpyAsync(hist, h.p, sizeof(unsigned) * mb, cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    *maxbin = mb;
    return PFC_OK;
}

extern "C" int pfc_cvd_q6(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx,
                          uint32_t *nb, float *ql, float *ql_global) {
    if (!x || !y || !z || n < 0 || !nb || !ql || !ql_global || L <= 0 || M <= 0 || N <= 0)
        return set_error(PFC_E_INVALID, "bad arguments to pfc_cvd_q6");
    if (n == 0) {
        *ql_global = std::numeric_limits<float>::quiet_NaN();  // the reference divides 0 by 0
        return PFC_OK;
    }
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    DevBuf r, o;
    rc = upload_records(x, y, z, n, r, st);
    if (rc != PFC_OK) return rc;
    ATRY(o.alloc((size_t)n * (sizeof(unsigned) + sizeof(float)), st));
    const float *d = (const float *)r.p;
    unsigned *dnb = (unsigned *)o.p;
    float *dql = (float *)(dnb + n);
    rc = cvd_q6_dev(d, d + n, d + 2 * n, n, L, M, N, dx, dnb, dql, ql_global, st);
    if (rc != PFC_OK) return rc;
    ATRY(cudaMemcpyAsync(nb, dnb, n * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    ATRY(cudaMemcpyAsync(ql, dql, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    return PFC_OK;
}

extern "C" int pfc_elastic3d(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                             float benchel, double *strain, uint32_t *nb) {
    if (n < 0 || (n > 0 && (!x || !y || !z || !strain || !nb))) return set_error(PFC_E_INVALID, "bad arguments to pfc_elastic3d");
    if (n == 0) return PFC_OK;
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    DevBuf b;
    ATRY(b.alloc((size_t)n * (4 * sizeof(double) + sizeof(uint32_t)), st));
    double *dx_ = (double *)b.p, *dy = dx_ + n, *dz = dy + n, *ds = dz + n;
    uint32_t *dnb = (uint32_t *)(ds + n);
    ATRY(cudaMemcpyAsync(dx_, x, n * sizeof(double), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(dy, y, n * sizeof(double), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(dz, z, n * sizeof(double), cudaMemcpyHostToDevice, st));
    rc = elastic3d_dev(dx_, dy, dz, n, L, M, N, dx, benchel, ds, dnb, st);
    if (rc != PFC_OK) return rc;
    ATRY(cudaMemcpyAsync(strain, ds, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATRY(cudaMemcpyAsync(nb, dnb, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    return PFC_OK;
}

extern "C" int pfc_cryst_order(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                               double *q4, double *q6) {
    if (n < 0 || (n > 0 && (!x || !y || !z || !q4 || !q6))) return set_error(PFC_E_INVALID, "bad arguments to pfc_cryst_order");
    if (n == 0) return PFC_OK;
    cudaStream_t st;
    int rc = host_ctx(&st);
    if (rc != PFC_OK) return rc;
    DevBuf b;
    ATRY(b.alloc((size_t)n * 5 * sizeof(double), st));
    double *dx_ = (double *)b.p, *dy = dx_ + n, *dz = dy + n, *d4 = dz + n, *d6 = d4 + n;
    ATRY(cudaMemcpyAsync(dx_, x, n * sizeof(double), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(dy, y, n * sizeof(double), cudaMemcpyHostToDevice, st));
    ATRY(cudaMemcpyAsync(dz, z, n * sizeof(double), cudaMemcpyHostToDevice, st));
    rc = cryst_order_dev(dx_, dy, dz, n, L, M, N, dx, d4, d6, st);
    if (rc != PFC_OK) return rc;
    ATRY(cudaMemcpyAsync(q4, d4, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATRY(cudaMemcpyAsync(q6, d6, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ATRY(cudaStreamSynchronize(st));
    return PFC_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free Misfit peak finder.
//
// For callers that cannot allocate device memory: a serving loop whose admission
// controller has already committed the whole HBM budget to resident runs, or a
// host thread that must not trigger the device-wide synchronisation that cudaMalloc
// and cudaFree imply while other streams are busy.  The caller passes device
// buffers for the fields and the atoms; the compaction's per-block counts and
// offsets live in the file-scope array below, sized for fields of up to
// PFC_NOALLOC_MAX_POINTS points (2048 x 2048).  Every GPU that loads the library
// holds the array (about 32 KB) until the process exits.
// ---------------------------------------------------------------------------
namespace pfc {
static constexpr long NOALLOC_MAX_POINTS = 2048L * 2048L;
static constexpr int NOALLOC_MAX_BLOCKS = (int)((NOALLOC_MAX_POINTS + CSPAN - 1) / CSPAN);
// block counts [0, nb), exclusive offsets [nb, 2nb) and the total at [2nb]
static __device__ __align__(256) int g_noalloc_scratch[2 * NOALLOC_MAX_BLOCKS + 2];
static std::mutex g_noalloc_mu;
static int *g_noalloc_addr[64] = {nullptr};  // device address of g_noalloc_scratch, per device ordinal
}  // namespace pfc

extern "C" int pfc_phimax_misfit_noalloc(const float *d_phi, const float *d_con, int L, int M, float dx, float con0,
                                         double *d_out5, int cap, int *count, void *stream) {
    using namespace pfc;
    if (!d_phi || !d_con || !count || L <= 0 || M <= 0 || cap < 0 || (cap > 0 && !d_out5))
        return set_error(PFC_E_INVALID, "bad arguments to pfc_phimax_misfit_noalloc");
    const long n = (long)L * M;
    if (n > NOALLOC_MAX_POINTS)
        return set_error(PFC_E_INVALID, "pfc_phimax_misfit_noalloc: L*M = " + std::to_string(n) +
                                            " exceeds the allocation-free limit of 4194304 points (2048 x 2048)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_error(PFC_E_INVALID, "device ordinal beyond 63");
    int *scratch = nullptr;
    {
        // first call on this device: look up the array's device address (host code
        // cannot use the symbol itself as a device pointer)
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            e = cudaGetSymbolAddress((void **)&g_noalloc_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
            }
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = (int)((n + CSPAN - 1) / CSPAN);
    // k_count writes every count and k_scan every offset and the total before they
    // are read, so nothing left by an earlier call needs clearing.
    MisfitPeak f{d_phi, d_con, L, M, dx, con0};
    k_count<<<nb, CBLK, 0, st>>>(f, n, scratch);
    k_scan<<<1, 1024, 0, st>>>(scratch, nb, scratch + nb);
    k_emit<<<nb, CBLK, 0, st>>>(f, n, scratch + nb, d_out5, cap);
    int total = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, scratch + 2 * nb, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "pfc_phimax_misfit_noalloc");
    if (total == 0) {
        if (cap > 0) k_misfit_fallback<<<1, 32, 0, st>>>(d_phi, d_con, L, M, dx, con0, d_out5);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_error(e, "pfc_phimax_misfit_noalloc fallback");
        total = 1;
    }
    *count = total;
    return PFC_OK;
}
