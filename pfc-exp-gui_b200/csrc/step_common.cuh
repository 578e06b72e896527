// step_common.cuh -- pieces of the fused FP32 step (step_fp32.cu) that do not depend on
// its kernels: tile geometry, the C2 kernel as the reference's float table holds it,
// and launch helpers.
#pragma once

#include "fft_core.cuh"
#include "pfc_internal.h"
#include "tile_io.cuh"

namespace pfc {

constexpr int COL_TILE = 4096;  // complex elements per column-kernel tile (32 KB in FP32)
constexpr int COL_TILE_MAX = 16;  // widest column tile (packed columns); the row walks' bound

// Column-kernel tile: L rows x C packed columns, C a power of two in [1, COL_TILE_MAX]
// with 512 <= C*L <= 8192 complex elements (three such buffers per CTA: 13 KB to 204 KB).
constexpr bool col_tile_ok(int L, int C) { return C >= 1 && C <= COL_TILE_MAX && C * L >= 512 && C * L <= 8192; }
// Column tile of the mixed-precision path: L rows x C packed columns, 512 <= C*L <= 4096
// complex values (its shared buffers hold double2).
constexpr bool mcol_tile_ok(int L, int C) { return C >= 1 && C <= COL_TILE_MAX && C * L >= 512 && C * L <= 4096; }
constexpr int MROW_TILE = 2048;  // complex doubles per mixed row-kernel CTA (row step: 2 sequences per row)
// Rows per mixed row-kernel CTA: MROW_TILE/2 points of rows, and at least two rows up to
// M = 1024, so that a CTA's loads of a width-2 column tile are whole 32-byte sectors.
constexpr int mrow_rpc(int M) {
    const int a = (MROW_TILE / 2) / M, b = 2048 / M < 2 ? 2048 / M : 2;
    return a > b ? a : (b > 1 ? b : 1);
}

template <int L, int C> struct ColCfg {
    static constexpr int NT = (C * L / 16) < 32 ? 32 : (C * L / 16);
    // CTAs per SM that the shared memory leaves room for (two at C*L = 4096)
    static constexpr int MINB = (8192 / (C * L)) > 8 ? 8 : ((8192 / (C * L)) < 1 ? 1 : 8192 / (C * L));
};

// C2 correlation kernel at |k| = sqrtf(ks), as the reference builds its float table
// (misfit_uniform_time_seed_fftw_early.cpp:700-750): exp in double of float arguments.
__device__ __forceinline__ float c2_ref(const C2Params &p, float ks) {
    const float s = __fsqrt_rn(ks);
    if (s <= p.kc) {
        const double d = (double)__fsub_rn(s, p.k1);
        return (float)(exp(-(double)p.q1 * (double)p.q1) * exp(-(d * d) / (double)p.gg1));
    }
    const double d = (double)__fsub_rn(s, p.k2);
    return (float)(exp(-(double)p.q2 * (double)p.q2) * exp(-(d * d) / (double)p.gg2));
}

// Double products and sums that the compiler never fuses into an fma or splits (the mixed
// path writes its pointwise arithmetic with these and explicit fma(), so that equal inputs
// round equally in every kernel and every inlined copy).
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Natural logarithm in double for the mixed path's pointwise terms, by the table-driven
// method of P. T. P. Tang (ACM TOMS 16(4):378-400, 1990): x = 2^e m with m in [1, 2),
// F = 1 + j/128 the breakpoint nearest m (j = 0 .. 128), and
//   log x = e ln2 + log F + log1p(r),  r = (m - F) / F,  |r| <= 2^-8,
// log1p(r) by its Taylor series through r^7 (truncation below 2^-59 relative).  m - F is
// exact (m and F are within a factor of two); tab[j] = (log F, 1/F) in double, built on
// the host (LOG_TABLE_SIZE entries).  Absolute error below 3e-16 on [1/2, 2], a few
// units in the last place elsewhere.  Zero, negative, subnormal, infinite and NaN
// arguments take log() itself (the IEEE special values the run's non-finite check sees).
__device__ __forceinline__ double log_tab(double x, const double2 *__restrict__ tab) {
    if (!(x >= 0x1p-1022 && x <= 0x1.fffffffffffffp+1023)) return log(x);
    const long long bits = __double_as_longlong(x);
    const int e = (int)(bits >> 52) - 1023;
    const long long mant = bits & 0x000fffffffffffffLL;
    const int j = (int)((mant + (1LL << 44)) >> 45);  // nearest multiple of 2^-7
    const double m = __longlong_as_double(mant | 0x3ff0000000000000LL);
    const double2 t = __ldg(tab + j);
    const double r = (m - (1.0 + (double)j * 0.0078125)) * t.y;
    double q = 1.0 / 7.0;
    q = fma(q, r, -1.0 / 6.0);
    q = fma(q, r, 0.2);
    q = fma(q, r, -0.25);
    q = fma(q, r, 1.0 / 3.0);
    q = fma(q, r, -0.5);
    const double p = fma(q * r, r, r);  // r + r^2 (-1/2 + r/3 - ...)
    return fma((double)e, 0.6931471805599453, t.x) + p;
}

// Row-space element (l, km) of a run: column-tile-major, ((km/CT)*L + l)*CT + km%CT.
__device__ __forceinline__ long rs_index(const RunDesc &d, int l, int km) {
    return ((long)(km >> d.lct) * d.L + l) * d.CT + (km & (d.CT - 1));
}

// Loop over the row-space elements (l0 + r, km), r < RPC, km <= M/2, in an order
// that walks each column tile's contiguous RPC*CT block: w -> (tile t, row r, col c).
// RPC and CT are powers of two, so the block split is a shift and a mask.
template <int n> struct ilog2 {
    static constexpr int value = n <= 1 ? 0 : 1 + ilog2<n / 2>::value;
};
template <> struct ilog2<1> {
    static constexpr int value = 0;
};
#define ROW_TILE_LOOP(RPC, H, NT, ...)                                     \
    {                                                                       \
        const int _ct = d.CT, _lct = d.lct;                                 \
        const int _lblk = ilog2<(RPC)>::value + _lct;                       \
        const int _total = d.T << _lblk;                                    \
        for (int w = threadIdx.x; w < _total; w += (NT)) {                  \
            const int t = w >> _lblk, rem = w & ((1 << _lblk) - 1);         \
            const int r = rem >> _lct, k = (t << _lct) + (rem & (_ct - 1)); \
            if (k > (H)) continue;                                          \
            const int l = l0 + r;                                           \
            (void)l;                                                        \
            __VA_ARGS__                                                     \
        }                                                                   \
    }

// Spectrum of the noise field at mode (l, km) of step t.  The reference draws real-space
// white noise with a sequential polar Box-Muller generator (Gauss, MIS:951-981) and
// transforms it (p5); the transform of white noise is itself white, so the modes are
// drawn here directly, with the distribution the reference's masks leave
// (MIS:1002-1003): re and im independent N(0, P/4), except at the four self-conjugate
// modes (l in {0, L/2}, km in {0, M/2}) where re ~ N(0, P) and im = 0; along the
// self-conjugate columns km = 0 and M/2, mode L - l is the conjugate of mode l.
// Stream: the two normals of canonical mode c = (t*L + l)*(M/2 + 1) + km come from
// Box-Muller of the splitmix64 outputs at positions 2c and 2c + 1 of the run's key.
static __device__ __forceinline__ unsigned long long sm64_out(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static __device__ float2 noise_mode(unsigned long long key, int t, int l, int km, int L, int M) {
    const int H = M / 2;
    bool conj = false;
    if ((km == 0 || km == H) && l > L / 2) {
        l = L - l;
        conj = true;
    }
    const unsigned long long c = ((unsigned long long)t * L + l) * (unsigned long long)(H + 1) + km;
    const unsigned long long g = 0x9E3779B97F4A7C15ULL;
    const unsigned long long w1 = sm64_out(key + (2 * c + 1) * g), w2 = sm64_out(key + (2 * c + 2) * g);
    const float u1 = ((float)(w1 >> 40) + 0.5f) * (1.0f / 16777216.0f);  // (0, 1)
    const float u2 = (float)(w2 >> 40) * (1.0f / 16777216.0f);           // [0, 1)
    const float rad = sqrtf(-2.0f * logf(u1));
    float sn, cs;
    sincospif(2.0f * u2, &sn, &cs);
    const float P = (float)L * (float)M;
    if ((l == 0 || l == L / 2) && (km == 0 || km == H)) return make_float2(sqrtf(P) * rad * cs, 0.0f);
    const float s = 0.5f * sqrtf(P);
    return make_float2(s * rad * cs, conj ? -s * rad * sn : s * rad * sn);
}

static inline int log2i(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// Opt in to more than 48 KB of dynamic shared memory, once per kernel and device
// (the attribute call is not a stream operation, so it is also done before any
// graph capture through prepare_size()).
template <typename K> static inline cudaError_t set_smem(K kernel, size_t bytes, unsigned &mask) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (mask & (1u << dev)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) mask |= 1u << dev;
    return e;
}

template <int n> static constexpr size_t smem_bytes() { return sizeof(float2) * padded_len<n>::value; }

// Streaming multiprocessors of the current device (the persistent grid's width).
static inline int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

#define PFC_SIZE_SWITCH(n, FN, ...)             \
    switch (n) {                                \
        case 32: return FN<32>(__VA_ARGS__);    \
        case 64: return FN<64>(__VA_ARGS__);    \
        case 128: return FN<128>(__VA_ARGS__);  \
        case 256: return FN<256>(__VA_ARGS__);  \
        case 512: return FN<512>(__VA_ARGS__);  \
        case 1024: return FN<1024>(__VA_ARGS__); \
        case 2048: return FN<2048>(__VA_ARGS__); \
        default: return cudaErrorInvalidValue;  \
    }

}  // namespace pfc
