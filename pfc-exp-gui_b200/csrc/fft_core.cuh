// fft_core.cuh -- shared-memory Stockham FFT building blocks for sm_100a.
//
// The reference transforms every field with FFTW's complex 3-D DFT
// (src/experiment/misfit_uniform_time_seed_fftw_early.cpp:438-452, FFTW_ESTIMATE,
// unnormalised, exp(-2 pi i jk/n) forward).  Here the transforms are written from
// scratch: a batch of NB interleaved sequences of length N (element e of sequence b
// at index e*NB + b, so consecutive threads touch consecutive words) is transformed
// by Stockham stages of radix 16 (plus one radix-2/4/8 stage); each thread holds a
// fixed set of 16 complex values per stage in registers.  Natural order in and out.
//
// A stage reads its inputs from one place and writes its outputs to another:
// global memory (a contiguous tile with the same e*NB + b layout), shared memory
// (padded by one element per 16 to spread bank accesses), or registers.  The
// first stage of a transform can therefore load straight from HBM and the last
// can store straight to HBM or stay in registers for a pointwise epilogue.
//
// Twiddles come from a per-length table computed on the host in double and rounded
// once to the working precision, laid out by stage (twiddle_offset): the R factors
// exp(-2 pi i r k / (Ns R)), r < R, that one butterfly of a stage needs are
// contiguous, so an FP32 thread fetches them with R/2 16-byte loads; an FP64 thread
// loads the base factor r = 1 and forms the others (twiddle_powers).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace pfc {

// ---------------------------------------------------------------------------
// complex helpers (float2 / double2)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// The FP64 products are explicit fma() and __dmul_rn (never fused or split by the
// compiler), so a butterfly rounds the same way in every kernel that inlines it: two
// kernels that transform the same sequence give the same bits.
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -__dmul_rn(a.y, b.y)), fma(a.x, b.y, __dmul_rn(a.y, b.x)));
}
// multiply by conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, __dmul_rn(a.y, b.y)), fma(a.y, b.x, -__dmul_rn(a.x, b.y)));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// widen a stored value to the arithmetic type of a transform (float2 -> double2 for the
// mixed-precision path; the identity otherwise)
template <typename C> __device__ __forceinline__ C to_c(float2 v);
template <> __device__ __forceinline__ float2 to_c<float2>(float2 v) { return v; }
template <> __device__ __forceinline__ double2 to_c<double2>(float2 v) { return make_double2(v.x, v.y); }
template <typename C> __device__ __forceinline__ C to_c(double2 v) { return v; }

// multiply by -i (forward) or +i (inverse)
template <bool FWD, typename C> __device__ __forceinline__ C mul_mi(C a) {
    return FWD ? mk(a.y, -a.x) : mk(-a.y, a.x);
}

// shared-memory padding: one spare element per 16
__device__ __forceinline__ int spad(int i) { return i + (i >> 4); }
template <int n> struct padded_len {
    static constexpr int value = n + (n >> 4) + 1;
};

// ---------------------------------------------------------------------------
// Radix butterflies (in registers).  FWD uses exp(-2 pi i / R), inverse exp(+).
// ---------------------------------------------------------------------------
template <bool FWD, typename C> __device__ __forceinline__ void dft2(C &a0, C &a1) {
    C t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

template <bool FWD, typename C> __device__ __forceinline__ void dft4(C &a0, C &a1, C &a2, C &a3) {
    C t0 = cadd(a0, a2), t1 = csub(a0, a2);
    C t2 = cadd(a1, a3), t3 = mul_mi<FWD>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

template <typename R> struct kconst;
template <> struct kconst<float> {
    static __device__ __forceinline__ float h() { return 0.70710678118654752f; }
    static __device__ __forceinline__ float c8() { return 0.92387953251128674f; }
    static __device__ __forceinline__ float s8() { return 0.38268343236508977f; }
};
template <> struct kconst<double> {
    static __device__ __forceinline__ double h() { return 0.70710678118654752440; }
    static __device__ __forceinline__ double c8() { return 0.92387953251128675613; }
    static __device__ __forceinline__ double s8() { return 0.38268343236508977173; }
};

template <typename C> struct real_of;
template <> struct real_of<float2> { typedef float T; };
template <> struct real_of<double2> { typedef double T; };

// multiply by w8^k for k = 1, 3 where w8 = exp(-+2 pi i / 8)
template <bool FWD, typename C> __device__ __forceinline__ C w8_1(C a) {
    typedef typename real_of<C>::T R;
    const R h = kconst<R>::h();
    return FWD ? mk(h * (a.x + a.y), h * (a.y - a.x)) : mk(h * (a.x - a.y), h * (a.x + a.y));
}
template <bool FWD, typename C> __device__ __forceinline__ C w8_3(C a) {
    typedef typename real_of<C>::T R;
    const R h = kconst<R>::h();
    return FWD ? mk(h * (a.y - a.x), -h * (a.x + a.y)) : mk(-h * (a.x + a.y), h * (a.x - a.y));
}

template <bool FWD, typename C> __device__ __forceinline__ void dft8(C *a) {
    C e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    C o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<FWD>(e0, e1, e2, e3);
    dft4<FWD>(o0, o1, o2, o3);
    o1 = w8_1<FWD>(o1);
    o2 = mul_mi<FWD>(o2);
    o3 = w8_3<FWD>(o3);
    a[0] = cadd(e0, o0);
    a[4] = csub(e0, o0);
    a[1] = cadd(e1, o1);
    a[5] = csub(e1, o1);
    a[2] = cadd(e2, o2);
    a[6] = csub(e2, o2);
    a[3] = cadd(e3, o3);
    a[7] = csub(e3, o3);
}

// (a.x c + a.y s, a.y c - a.x s): a rotated by exp(-i theta), c = cos, s = sin
__device__ __forceinline__ float2 rot(float2 a, float c, float s) { return mk(a.x * c + a.y * s, a.y * c - a.x * s); }
__device__ __forceinline__ double2 rot(double2 a, double c, double s) {
    return mk(fma(a.x, c, __dmul_rn(a.y, s)), fma(a.y, c, -__dmul_rn(a.x, s)));
}

// multiply by w16^j (j = n2*k1 in 0..9), w16 = exp(-+2 pi i / 16)
template <bool FWD, typename C> __device__ __forceinline__ C w16(C a, int j) {
    typedef typename real_of<C>::T R;
    const R c1 = kconst<R>::c8(), s1 = kconst<R>::s8(), h = kconst<R>::h();
    R c, s;  // exp(-i theta) = c - i s with theta = 2 pi j / 16
    switch (j) {
        case 0: return a;
        case 1: c = c1; s = s1; break;
        case 2: c = h; s = h; break;
        case 3: c = s1; s = c1; break;
        case 4: return mul_mi<FWD>(a);
        case 5: c = -s1; s = c1; break;
        case 6: c = -h; s = h; break;
        case 7: c = -c1; s = s1; break;
        case 8: return mk(-a.x, -a.y);
        default: c = -c1; s = -s1; break;  // 9
    }
    if (!FWD) s = -s;
    return rot(a, c, s);
}

template <bool FWD, typename C> __device__ __forceinline__ void dft16(C *a) {
    // 16 = 4 x 4: X[k1 + 4 k2] = sum_n2 w4^(n2 k2) w16^(n2 k1) sum_n1 a[4 n1 + n2] w4^(n1 k1)
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<FWD>(a[n2], a[n2 + 4], a[n2 + 8], a[n2 + 12]);
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) a[n2 + 4 * k1] = w16<FWD>(a[n2 + 4 * k1], n2 * k1);
    C b[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C x0 = a[0 + 4 * k1], x1 = a[1 + 4 * k1], x2 = a[2 + 4 * k1], x3 = a[3 + 4 * k1];
        dft4<FWD>(x0, x1, x2, x3);
        b[k1 + 0] = x0;
        b[k1 + 4] = x1;
        b[k1 + 8] = x2;
        b[k1 + 12] = x3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = b[i];
}

template <int R, bool FWD, typename C> __device__ __forceinline__ void dftR(C *a) {
    if constexpr (R == 2) dft2<FWD>(a[0], a[1]);
    else if constexpr (R == 4) dft4<FWD>(a[0], a[1], a[2], a[3]);
    else if constexpr (R == 8) dft8<FWD>(a);
    else if constexpr (R == 16) dft16<FWD>(a);
}

// ---------------------------------------------------------------------------
// Radix plan: N = RM^a * r with RM the main radix and r < RM a power of two; the small
// radix comes last.  The main radix may follow the element type (main_radix); it is 16
// for both FP32 and FP64.  (FP64 transforms were measured with radix 8 too: twice the
// threads and half the registers per thread, but the extra shared-memory stage made
// the mixed step 8 % slower at 1024^2.)
// ---------------------------------------------------------------------------
template <typename C> struct main_radix {
    static constexpr int value = 16;
};
__host__ __device__ constexpr int clog2(int n) { return n <= 1 ? 0 : 1 + clog2(n / 2); }
template <int N, int RM = 16> struct radix_plan {
    static constexpr int log2n = clog2(N);
    static constexpr int lr = clog2(RM);
    static constexpr int nmain = log2n / lr;
    static constexpr int tail = 1 << (log2n % lr);
    static constexpr int stages = nmain + (tail > 1 ? 1 : 0);
    static constexpr int last_radix = tail > 1 ? tail : (log2n == 0 ? 1 : RM);
};

template <int N, int NB, int NT, int R> struct StageShape {
    static constexpr int ITEMS = NB * (N / R);
    static constexpr int PER_T = (ITEMS + NT - 1) / NT;
    static constexpr bool EXACT = ITEMS % NT == 0;
};

// FP32 twiddle table of one length (radix-16 plans): every stage but the first (which has
// Ns = 1 and no twiddles) owns Ns*R entries, entry k*R + r = exp(-2 pi i r k / (Ns R)).
// All stages before the last have radix 16, so the stage with Ns = 16^m starts at
// 16 * (16 + 256 + ... + 16^(m-1)) = 16 (Ns - 16) / 15.  (The FP64 table of a length N
// holds exp(-2 pi i j / N), j < N: a butterfly's base factor is entry k N / (Ns R).)
__host__ __device__ constexpr int twiddle_offset(int Ns) { return Ns < 16 ? 0 : 16 * ((Ns - 16) / 15); }
// entries of the whole table of length N (at most 2N for N <= 2048)
__host__ __device__ constexpr int twiddle_entries(int N) {
    int total = 0, ns = 1, rem = N;
    while (rem > 1) {
        const int r = rem >= 16 ? 16 : rem;
        if (ns > 1) total += ns * r;
        ns *= r;
        rem /= r;
    }
    return total;
}

// the R twiddles of one butterfly (t[0] = 1 is loaded but not used)
template <int R> __device__ __forceinline__ void load_twiddles(const float2 *__restrict__ p, float2 (&t)[R]) {
    const float4 *p4 = reinterpret_cast<const float4 *>(p);
#pragma unroll
    for (int i = 0; i < R / 2; ++i) {
        const float4 q = __ldg(p4 + i);
        t[2 * i] = make_float2(q.x, q.y);
        t[2 * i + 1] = make_float2(q.z, q.w);
    }
}
template <int R> __device__ __forceinline__ void load_twiddles(const double2 *__restrict__ p, double2 (&t)[R]) {
#pragma unroll
    for (int i = 0; i < R; ++i) t[i] = __ldg(p + i);
}

// FP64 stages multiply by the powers w^r, r < R, of one loaded base factor
// w = exp(-2 pi i k / (Ns R)) (table entry k*R + 1) instead of loading all R factors: a
// double2 factor is 16 bytes, as much L1 traffic per element as the data itself.  Each
// power is a product of two lower powers (p[r] = p[r/2] p[r - r/2]), so it carries at most
// log2(R) + 1 roundings of double (~5e-16), well below what a loaded FP32 factor carries.
template <int R, bool FWD> __device__ __forceinline__ void twiddle_powers(double2 (&v)[R], double2 w) {
    double2 p[R];
    p[0] = make_double2(1.0, 0.0);
    p[1] = w;
#pragma unroll
    for (int r = 2; r < R; ++r) p[r] = cmul(p[r / 2], p[r - r / 2]);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = FWD ? cmul(v[r], p[r]) : cmulc(v[r], p[r]);
}

// Memory spaces a stage reads from / writes to.
enum : int { SP_SMEM = 0, SP_GLOBAL = 1, SP_REGS = 2 };

// keeps a parameter out of template argument deduction (it may be passed nullptr)
template <typename T> struct nodeduce {
    typedef T type;
};

// Transform applied to each value a transform's first stage loads: v -> f(e, b, v)
// with e the element index along the sequence and b the sequence.
struct Identity {
    template <typename C> __device__ __forceinline__ C operator()(int, int, C v) const { return v; }
};

// One Stockham stage of radix R on NB interleaved sequences of length N; NS is the
// product of the radices of the earlier stages.
// IN/OUT: SP_SMEM (padded shared array), SP_GLOBAL (plain array).  OUT may also be
// SP_REGS: the stage's outputs are left in v (element e = j + r*NS of sequence b,
// item w = tid + q*NT, b = w % NB, j = w / NB) and nothing is stored.
// A stage whose input and output are the same shared array synchronises between
// its loads and its stores.
// A stage that reads global memory (or an unpadded staging buffer) may read a narrower
// stored type CI than its arithmetic type C (float2 into double2 arithmetic).
template <int N, int NB, int NT, int R, int NS, bool FWD, int IN, int OUT, typename C, typename XF = Identity,
          typename CI = C>
__device__ __forceinline__ void stage(const CI *__restrict__ in, typename nodeduce<C>::type *out, const C *__restrict__ tw,
                                      C (&v)[StageShape<N, NB, NT, R>::PER_T][R], XF xf = XF()) {
    typedef StageShape<N, NB, NT, R> S;
    constexpr int DIN = (N / R) * NB;  // element offset between a butterfly's inputs
    constexpr int DOUT = NS * NB;      // ... and between its outputs
    const int tid = threadIdx.x;
    // a stage that only writes shared memory must not overtake earlier readers of it
    if (IN != SP_SMEM && OUT == SP_SMEM) __syncthreads();
#pragma unroll
    for (int q = 0; q < S::PER_T; ++q) {
        const int w = tid + q * NT;  // = j * NB + b
        if (S::EXACT || w < S::ITEMS) {
            const int b = w % NB, j = w / NB;
            const int pw = spad(w);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                C x;
                if constexpr (IN != SP_SMEM)
                    x = to_c<C>(in[w + r * DIN]);
                else if constexpr (DIN % 16 == 0)  // spad(w + r*DIN) = spad(w) + r*DIN*17/16
                    x = in[pw + r * (DIN + DIN / 16)];
                else
                    x = in[spad(w + r * DIN)];
                v[q][r] = xf(j + r * (N / R), b, x);
            }
        }
    }
    if (IN == SP_SMEM && OUT == SP_SMEM) __syncthreads();
#pragma unroll
    for (int q = 0; q < S::PER_T; ++q) {
        const int w = tid + q * NT;
        if (S::EXACT || w < S::ITEMS) {
            const int b = w % NB, j = w / NB;
            const int k = j % NS;
            if constexpr (NS > 1) {
                if constexpr (std::is_same<C, double2>::value) {
                    twiddle_powers<R, FWD>(v[q], __ldg(tw + k * (N / (NS * R))));
                } else {
                    C t[R];
                    load_twiddles<R>(tw + twiddle_offset(NS) + k * R, t);
#pragma unroll
                    for (int r = 1; r < R; ++r) v[q][r] = FWD ? cmul(v[q][r], t[r]) : cmulc(v[q][r], t[r]);
                }
            }
            dftR<R, FWD>(v[q]);
            if constexpr (OUT != SP_REGS) {
                const int e0 = ((j / NS) * NS * R + k) * NB + b;
                const int pe = spad(e0);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if constexpr (OUT != SP_SMEM)
                        out[e0 + r * DOUT] = v[q][r];
                    else if constexpr (DOUT % 16 == 0)  // as for the loads
                        out[pe + r * (DOUT + DOUT / 16)] = v[q][r];
                    else
                        out[spad(e0 + r * DOUT)] = v[q][r];
                }
            }
        }
    }
    if (OUT == SP_SMEM) __syncthreads();
}

// Values a thread holds after a transform of element type C that ends in registers.
template <int N, int NB, int NT, typename C = float2> struct RegOut {
    typedef radix_plan<N, main_radix<C>::value> P;
    static constexpr int R = P::last_radix;
    static constexpr int PER_T = StageShape<N, NB, NT, R>::PER_T;
    static constexpr int NS = N / R;  // Ns of the last stage
};

// The main-radix stages between the first and the last, in place in shared memory.
template <int N, int NB, int NT, int NS, int LAST_NS, bool FWD, typename C>
__device__ __forceinline__ void middle_stages(
    C *s, const C *__restrict__ tw,
    C (&v)[StageShape<N, NB, NT, main_radix<C>::value>::PER_T][main_radix<C>::value]) {
    constexpr int RM = main_radix<C>::value;
    if constexpr (NS < LAST_NS) {
        stage<N, NB, NT, RM, NS, FWD, SP_SMEM, SP_SMEM>(s, s, tw, v);
        middle_stages<N, NB, NT, NS * RM, LAST_NS, FWD>(s, tw, v);
    }
}

// Work a transform runs right after its first stage (the first stage ends with a
// barrier, so `src` is free then): e.g. start loading the next input into it.
struct NoHook {
    __device__ __forceinline__ void operator()() const {}
};

// Full transform of NB interleaved length-N sequences.
//   IN  = SP_GLOBAL: the first stage reads the unpadded array `src` (global memory,
//         or a shared staging buffer); SP_SMEM: reads the padded shared array `src`
//         (which may be `s` itself or another buffer).  Every value it loads passes
//         through xf(e, b, v).
//   OUT = SP_GLOBAL: the last stage writes global `dst`; SP_SMEM: writes the padded
//         shared array `dst`; SP_REGS: the output stays in `last` (RegOut layout).
// Intermediate stages run in place in the padded shared scratch `s`; after the first
// stage af() runs.  Callers must __syncthreads() before a transform that reads
// shared data they wrote; a transform whose last stage writes shared memory
// synchronises before returning.
template <int N, int NB, int NT, bool FWD, int IN, int OUT, typename C, typename XF = Identity, typename AF = NoHook,
          typename CI = C>
__device__ __forceinline__ void fft(const CI *src, C *s, typename nodeduce<C>::type *dst,
                                    const C *__restrict__ tw,
                                    C (&last)[RegOut<N, NB, NT, C>::PER_T][RegOut<N, NB, NT, C>::R], XF xf = XF(),
                                    AF af = AF()) {
    constexpr int RM = main_radix<C>::value;
    typedef radix_plan<N, RM> P;
    if constexpr (P::stages == 1) {
        stage<N, NB, NT, P::last_radix, 1, FWD, IN, OUT>(src, dst, tw, last, xf);
        if constexpr (!std::is_same<AF, NoHook>::value) {
            __syncthreads();  // every thread has read src
            af();
        }
    } else {
        typedef StageShape<N, NB, NT, RM> SM;
        C v[SM::PER_T][RM];
        // first stage (main radix): src -> scratch
        stage<N, NB, NT, RM, 1, FWD, IN, SP_SMEM>(src, s, tw, v, xf);
        af();
        middle_stages<N, NB, NT, RM, RegOut<N, NB, NT, C>::NS, FWD>(s, tw, v);
        // last stage: scratch -> dst / registers
        stage<N, NB, NT, P::last_radix, RegOut<N, NB, NT, C>::NS, FWD, SP_SMEM, OUT>(s, dst, tw, last);
    }
}

// Convenience: in-place FFT of a padded shared array.
template <int N, int NB, int NT, bool FWD, typename C>
__device__ __forceinline__ void fft_smem(C *s, const C *__restrict__ tw) {
    C last[RegOut<N, NB, NT, C>::PER_T][RegOut<N, NB, NT, C>::R];
    fft<N, NB, NT, FWD, SP_SMEM, SP_SMEM>(s, s, s, tw, last);
}

}  // namespace pfc
