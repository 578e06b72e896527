// tile_io.cuh -- tile staging (cp.async or TMA bulk copies into shared memory, float4 stores out) and the
// multipliers an inverse transform's first stage applies, used by the column kernel
// (col_kernel.cuh).
#pragma once

#include "fft_core.cuh"
#include "pfc_internal.h"

namespace pfc {

// multiplier applied by an inverse transform's first stage: P * g(l, km)
struct ScaleByTable {
    const float2 *tab;  // kc2 tile (c2a, c2b)
    int C, which;       // which: 0 = .x, 1 = .y
    __device__ __forceinline__ float2 operator()(int e, int b, float2 v) const {
        const float2 t = tab[e * C + b];
        const float g = which == 0 ? t.x : t.y;
        return make_float2(v.x * g, v.y * g);
    }
};
// -i k P along l (which = 0, krefl) or m (which = 1, krefm)
struct GradientOf {
    const float *krefl, *krefm;
    int km0, H, which;
    __device__ __forceinline__ float2 operator()(int e, int b, float2 v) const {
        const int km = km0 + b;
        const float kv = which == 0 ? krefl[e] : krefm[km <= H ? km : 0];
        return make_float2(kv * v.y, -kv * v.x);
    }
};

// Two ways of staging an input tile (L*C float2: a contiguous, 16-byte aligned block
// whose size is a multiple of 16 bytes) into the unpadded staging buffer q.  Both put
// the same bytes in the same place, so results do not depend on the choice; which is
// faster depends on the kernel's register budget, and the autotuner picks per grid.
//   STAGE_ASYNC: every thread issues 16-byte cp.async copies tracked by its own commit
//     group; a wait is wait_group 0 followed by a barrier.
//   STAGE_BULK: one thread issues a single TMA bulk copy (cp.async.bulk) that completes
//     on a shared-memory mbarrier (one per CTA, one copy in flight at a time); every
//     thread waits on the barrier's phase.  The wait is bounded in time: a CTA whose
//     copy does not arrive sets the fault word and stops (CTA-uniformly).
constexpr int STAGE_ASYNC = COL_STAGE_ASYNC, STAGE_BULK = COL_STAGE_BULK;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// ---- STAGE_ASYNC ----
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
template <int L, int C, int NT> __device__ __forceinline__ void tile_prefetch(const float2 *__restrict__ g, float2 *q) {
    for (int i = threadIdx.x; i < L * C / 2; i += NT) cp_async16(q + 2 * i, g + 2 * i);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// this thread's copies have landed; the barrier makes every thread's visible
__device__ __forceinline__ void tile_wait_async() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
}

// ---- STAGE_BULK ----
// bound of a tile wait, and of the last wait of a CTA that gave up (nanoseconds of
// %globaltimer time)
constexpr unsigned long long STAGE_WAIT_NS = 1000000000ull;
constexpr unsigned long long STAGE_DRAIN_NS = 100000000ull;

// all threads; thread 0 initialises the barrier (shared address bar) for one arrival
// per phase
__device__ __forceinline__ void stage_init(unsigned bar) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
}

// thread 0: copy `bytes` from global g into shared q (the threads' earlier reads of q
// are complete: callers issue after a barrier)
__device__ __forceinline__ void stage_issue(unsigned bar, const void *g, void *q, unsigned bytes) {
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                         smem_u32(q)),
                     "l"(g), "r"(bytes), "r"(bar)
                     : "memory");
    }
}

__device__ __forceinline__ bool stage_poll(unsigned bar, unsigned phase) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(phase)
                 : "memory");
    return done != 0;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// wait until completion `phase` of the barrier or until limit_ns have passed; true when
// the phase completed
__device__ __forceinline__ bool stage_try(unsigned bar, unsigned phase, unsigned long long limit_ns) {
    if (stage_poll(bar, phase)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (stage_poll(bar, phase)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// all threads: wait for completion `phase` (the parity of the number of copies this
// barrier completed before it) of the copy in flight.  Returns false, the same in every
// thread of the CTA, when it did not arrive within limit_ns; the fault word is then set
// and the caller returns.  A CTA with a second bulk-copy barrier (has_other) also gives
// a copy in flight on that one a last wait: one of its two phases is the completed
// previous one and returns at once, the other ends when its copy lands or after
// STAGE_DRAIN_NS.
__device__ __forceinline__ bool tile_wait(unsigned bar, unsigned phase, int *fault,
                                          unsigned long long limit_ns = STAGE_WAIT_NS, bool has_other = false,
                                          unsigned other = 0) {
    const bool ok = stage_try(bar, phase, limit_ns);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
            *(volatile int *)fault = 1;
            if (has_other) {
                stage_try(other, 0u, STAGE_DRAIN_NS);
                stage_try(other, 1u, STAGE_DRAIN_NS);
            }
        }
        stage_try(bar, phase, STAGE_DRAIN_NS);  // a last, shorter wait for a copy still in flight
        return false;
    }
    return true;
}

// ---- the interface the column kernel uses ----
template <int L, int C, int NT, int STAGE> struct Stager {
    unsigned bar;    // STAGE_BULK: shared address of the completion barrier
    float2 *q;       // staging buffer
    bool has_other;  // the CTA has a second bulk-copy barrier, `other`, to drain on a fault
    unsigned other;
    // all threads, once, before the first copy
    __device__ __forceinline__ void init() const {
        if constexpr (STAGE == STAGE_BULK) stage_init(bar);
    }
    // all threads, after every thread's last read of q
    __device__ __forceinline__ void issue(const float2 *src) const {
        if constexpr (STAGE == STAGE_BULK)
            stage_issue(bar, src, q, (unsigned)(L * C * sizeof(float2)));
        else
            tile_prefetch<L, C, NT>(src, q);
    }
    // all threads: wait for the copy in flight, completion `phase` of the barrier
    // (STAGE_BULK); false, CTA-uniformly, when a bounded wait gave up
    __device__ __forceinline__ bool wait(unsigned phase, int *fault) const {
        if constexpr (STAGE == STAGE_BULK) {
            return tile_wait(bar, phase, fault, STAGE_WAIT_NS, has_other, other);
        } else {
            tile_wait_async();
            return true;
        }
    }
    // before the CTA exits: no copy outlives it
    __device__ __forceinline__ void finish() const {
        if constexpr (STAGE == STAGE_ASYNC) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
};

// A shared slot for one plane of a coefficient table tile (n doubles, a contiguous,
// 16-byte aligned block of 16-byte multiple size), filled by TMA bulk copies that complete
// on their own barrier (one copy in flight at a time; bounded waits as tile_wait's).
struct TableStager {
    unsigned bar;   // shared address of the completion barrier
    double *t;      // the slot
    unsigned bytes;
    unsigned other;  // the input stager's barrier (STAGE_BULK), drained on a fault
    bool has_other;
    __device__ __forceinline__ void init() const { stage_init(bar); }
    // all threads, after every thread's last read of the slot
    __device__ __forceinline__ void issue(const double *src) const { stage_issue(bar, src, t, bytes); }
    __device__ __forceinline__ bool wait(unsigned phase, int *fault) const {
        return tile_wait(bar, phase, fault, STAGE_WAIT_NS, has_other, other);
    }
};
// a transform's hook: fill the table slot once the first stage has read it
struct TableFetch {
    TableStager ts;
    const double *src;
    __device__ __forceinline__ void operator()() const {
        if (src) ts.issue(src);
    }
};

// a transform's hook: start the next tile's copy once the first stage has read the buffer
template <typename ST> struct Prefetch {
    ST st;
    const float2 *src;
    __device__ __forceinline__ void operator()() const {
        if (src) st.issue(src);
    }
};

template <int L, int C, int NT> __device__ __forceinline__ void tile_out(const float2 *sm, float2 *__restrict__ g) {
    float4 *g4 = reinterpret_cast<float4 *>(g);
    for (int i = threadIdx.x; i < L * C / 2; i += NT) {
        const float2 a = sm[spad(2 * i)], b = sm[spad(2 * i + 1)];
        g4[i] = make_float4(a.x, a.y, b.x, b.y);
    }
}

}  // namespace pfc
