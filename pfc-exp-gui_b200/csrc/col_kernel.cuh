// col_kernel.cuh -- the column kernel of the fused FP32 step (included by step_fp32.cu).
//
// Work item: a tile of L rows x C packed columns of one run (a contiguous block of
// the row-space layout).  CTAs are persistent and take items in turn.  For phi and
// then con:
//   the field's tile is transformed forward into the parked buffer P,
//   its nonlinear term's tile is transformed forward in place in the scratch s,
//   the semi-implicit update runs in place in P (MAINEQUATIONC2_NOI / C2MIX,
//     MIS:983-1014, CVD:865-886) with the FP64-built factors of the shared
//     coefficient table (and the noise term when axx > 0),
//   each output is an inverse transform whose first stage reads P through a
//     multiplier (1, C2A, C2B for phi, MIS:807-810; 1 and the -i k gradients for
//     con at checkpoints, MIS:884-889) into s, copied s -> HBM (float4).
// Inputs are staged into an unpadded buffer Q, which a transform's first stage reads
// directly, by 16-byte cp.async copies (STAGE_ASYNC) or by one TMA bulk copy per tile
// completing on a shared-memory mbarrier (STAGE_BULK; waits bounded in time, a CTA
// whose copy does not arrive sets the context's fault word and returns); the
// autotuner picks the method with the width.  Each load is issued as soon as the
// previous transform's first stage has consumed Q, so it streams in while that
// transform, the update and the output transforms run; the next item's phi tile
// streams in during the current item's con work.  Two CTAs of 256 threads
// per SM at C*L = 4096 (2 x 100 KB of shared memory, 128 registers); the tile width C
// of a grid is chosen per device by the autotuner (engine.cu).

// Tile staging (Stager, Prefetch, tile_out) and the
// ScaleByTable / GradientOf multipliers come from tile_io.cuh.

// Spectrum of the noise field at mode (l, km) of step t.  The reference draws real-space
// white noise with a sequential polar Box-Muller generator (Gauss, MIS:951-981) and
// transforms it (p5); the transform of white noise is itself white, so the modes are
// drawn here directly, with the distribution the reference's masks leave
// (MIS:1002-1003): re and im independent N(0, P/4), except at the four self-conjugate
// modes (l in {0, L/2}, km in {0, M/2}) where re ~ N(0, P) and im = 0; along the
// self-conjugate columns km = 0 and M/2, mode L - l is the conjugate of mode l.
// Stream: the two normals of canonical mode c = (t*L + l)*(M/2 + 1) + km come from
// Box-Muller of the splitmix64 outputs at positions 2c and 2c + 1 of the run's key.
__device__ __forceinline__ unsigned long long sm64_out(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ float2 noise_mode(unsigned long long key, int t, int l, int km, int L, int M) {
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

template <int L, int C, int MODE, int STAGE>
__global__ void __launch_bounds__(ColCfg<L, C>::NT, ColCfg<L, C>::MINB)
    k_col_step(const RunDesc *__restrict__ runs, int nruns, const float2 *__restrict__ tw, int *fault) {
    constexpr int NT = ColCfg<L, C>::NT;
    constexpr int SPAD = padded_len<C * L>::value;
    typedef RegOut<L, C, NT> RO;  // register scratch the transforms need for their last stage
    extern __shared__ __align__(16) float2 smem[];
    __shared__ __align__(8) unsigned long long stage_bar;  // completion barrier of the tile copies
    float2 *s = smem;               // FFT scratch
    float2 *Pk = smem + SPAD;       // parked spectrum
    float2 *Q = smem + 2 * SPAD;    // staging buffer (16-byte aligned: 2*SPAD float2)
    const int T = runs[0].T;        // all runs of a launch share L and M
    const int items = nruns * T;
    float2 b[RO::PER_T][RO::R];
    int item = blockIdx.x;
    if (item >= items) return;
    typedef Stager<L, C, NT, STAGE> ST;
    const ST st{smem_u32(&stage_bar), Q};
    st.init();
    auto tile_of = [&](int it) { return (long)(it % T) * L * C; };
    st.issue(runs[item / T].psi + tile_of(item));
    for (; item < items; item += gridDim.x) {
        const RunDesc &d = runs[item / T];
        const int H = d.M / 2;
        const long tile = tile_of(item);
        const int km0 = (item % T) * C;
        const int next = item + gridDim.x;
        const float2 *next_psi = next < items ? runs[next / T].psi + tile_of(next) : nullptr;
        const float invL = 1.0f / (float)L;
        // barrier phase of this item's first wait: an item of the step modes waits four
        // times (phases 0, 1, 0, 1), a COL_PREPARE item once (the iteration's parity)
        const unsigned p0 = MODE == COL_PREPARE ? (unsigned)((item - (int)blockIdx.x) / (int)gridDim.x) & 1u : 0u;
        const float mn_dt = d.k.dynamic_mn * d.dt, mc_dt = d.k.dynamic_mc * d.dt;

        // ---- phi ----
        if (!st.wait(p0, fault)) return;
        if (MODE == COL_PREPARE) {
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, next_psi});
        } else {
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, d.inn + tile});
            if (!st.wait(1u, fault)) return;
            fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, s, tw, b, Identity(), Prefetch<ST>{st, d.con + tile});
        }
        const int nstep = (MODE != COL_PREPARE && d.noise_amp != 0.0f) ? *d.step_ctr : -1;
        for (int e = threadIdx.x; e < L * C; e += NT) {
            const int l = e / C, c = e % C, km = km0 + c;
            const int pi = spad(e);
            float2 v = Pk[pi];
            if (MODE != COL_PREPARE) {
                // (psi^ - Mn dt k^2 N^ [+ dt b0 xi^ |k| lowpass]) / (1 + Mn dt k^2) / L; the
                // FP64-built factor is 0 at k = 0
                const float kl = d.krefl[l], kmv = d.krefm[km <= H ? km : 0];
                const float ks = kl * kl + kmv * kmv;
                const float an = mn_dt * ks;
                const float2 nh = s[pi];
                const float f = d.kden[tile + e].x;
                float rx = v.x - an * nh.x, ry = v.y - an * nh.y;
                if (nstep >= 0 && km <= H) {
                    // MAINEQUATIONC2_NOI's noise term (MIS:1002-1003), lowpass at |k| = 2 pi
                    const float2 xi = noise_mode(d.noise_key, nstep, l, km, L, d.M);
                    const float sk = sqrtf(ks);
                    const float w = d.noise_amp * sk * (0.5f - 0.5f * tanhf((sk - 6.2831852f) / 0.1f));
                    rx += w * xi.x;
                    ry += w * xi.y;
                }
                v = make_float2(rx * f, ry * f);
            } else {
                v = (l == 0 && km == 0) ? make_float2(0.f, 0.f) : cscale(v, invL);
            }
            Pk[pi] = v;
        }
        __syncthreads();
        if (MODE != COL_PREPARE) {
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b);
            tile_out<L, C, NT>(s, d.psi + tile);
        }
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, ScaleByTable{d.kc2 + tile, C, 0});
        tile_out<L, C, NT>(s, d.ca + tile);
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, ScaleByTable{d.kc2 + tile, C, 1});
        tile_out<L, C, NT>(s, d.cb + tile);
        if (MODE == COL_PREPARE) continue;

        // ---- con ----
        if (!st.wait(0u, fault)) return;
        fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, Pk, tw, b, Identity(), Prefetch<ST>{st, d.inc + tile});
        if (!st.wait(1u, fault)) return;
        fft<L, C, NT, true, SP_GLOBAL, SP_SMEM>(Q, s, s, tw, b, Identity(), Prefetch<ST>{st, next_psi});
        for (int e = threadIdx.x; e < L * C; e += NT) {
            const int l = e / C, c = e % C, km = km0 + c;
            const int pi = spad(e);
            // (c^ - Mc dt k^2 I^) / (1 + Mc dt alpha k^4) / L; the FP64-built factor is 0 at k = 0
            const float kl = d.krefl[l], kmv = d.krefm[km <= H ? km : 0];
            const float ac = mc_dt * (kl * kl + kmv * kmv);
            const float f = d.kden[tile + e].y;
            const float2 ih = s[pi];
            const float2 v = Pk[pi];
            Pk[pi] = make_float2((v.x - ac * ih.x) * f, (v.y - ac * ih.y) * f);
        }
        __syncthreads();
        fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b);
        tile_out<L, C, NT>(s, d.con + tile);
        if (MODE == COL_STEP_CHECKPOINT) {
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, GradientOf{d.krefl, d.krefm, km0, H, 0});
            tile_out<L, C, NT>(s, d.gx + tile);
            fft<L, C, NT, false, SP_SMEM, SP_SMEM>(Pk, s, s, tw, b, GradientOf{d.krefl, d.krefm, km0, H, 1});
            tile_out<L, C, NT>(s, d.gy + tile);
        }
    }
    st.finish();  // every copy issued has been waited for: the last item issues none (next_psi = null)
}
