/*
 * pfc_oracle.c -- CPU restatement of the reference's hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Only tests/, the smoke check and bench.py's CPU baseline call this library, and
 * only as the checker.  The product (pfc-exp-gui_b200/) never links or loads it.
 *
 * Every function cites the reference routine it restates (paths within
 * zhiqing0205/PFC-Exp-GUI: MIS = src/experiment/misfit_uniform_time_seed_fftw_early.cpp,
 * CVD = src/experiment/cvd.cpp, ELA = src/experiment/elastic.cpp,
 * COM = src/experiment/pfc_common.h).
 *
 * Precision.  In exact mode every float/double conversion of the C++ reference is
 * reproduced: a C++ call such as sqrt(float) or cos(float) resolves to the float
 * overload and is written sqrtf/cosf here; pow(float, int) promotes to double and
 * stays pow; values assigned to float locals are rounded with (float) casts.  The
 * file is compiled with gcc -O2 for x86-64 without -ffast-math or FMA, the same
 * arithmetic environment as the reference binary, so with the same FFT
 * (fftw_shim/fftw_shim.c) the two produce identical bits.  exact = 0 runs the same
 * scheme with every intermediate in double ("pure FP64").
 */
#define _POSIX_C_SOURCE 200809L
#include "pfc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

#define PI_REF 3.1415926 /* COM:152 "#define pi 3.1415926" */

/* ------------------------------------------------------------------------- */
/* Model constants (MIS:116-143, CVD:26-53).                                  */
/* ------------------------------------------------------------------------- */
typedef struct {
    float gaa1, gaa2, gab1, gab2;
    float niu, ksi;
    float ka0, ka1, ka2, sigMa1, sigMa2;
    float kb0, kb1, kb2, sigMb1, sigMb2;
    float para_c0, dynamic_mn, dynamic_mc, para_alpha, para_w;
} model_consts;

static void consts_for(int model, model_consts *k) {
    const float a_lattice = 1.0f;
    k->gaa1 = 0.8f;
    k->gaa2 = (float)(k->gaa1 * sqrt(2.));
    k->gab1 = 0.8f;
    k->gab2 = (float)(k->gaa2 * sqrt(2.));
    k->niu = 1.4f;
    k->ksi = 1.f;
    k->ka0 = (float)(2.0 * PI_REF / a_lattice);
    k->ka1 = (float)(2.0 * PI_REF);
    k->ka2 = (float)(sqrt(2.0) * k->ka1);
    k->sigMa1 = 0.55f;
    k->sigMa2 = 0.55f;
    k->sigMb1 = 0.55f;
    k->sigMb2 = 0.55f;
    k->para_c0 = 0.5f;
    k->para_alpha = 0.5f;
    k->para_w = 0.02f;
    if (model == ORC_MODEL_CVD) {
        const float b_lattice = (float)(sqrt(3.0) / 2.0);     /* CVD:33 */
        k->kb0 = (float)(2.5 * PI_REF / b_lattice);          /* CVD:42 */
        k->kb1 = (float)(5.0 * PI_REF / sqrt(3.0));
        k->kb2 = (float)(k->kb1 * sqrt(2.0));
        k->dynamic_mn = 1.f;                                  /* CVD:45 */
        k->dynamic_mc = 1.f;
    } else {
        const float b_lattice = 0.88f;                        /* MIS:123 */
        k->kb0 = (float)(2.0 * PI_REF / b_lattice);          /* MIS:131 */
        k->kb1 = k->kb0;
        k->kb2 = (float)(k->kb1 * sqrt(2.0));
        k->dynamic_mn = 0.1f;                                 /* MIS:134 */
        k->dynamic_mc = 10.f;
    }
}

void orc_default_params(int model, orc_params *p) {
    memset(p, 0, sizeof(*p));
    p->model = model;
    p->L = 256;
    p->M = 256;
    p->N = 1;
    p->seed = 20200604u; /* COM:154 FIXED_SEED */
    p->exact = 1;
    p->dt = 0.05f;
    p->dx = 0.125f;
    p->con0 = 0.2f;
    p->axx = 0.0f;
    if (model == ORC_MODEL_CVD) {
        p->u0 = 0.01f; /* CVD:35 */
        p->sig = 0.03f;
        p->grainx = p->grainy = p->grainz = 1;
    } else {
        p->u0 = 0.05f; /* MIS:125 */
        p->sig = 0.05f;
        p->grainx = 16; /* MIS:138 */
        p->grainy = 16;
        p->grainz = 1;
    }
}

/* ------------------------------------------------------------------------- */
/* RNG (COM:165-181).                                                         */
/* ------------------------------------------------------------------------- */
uint64_t orc_splitmix64_next(uint64_t *state) {
    uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

double orc_rng_u01(uint64_t *state) {
    const double inv = 1.0 / 9007199254740992.0;
    return (double)(orc_splitmix64_next(state) >> 11) * inv;
}

static double rng_u11(uint64_t *state) { return 2.0 * orc_rng_u01(state) - 1.0; }

void orc_dft3d(int n0, int n1, int n2, const double *in, double *out, int sign) {
    pfc_shim_dft_3d(n0, n1, n2, (const fftw_complex *)in, (fftw_complex *)out, sign);
}

/* ------------------------------------------------------------------------- */
/* Run state.                                                                 */
/* ------------------------------------------------------------------------- */
struct orc_run {
    orc_params p;
    model_consts k;
    long P;
    float b0;
    int dnx, dny, dnz;
    /* complex double arrays, 2*P doubles each (re, im interleaved) */
    double *phi, *con, *phiHat, *conHat;
    double *in1, *in2, *in3, *inn, *inc, *outn, *outc;
    double *c2adenp, *c2bdenp, *c2aden, *c2bden;
    double *gra1, *gra2, *gra3, *grao1, *grao2, *grao3, *grac;
    double *nois, *noisf;
    float *C2AHat, *C2BHat;   /* exact mode tables (MIS:425-427) */
    double *C2AHd, *C2BHd;    /* pure mode tables */
    float *krefl, *krefm, *krefn;
    double *kdl, *kdm, *kdn;
};

#define RE(a, i) (a)[2 * (i)]
#define IM(a, i) (a)[2 * (i) + 1]

static double *cz(long P) { return (double *)calloc((size_t)(2 * P), sizeof(double)); }

orc_run *orc_create(const orc_params *p) {
    orc_run *r = (orc_run *)calloc(1, sizeof(orc_run));
    r->p = *p;
    consts_for(p->model, &r->k);
    r->P = (long)p->L * p->M * p->N;
    const long P = r->P;
    double **arrs[] = {&r->phi,  &r->con,  &r->phiHat, &r->conHat, &r->in1,     &r->in2,     &r->in3,
                       &r->inn,  &r->inc,  &r->outn,   &r->outc,   &r->c2adenp, &r->c2bdenp, &r->c2aden,
                       &r->c2bden, &r->gra1, &r->gra2, &r->gra3,   &r->grao1,   &r->grao2,   &r->grao3,
                       &r->grac, &r->nois, &r->noisf};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) *arrs[i] = cz(P);
    r->C2AHat = (float *)calloc((size_t)P, sizeof(float));
    r->C2BHat = (float *)calloc((size_t)P, sizeof(float));
    r->C2AHd = (double *)calloc((size_t)P, sizeof(double));
    r->C2BHd = (double *)calloc((size_t)P, sizeof(double));
    r->krefl = (float *)calloc((size_t)p->L, sizeof(float));
    r->krefm = (float *)calloc((size_t)p->M, sizeof(float));
    r->krefn = (float *)calloc((size_t)p->N, sizeof(float));
    r->kdl = (double *)calloc((size_t)p->L, sizeof(double));
    r->kdm = (double *)calloc((size_t)p->M, sizeof(double));
    r->kdn = (double *)calloc((size_t)p->N, sizeof(double));
    /* RecomputeDerivedParams (MIS:162-179). */
    r->dnx = p->grainx > 0 ? p->L / p->grainx : 0;
    r->dny = p->grainy > 0 ? p->M / p->grainy : 0;
    r->dnz = p->grainz > 0 ? p->N / p->grainz : 0;
    if (p->dx > 0.0f && p->dt > 0.0f && p->axx >= 0.0f)
        r->b0 = (float)sqrt(p->axx / p->dx / p->dx / p->dx / p->dt);
    else
        r->b0 = 0.0f;
    return r;
}

void orc_destroy(orc_run *r) {
    if (!r) return;
    double *arrs[] = {r->phi,     r->con,     r->phiHat, r->conHat, r->in1,  r->in2,    r->in3,  r->inn,
                      r->inc,     r->outn,    r->outc,   r->c2adenp, r->c2bdenp, r->c2aden, r->c2bden, r->gra1,
                      r->gra2,    r->gra3,    r->grao1,  r->grao2,  r->grao3, r->grac,   r->nois, r->noisf,
                      r->C2AHd,   r->C2BHd,   r->kdl,    r->kdm,    r->kdn};
    for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); ++i) free(arrs[i]);
    free(r->C2AHat);
    free(r->C2BHat);
    free(r->krefl);
    free(r->krefm);
    free(r->krefn);
    free(r);
}

/* ks (COM:237-239): k^2 in float. */
static inline float ks_f(const orc_run *r, int l, int m, int n) {
    return r->krefl[l] * r->krefl[l] + r->krefm[m] * r->krefm[m] + r->krefn[n] * r->krefn[n];
}
static inline double ks_d(const orc_run *r, int l, int m, int n) {
    return r->kdl[l] * r->kdl[l] + r->kdm[m] * r->kdm[m] + r->kdn[n] * r->kdn[n];
}

/* k-vectors (MIS:455-462): Nyquist index positive, (l - L) above it. */
static void kref_init(orc_run *r) {
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    const float dx = r->p.dx;
    for (int l = 0; l < L / 2 + 1; l++) r->krefl[l] = (float)((double)l * 2.0 * PI_REF / (double)((float)L * dx));
    for (int l = L / 2 + 1; l < L; l++) r->krefl[l] = (float)((double)(l - L) * 2.0 * PI_REF / (double)((float)L * dx));
    for (int m = 0; m < M / 2 + 1; m++) r->krefm[m] = (float)((double)m * 2.0 * PI_REF / (double)((float)M * dx));
    for (int m = M / 2 + 1; m < M; m++) r->krefm[m] = (float)((double)(m - M) * 2.0 * PI_REF / (double)((float)M * dx));
    for (int n = 0; n < N / 2 + 1; n++) r->krefn[n] = (float)((double)n * 2.0 * PI_REF / (double)((float)N * dx));
    for (int n = N / 2 + 1; n < N; n++) r->krefn[n] = (float)((double)(n - N) * 2.0 * PI_REF / (double)((float)N * dx));
    for (int l = 0; l < L; l++) r->kdl[l] = (double)(l <= L / 2 ? l : l - L) * 2.0 * PI_REF / ((double)L * dx);
    for (int m = 0; m < M; m++) r->kdm[m] = (double)(m <= M / 2 ? m : m - M) * 2.0 * PI_REF / ((double)M * dx);
    for (int n = 0; n < N; n++) r->kdn[n] = (double)(n <= N / 2 ? n : n - N) * 2.0 * PI_REF / ((double)N * dx);
}

/* Two-peak correlation kernel (MIS:700-750 C2AK/C2BK; CVD:658-708 identical).
 * g1, g2: Gaussian widths; k1, k2: peak positions; s1, s2: sigma_M. */
static void c2_table(orc_run *r, float g1, float g2, float k1, float k2, float s1, float s2, float *out_f,
                     double *out_d) {
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    const float sig = r->p.sig;
    /* exact mode, float locals as in MIS:702-706 */
    float aa1 = (float)pow(sig / s1, 2);
    float aa2 = (float)pow(sig / s2, 2);
    float bb1 = (float)(1. / (2. * g1 * g1));
    float bb2 = (float)(1. / (2. * g2 * g2));
    float D = bb1 * k1 - bb2 * k2;
    float E = aa1 - aa2 + bb1 * k1 * k1 - bb2 * k2 * k2;
    float kc = (float)(((double)D + sqrt(pow(D, 2) - (double)((bb1 - bb2) * E))) / (double)(bb1 - bb2));
    if (g1 == g2) kc = (aa2 - aa1 + bb1 * (k2 * k2 - k1 * k1)) / (2 * bb1 * (k2 - k1));
    /* pure mode */
    double daa1 = pow((double)sig / s1, 2), daa2 = pow((double)sig / s2, 2);
    double dbb1 = 1. / (2. * g1 * g1), dbb2 = 1. / (2. * g2 * g2);
    double dD = dbb1 * k1 - dbb2 * k2;
    double dE = daa1 - daa2 + dbb1 * k1 * k1 - dbb2 * k2 * k2;
    double dkc = (dD + sqrt(dD * dD - (dbb1 - dbb2) * dE)) / (dbb1 - dbb2);
    if (g1 == g2) dkc = (daa2 - daa1 + dbb1 * ((double)k2 * k2 - (double)k1 * k1)) / (2 * dbb1 * ((double)k2 - k1));
    for (int l = 0; l < L; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) {
                const long i = n + (long)N * (m + (long)M * l);
                const float s = sqrtf(ks_f(r, l, m, n));
                if (s <= kc) out_f[i] = (float)(exp(-pow(sig / s1, 2)) * exp(-pow(s - k1, 2) / (2 * g1 * g1)));
                if (s > kc) out_f[i] = (float)(exp(-pow(sig / s2, 2)) * exp(-pow(s - k2, 2) / (2 * g2 * g2)));
                const double sd = sqrt(ks_d(r, l, m, n));
                const double q1 = (double)sig / s1, q2 = (double)sig / s2;
                if (sd <= dkc)
                    out_d[i] = exp(-q1 * q1) * exp(-(sd - k1) * (sd - k1) / (2.0 * g1 * g1));
                else
                    out_d[i] = exp(-q2 * q2) * exp(-(sd - k2) * (sd - k2) / (2.0 * g2 * g2));
            }
}

/* INITIAL_dis (MIS:610-682): uniform u0/con0 plus seeded square-lattice grains. */
static void initial_dis(orc_run *r) {
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    const float dx = r->p.dx, u0 = r->p.u0, con0 = r->p.con0;
    const float A1 = 0.1427f, A2 = 0.106f;
    const int seed_m_max = M < 160 ? M : 160;
    const int start = 0;
    for (long i = 0; i < r->P; ++i) {
        RE(r->phi, i) = u0;
        IM(r->phi, i) = 0;
        RE(r->con, i) = con0;
        IM(r->con, i) = 1.0E-10;
    }
    const model_consts *k = &r->k;
    for (int iii = 0; iii < r->p.grainx; iii++)
        for (int jjj = 0; jjj < r->p.grainy; jjj++)
            for (int kkk = 0; kkk < r->p.grainz; kkk++) {
                const float center_x = (float)(r->dnx * iii + r->dnx / 2);
                const float center_y = (float)(r->dny * jjj + r->dny / 2);
                const float center_z = (float)(r->dnz * kkk + r->dnz / 2);
                const unsigned int center_sum = (unsigned int)((r->dnx * iii + r->dnx / 2) + (r->dny * jjj + r->dny / 2) +
                                                               (r->dnz * kkk + r->dnz / 2));
                uint64_t st = (uint64_t)(r->p.seed ^ (center_sum * 2654435761u));
                const double v1 = 80.0 * (orc_rng_u01(&st) - 0.5);
                (void)orc_rng_u01(&st); /* v2, unused (MIS:642) */
                const float theta = (float)(v1 * PI_REF / 180);
                const float cth = cosf(theta);
                const double cother = cos(PI_REF / 2 - (double)theta - (double)(iii + jjj + kkk) * PI_REF);
                const float kk = (1 - con0) * k->ka0 + con0 * k->kb0;
                const double limx = (double)((float)L * dx / (float)r->p.grainx) / 2. - 0.2;
                const double limy = (double)((float)M * dx / (float)r->p.grainy) / 2. - 0.2;
                for (int l = 0; l < L; l++)
                    for (int m = 0; m < seed_m_max; m++)
                        for (int n = 0; n < N; n++) {
                            const int lx = l + start;
                            const float xx = ((float)start - center_x + (float)l) * dx;
                            const float yy = ((float)m - center_y) * dx;
                            const float zz = ((float)n - center_z) * dx;
                            const int X = (int)((double)((float)lx * cth) + (double)m * cother);
                            const int Y = (int)((double)((float)m * cth) - (double)lx * cother);
                            if ((double)fabsf(xx) < limx && (double)fabsf(yy) < limy && (double)fabsf(zz) < 4.3) {
                                const float cx = cosf(kk * (float)X * dx);
                                const float cy = cosf(kk * (float)Y * dx);
                                RE(r->phi, n + (long)N * (m + (long)M * l)) =
                                    2 * A1 * (cx + cy) + 4 * A2 * cx * cy + u0;
                            }
                        }
            }
}

/* INITIAL_C2 (CVD:587-642): A-lattice below m = M/2, B-lattice above. */
static void initial_c2(orc_run *r) {
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    const float dx = r->p.dx, u0 = r->p.u0, con0 = r->p.con0;
    const float A1 = 0.15f, A2 = 0.106f;
    const float w3 = (float)(0. * PI_REF / 180);
    const float cw = cosf(w3), sw = sinf(w3);
    const model_consts *k = &r->k;
    for (int l = 0; l < L; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) {
                const long i = n + (long)N * (m + (long)M * l);
                const float x = (float)(0 - L / 2 + l) * dx;
                const float y = (float)(m - M / 2) * dx;
                IM(r->phi, i) = 0;
                IM(r->con, i) = 1.0E-10;
                const float kx = (m < M / 2) ? k->ka0 : k->kb0;
                const float c1 = cosf(kx * x * cw + kx * y * sw);
                const float c2 = cosf(-x * kx * sw + kx * y * cw);
                const float c3 = cosf(kx * x * cw + kx * y * sw);
                const float c4 = cosf(-x * kx * sw + y * kx * cw);
                RE(r->phi, i) = 2 * A1 * (c1 + c2) + 4 * A2 * c3 * c4 + u0;
                RE(r->con, i) = (m < M / 2) ? con0 : 1 - con0;
            }
}

void orc_init(orc_run *r) {
    kref_init(r);
    const model_consts *k = &r->k;
    c2_table(r, k->gaa1, k->gaa2, k->ka1, k->ka2, k->sigMa1, k->sigMa2, r->C2AHat, r->C2AHd);
    c2_table(r, k->gab1, k->gab2, k->kb1, k->kb2, k->sigMb1, k->sigMb2, r->C2BHat, r->C2BHd);
    if (r->p.model == ORC_MODEL_CVD)
        initial_c2(r);
    else
        initial_dis(r);
}

/* ------------------------------------------------------------------------- */
/* Step pieces.                                                               */
/* ------------------------------------------------------------------------- */
static void fft_fwd(const orc_run *r, const double *in, double *out) {
    pfc_shim_dft_3d(r->p.L, r->p.M, r->p.N, (const fftw_complex *)in, (fftw_complex *)out, FFTW_FORWARD);
}
static void fft_bwd(const orc_run *r, const double *in, double *out) {
    pfc_shim_dft_3d(r->p.L, r->p.M, r->p.N, (const fftw_complex *)in, (fftw_complex *)out, FFTW_BACKWARD);
}

/* UPDATEINN3 (MIS:773-784). */
static void update_inn3(orc_run *r) {
    const double niu = r->k.niu, ksi = r->k.ksi;
    for (long i = 0; i < r->P; ++i) {
        const double ph = RE(r->phi, i);
        RE(r->in1, i) = -niu * pow(ph, 2) / 2.0 + ksi * pow(ph, 3) / 3.0;
        IM(r->in1, i) = 0.0;
    }
}

/* UPDATEINFMIX (MIS:786-798). */
static void update_infmix(orc_run *r) {
    const double w = r->k.para_w, c0 = r->k.para_c0;
    for (long i = 0; i < r->P; ++i) {
        const double c = RE(r->con, i);
        RE(r->in2, i) = w * (c * log(c / c0) + (1.0 - c) * log((1.0 - c) / (1.0 - c0)));
        IM(r->in2, i) = 0.0;
    }
}

/* UPDATEINFCMIX (MIS:801-833): c2a/c2b = IFFT(C2 * phiHat)/P, then in3. */
static void update_infcmix(orc_run *r) {
    const long P = r->P;
    const int LMN = r->p.L * r->p.M * r->p.N;
    for (long i = 0; i < P; ++i) {
        const double a = r->p.exact ? (double)r->C2AHat[i] : r->C2AHd[i];
        const double b = r->p.exact ? (double)r->C2BHat[i] : r->C2BHd[i];
        RE(r->c2adenp, i) = a * RE(r->phiHat, i);
        IM(r->c2adenp, i) = a * IM(r->phiHat, i);
        RE(r->c2bdenp, i) = b * RE(r->phiHat, i);
        IM(r->c2bdenp, i) = b * IM(r->phiHat, i);
    }
    fft_bwd(r, r->c2adenp, r->c2aden);
    fft_bwd(r, r->c2bdenp, r->c2bden);
    for (long i = 0; i < P; ++i) {
        RE(r->c2aden, i) = RE(r->c2aden, i) / LMN;
        IM(r->c2aden, i) = IM(r->c2aden, i) / LMN;
        RE(r->c2bden, i) = RE(r->c2bden, i) / LMN;
        IM(r->c2bden, i) = IM(r->c2bden, i) / LMN;
        const double c = RE(r->con, i);
        RE(r->in3, i) = -(1.0 - 3.0 * pow(c, 2) + 2.0 * pow(c, 3)) * (RE(r->c2aden, i)) -
                        (1.0 - 3.0 * pow((1.0 - c), 2) + 2.0 * pow((1.0 - c), 3)) * (RE(r->c2bden, i));
        IM(r->in3, i) = 0.0;
    }
}

/* UPDATEINC2MIX (MIS:835-848). */
static void update_inc2mix(orc_run *r) {
    for (long i = 0; i < r->P; ++i) {
        RE(r->inn, i) = RE(r->in1, i) + RE(r->in2, i) + RE(r->in3, i);
        IM(r->inn, i) = 0.0;
    }
}

/* UPDATEINC2MIXC (MIS:851-874): the four cmix terms are float locals. */
static void update_inc2mixc(orc_run *r) {
    const double w = r->k.para_w, c0 = r->k.para_c0;
    for (long i = 0; i < r->P; ++i) {
        const double ph = RE(r->phi, i), c = RE(r->con, i);
        const double a = RE(r->c2aden, i), b = RE(r->c2bden, i);
        if (r->p.exact) {
            const float cmix1 = (float)(w * (ph + 1.0) * log(c / c0));
            const float cmix2 = (float)(w * (ph + 1.0) * log((1.0 - c) / (1.0 - c0)));
            const float cmix3 = (float)(3.0 * ph * (a - b) * pow(c, 2));
            const float cmix4 = (float)(3.0 * ph * (-1.0 * a + b) * c);
            RE(r->inc, i) = cmix1 - cmix2 - cmix3 - cmix4;
        } else {
            const double cmix1 = w * (ph + 1.0) * log(c / c0);
            const double cmix2 = w * (ph + 1.0) * log((1.0 - c) / (1.0 - c0));
            const double cmix3 = 3.0 * ph * (a - b) * pow(c, 2);
            const double cmix4 = 3.0 * ph * (-1.0 * a + b) * c;
            RE(r->inc, i) = cmix1 - cmix2 - cmix3 - cmix4;
        }
        IM(r->inc, i) = 0.0;
    }
}

/* Gauss (MIS:951-981): polar Box-Muller on one sequential splitmix64 stream. */
static void gauss_noise(orc_run *r, int timestep) {
    uint64_t st = (uint64_t)r->p.seed;
    st ^= (uint64_t)((unsigned int)(0 + 1)) * 2654435761ULL;
    st ^= (uint64_t)((unsigned int)timestep) * 374761393ULL;
    for (long i = 0; i < r->P; ++i) {
        float v1 = 0, v2 = 0, r2 = 2.0f;
        while (r2 >= 1.0f || r2 <= 0.0f) {
            v1 = (float)rng_u11(&st);
            v2 = (float)rng_u11(&st);
            r2 = v1 * v1 + v2 * v2;
        }
        const float f = (float)sqrt(-2. * logf(r2) / r2);
        RE(r->nois, i) = f * v1;
        IM(r->nois, i) = 0.0;
    }
}

/* MAINEQUATIONC2_NOI (MIS:983-1014) and MAINEQUATIONC2MIX (MIS:928-949, CVD:865-886).
 * with_noise selects the Misfit form; when b0 == 0 the noise term is a signed zero
 * and is skipped. */
static void main_equation(orc_run *r, int with_noise) {
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    const float mn = r->k.dynamic_mn, mc = r->k.dynamic_mc, alpha = r->k.para_alpha, dt = r->p.dt;
    const int noise = with_noise && r->b0 != 0.0f;
    for (int l = 0; l < L; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) {
                const long i = n + (long)N * (m + (long)M * l);
                if (r->p.exact) {
                    const float kk = ks_f(r, l, m, n);
                    double nre = 0.0, nim = 0.0;
                    if (noise) {
                        const float detrx = (l == 0) ? 1.0f : 0.0f, detrxn = (l == L / 2) ? 1.0f : 0.0f;
                        const float detry = (m == 0) ? 1.0f : 0.0f, detryn = (m == M / 2) ? 1.0f : 0.0f;
                        const double lp = (0.5 - 0.5 * tanh(((double)sqrtf(kk) - 2.0 * PI_REF) / 0.1));
                        nre = (double)(dt * r->b0) * RE(r->noisf, i) * (double)sqrtf(kk) *
                              sqrt(fabs(0.5 + 0.5 * (double)(detrx + detrxn) * (double)(detry + detryn))) * lp;
                        nim = (double)(dt * r->b0) * IM(r->noisf, i) * (double)sqrtf(kk) *
                              sqrt(fabs(0.5 - 0.5 * (double)(detrx + detrxn) * (double)(detry + detryn))) * lp;
                    }
                    const float an = mn * dt * kk;
                    float Rhat1, Rhat2;
                    if (noise) {
                        Rhat1 = (float)(RE(r->phiHat, i) - (double)an * RE(r->outn, i) + nre);
                        Rhat2 = (float)(IM(r->phiHat, i) - (double)an * IM(r->outn, i) + nim);
                    } else {
                        Rhat1 = (float)(RE(r->phiHat, i) - (double)an * RE(r->outn, i));
                        Rhat2 = (float)(IM(r->phiHat, i) - (double)an * IM(r->outn, i));
                    }
                    RE(r->phiHat, i) = Rhat1 / (1.0 + (double)an);
                    IM(r->phiHat, i) = Rhat2 / (1.0 + (double)an);
                    const float ac = mc * dt * kk;
                    const float Rhat3 = (float)(RE(r->conHat, i) - (double)ac * RE(r->outc, i));
                    const float Rhat4 = (float)(IM(r->conHat, i) - (double)ac * IM(r->outc, i));
                    const float dc = mc * dt * alpha * kk * kk;
                    RE(r->conHat, i) = Rhat3 / (1.0 + (double)dc);
                    IM(r->conHat, i) = Rhat4 / (1.0 + (double)dc);
                } else {
                    const double kk = ks_d(r, l, m, n);
                    double nre = 0.0, nim = 0.0;
                    if (noise) {
                        const double detrx = (l == 0), detrxn = (l == L / 2), detry = (m == 0), detryn = (m == M / 2);
                        const double lp = 0.5 - 0.5 * tanh((sqrt(kk) - 2.0 * PI_REF) / 0.1);
                        nre = (double)dt * r->b0 * RE(r->noisf, i) * sqrt(kk) *
                              sqrt(fabs(0.5 + 0.5 * (detrx + detrxn) * (detry + detryn))) * lp;
                        nim = (double)dt * r->b0 * IM(r->noisf, i) * sqrt(kk) *
                              sqrt(fabs(0.5 - 0.5 * (detrx + detrxn) * (detry + detryn))) * lp;
                    }
                    const double an = (double)mn * dt * kk;
                    RE(r->phiHat, i) = (RE(r->phiHat, i) - an * RE(r->outn, i) + nre) / (1.0 + an);
                    IM(r->phiHat, i) = (IM(r->phiHat, i) - an * IM(r->outn, i) + nim) / (1.0 + an);
                    const double ac = (double)mc * dt * kk;
                    const double dc = (double)mc * dt * alpha * kk * kk;
                    RE(r->conHat, i) = (RE(r->conHat, i) - ac * RE(r->outc, i)) / (1.0 + dc);
                    IM(r->conHat, i) = (IM(r->conHat, i) - ac * IM(r->outc, i)) / (1.0 + dc);
                }
            }
}

/* UPDATEINC2GRA (MIS:877-925): |grad c|^2 with the grao2-twice term of MIS:915. */
static void update_inc2gra(orc_run *r) {
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    for (int l = 0; l < L; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) {
                const long i = n + (long)N * (m + (long)M * l);
                const double kl = r->p.exact ? (double)r->krefl[l] : r->kdl[l];
                const double km = r->p.exact ? (double)r->krefm[m] : r->kdm[m];
                const double kn = r->p.exact ? (double)r->krefn[n] : r->kdn[n];
                RE(r->gra1, i) = 1.0 * kl * IM(r->conHat, i);
                IM(r->gra1, i) = -1.0 * kl * RE(r->conHat, i);
                RE(r->gra2, i) = 1.0 * km * IM(r->conHat, i);
                IM(r->gra2, i) = -1.0 * km * RE(r->conHat, i);
                RE(r->gra3, i) = 1.0 * kn * IM(r->conHat, i);
                IM(r->gra3, i) = -1.0 * kn * RE(r->conHat, i);
            }
    fft_bwd(r, r->gra1, r->grao1);
    fft_bwd(r, r->gra2, r->grao2);
    fft_bwd(r, r->gra3, r->grao3);
    for (long i = 0; i < r->P; ++i) {
        RE(r->grao1, i) = RE(r->grao1, i) / L / M / N;
        IM(r->grao1, i) = IM(r->grao1, i) / L / M / N;
        RE(r->grao2, i) = RE(r->grao2, i) / L / M / N;
        IM(r->grao2, i) = IM(r->grao2, i) / L / M / N;
        RE(r->grao3, i) = RE(r->grao3, i) / L / M / N;
        IM(r->grao3, i) = IM(r->grao3, i) / L / M / N;
        RE(r->grac, i) = pow(RE(r->grao1, i), 2) + pow(RE(r->grao2, i), 2) + pow(RE(r->grao2, i), 2);
        IM(r->grac, i) = 0.0;
    }
}

/* UPDATECOEF (MIS:686-697). */
static void update_coef(orc_run *r) {
    const int LMN = r->p.L * r->p.M * r->p.N;
    for (long i = 0; i < r->P; ++i) {
        RE(r->phi, i) = RE(r->phi, i) / LMN;
        IM(r->phi, i) = 0;
        RE(r->con, i) = RE(r->con, i) / LMN;
        IM(r->con, i) = 0.0;
    }
}

/* One step: MIS:479-501 (Misfit, with Gauss+p5 and MAINEQUATIONC2_NOI) or
 * CVD:400-422 (CVD, MAINEQUATIONC2MIX). */
void orc_step(orc_run *r, int t) {
    update_inn3(r);
    update_infmix(r);
    fft_fwd(r, r->phi, r->phiHat);   /* p1 */
    update_infcmix(r);
    update_inc2mix(r);
    update_inc2mixc(r);
    fft_fwd(r, r->inn, r->outn);     /* p8 */
    fft_fwd(r, r->inc, r->outc);     /* p9 */
    fft_fwd(r, r->con, r->conHat);   /* p6 */
    if (r->p.model == ORC_MODEL_MISFIT) {
        if (r->b0 != 0.0f) {
            gauss_noise(r, t);
            fft_fwd(r, r->nois, r->noisf); /* p5 */
        }
        main_equation(r, 1);
    } else {
        main_equation(r, 0);
    }
    update_inc2gra(r);
    fft_bwd(r, r->phiHat, r->phi);   /* p2 */
    fft_bwd(r, r->conHat, r->con);   /* p7 */
    update_coef(r);
    update_infcmix(r);
}

void orc_get_fields(const orc_run *r, double *phi, double *con) {
    for (long i = 0; i < r->P; ++i) {
        if (phi) phi[i] = RE(r->phi, i);
        if (con) con[i] = RE(r->con, i);
    }
}

void orc_set_fields(orc_run *r, const double *phi, const double *con) {
    for (long i = 0; i < r->P; ++i) {
        if (phi) {
            RE(r->phi, i) = phi[i];
            IM(r->phi, i) = 0.0;
        }
        if (con) {
            RE(r->con, i) = con[i];
            IM(r->con, i) = 0.0;
        }
    }
}

void orc_get_c2(const orc_run *r, float *c2a, float *c2b) {
    memcpy(c2a, r->C2AHat, sizeof(float) * (size_t)r->P);
    memcpy(c2b, r->C2BHat, sizeof(float) * (size_t)r->P);
}

void orc_get_kref(const orc_run *r, float *kl, float *km, float *kn) {
    memcpy(kl, r->krefl, sizeof(float) * (size_t)r->p.L);
    memcpy(km, r->krefm, sizeof(float) * (size_t)r->p.M);
    memcpy(kn, r->krefn, sizeof(float) * (size_t)r->p.N);
}

/* ENERGYC2 (MIS:1043-1092): float energy terms, double accumulation in l,m,n order. */
void orc_energy(const orc_run *r, double *e_over_p, double *mass_over_p) {
    const double niu = r->k.niu, ksi = r->k.ksi, w = r->k.para_w, c0 = r->k.para_c0, alpha = r->k.para_alpha;
    double EEsum = 0., DSsum = 0.;
    for (long i = 0; i < r->P; ++i) {
        const double ph = RE(r->phi, i), c = RE(r->con, i);
        if (r->p.exact) {
            const float e_id = (float)(pow(ph, 2) / 2.0 - niu * pow(ph, 3) / 6.0 + ksi * pow(ph, 4) / 12.0);
            const float e_mix =
                (float)((ph + 1.0) * w * (c * log(c / c0) + (1.0 - c) * log((1.0 - c) / (1.0 - c0))));
            const float e_ex = (float)(0.5 * ph * (RE(r->in3, i)) + alpha * RE(r->grac, i));
            const double denei = e_id + e_mix + e_ex;
            EEsum += denei;
        } else {
            const double e_id = pow(ph, 2) / 2.0 - niu * pow(ph, 3) / 6.0 + ksi * pow(ph, 4) / 12.0;
            const double e_mix = (ph + 1.0) * w * (c * log(c / c0) + (1.0 - c) * log((1.0 - c) / (1.0 - c0)));
            const double e_ex = 0.5 * ph * (RE(r->in3, i)) + alpha * RE(r->grac, i);
            EEsum += e_id + e_mix + e_ex;
        }
        DSsum += ph;
    }
    const int L = r->p.L, M = r->p.M, N = r->p.N;
    if (e_over_p) *e_over_p = EEsum / L / M / N;
    if (mass_over_p) *mass_over_p = DSsum / L / M / N;
}

/* ------------------------------------------------------------------------- */
/* Misfit peak finder (MIS:3261-3556).                                        */
/* ------------------------------------------------------------------------- */
static double nbv_d(const double *buf, long idx) {
    const double v = buf[idx];
    return isfinite(v) ? v : -INFINITY;
}

int orc_phimax_misfit(const double *phi, const double *con, int L, int M, float dx, float con0, double *out5, int cap,
                      int *num_found_raw) {
    /* buf / bufc: rows 0..L+1; the single-rank MPI stubs copy row 1 into row 0 and
     * row L into row L+1 (MIS:3289-3290, COM:101-110): edge replication in x. */
    const int n0 = L;
    const int N = 1;
    double *buf = (double *)calloc((size_t)M * (n0 + 2), sizeof(double));
    double *bufc = (double *)calloc((size_t)M * (n0 + 2), sizeof(double));
    for (int l = 1; l < n0 + 1; l++)
        for (int m = 0; m < M; m++) {
            buf[m + (long)M * l] = phi[m + (long)M * (l - 1)];
            bufc[m + (long)M * l] = con[m + (long)M * (l - 1)];
        }
    memcpy(buf, buf + M, sizeof(double) * M);
    memcpy(buf + (long)M * (n0 + 1), buf + (long)M * n0, sizeof(double) * M);
    memcpy(bufc, bufc + M, sizeof(double) * M);
    memcpy(bufc + (long)M * (n0 + 1), bufc + (long)M * n0, sizeof(double) * M);

    double global_max_phi = -INFINITY;
    int global_max_m = 0, global_max_l = 1;
    for (int l = 1; l < n0 + 1; ++l)
        for (int m = 0; m < M; ++m) {
            const double v = buf[m + (long)M * l];
            if (!isfinite(v)) continue;
            global_max_phi = global_max_phi > v ? global_max_phi : v; /* std::max(a, b): a < b ? b : a */
            if (v >= global_max_phi) {
                global_max_m = m;
                global_max_l = l;
            }
        }

    int num_atoms = 0;
    const long max_atoms = (long)M * n0 * N;
    for (int n = 0; n < N; n++)
        for (int m = 0; m < M; m++)
            for (int l = 1; l < n0 + 1; l++) {
                const double center = buf[m + (long)M * l];
                if (!isfinite(center) || center <= -0.07) continue;
                const int lf = l - 1, lb = l + 1;
                int mf = m - 1, mb = m + 1;
                if (mf < 0) mf = M - 1;
                if (mb > M - 1) mb = 0;
                const double nbs[8] = {nbv_d(buf, m + (long)M * lf),  nbv_d(buf, m + (long)M * lb),
                                       nbv_d(buf, mf + (long)M * l),  nbv_d(buf, mb + (long)M * l),
                                       nbv_d(buf, mb + (long)M * lb), nbv_d(buf, mb + (long)M * lf),
                                       nbv_d(buf, mf + (long)M * lb), nbv_d(buf, mf + (long)M * lf)};
                int ge_all = 1, gt_any = 0;
                for (int q = 0; q < 8; ++q) {
                    if (center < nbs[q]) ge_all = 0;
                    if (center > nbs[q]) gt_any = 1;
                }
                if (!(ge_all && gt_any)) continue;
                const double xtemp = (double)((float)(0 + l + 1) * dx);
                const double ytemp = (double)((float)(m + 1) * dx);
                const double ztemp = (double)((float)(n + 1) * dx);
                const double z0 = center;
                const double z1 = buf[m + (long)M * lb];
                const double z3 = buf[m + (long)M * lf];
                const double z4 = buf[mb + (long)M * l];
                const double z2 = buf[mf + (long)M * l];
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
                    const double half_dx = 0.5 * dx_d;
                    delta_x = delta_x < -half_dx ? -half_dx : (half_dx < delta_x ? half_dx : delta_x);
                    delta_y = delta_y < -half_dx ? -half_dx : (half_dx < delta_y ? half_dx : delta_y);
                    double phi_interp = z0;
                    if (isfinite(a3) && fabs(a3) > eps && isfinite(a1)) phi_interp -= 0.25 * a1 * a1 / a3;
                    if (isfinite(a4) && fabs(a4) > eps && isfinite(a2)) phi_interp -= 0.25 * a2 * a2 / a4;
                    if (isfinite(phi_interp)) phi_local = phi_interp;
                }
                if (num_atoms < max_atoms) {
                    if (num_atoms < cap) {
                        double *o = out5 + 5L * num_atoms;
                        o[0] = xtemp + delta_x;
                        o[1] = ytemp + delta_y;
                        o[2] = ztemp;
                        o[3] = phi_local;
                        const double c = bufc[m + (long)M * l];
                        o[4] = (double)(isfinite(c) ? (float)c : con0);
                    }
                    num_atoms++;
                }
            }
    if (num_found_raw) *num_found_raw = num_atoms;
    if (num_atoms == 0) {
        const double dx_d = (double)dx;
        if (cap > 0) {
            out5[0] = (0 + global_max_l + 1) * dx_d;
            out5[1] = (global_max_m + 1) * dx_d;
            out5[2] = dx_d;
            out5[3] = isfinite(global_max_phi) ? global_max_phi : 0.0;
            const double c = bufc[global_max_m + (long)M * global_max_l];
            out5[4] = (double)(isfinite(c) ? (float)c : con0);
        }
        num_atoms = 1;
    }
    free(buf);
    free(bufc);
    return num_atoms;
}

/* ------------------------------------------------------------------------- */
/* Elastic peak finder (ELA:2802-2921).                                       */
/* ------------------------------------------------------------------------- */
int orc_phimax_elastic(const double *phi, int L, int M, int N, float dx, double *out4, int cap) {
    const int n0 = L;
    const long P = (long)L * M * N;
    const long total = (long)M * N * (n0 + 2);
    float phimax = 0, phicut = 0.40f;
    for (long i = 0; i < P; ++i)
        if (phi[i] > phimax) phimax = (float)phi[i];
    const float pii = phimax;
    const float phic = (pii - pii * phicut);
    float *buf = (float *)calloc((size_t)total, sizeof(float));
    for (int l = 1; l < n0 + 1; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) buf[n + (long)N * (m + (long)M * l)] = (float)phi[n + (long)N * (m + (long)M * (l - 1))];
    memcpy(buf, buf + (long)M * N, sizeof(float) * (size_t)M * N);
    memcpy(buf + (long)M * N * (n0 + 1), buf + (long)M * N * n0, sizeof(float) * (size_t)M * N);

    int num_atoms = 0;
    for (int l = 1; l < n0 + 1; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) {
                const long c = n + (long)N * (m + (long)M * l);
                if (!(buf[c] > phic)) continue;
                const int lf = l - 1, lb = l + 1;
                int mf = m - 1, mb = m + 1, nf = n - 1, nb = n + 1;
                if (mf < 0) mf = M - 1;
                if (mb > M - 1) mb = 0;
                if (nf < 0) nf = N - 1;
                if (nb > N - 1) nb = 0;
                int mark = 1;
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
                            /* Out-of-range reads of the reference (ELA:2879 at the first and
                             * last buffer element) are defined as -inf: they never reject. */
                            if (idx < 0 || idx >= total) continue;
                            if (buf[idx] > buf[c]) mark = 0;
                        }
                if (mark != 1) continue;
                const double xtemp = (double)(0 + l), ytemp = (double)m, ztemp = (double)n;
                const double z0 = buf[c];
                const double z1 = buf[n + (long)N * (m + (long)M * lb)];
                const double z3 = buf[n + (long)N * (m + (long)M * lf)];
                const double z4 = buf[n + (long)N * (mb + (long)M * l)];
                const double z2 = buf[n + (long)N * (mf + (long)M * l)];
                const double z5 = buf[nb + (long)N * (m + (long)M * l)];
                const double z6 = buf[nf + (long)N * (m + (long)M * l)];
                const double a0 = z0;
                const double a1 = 0.5 * (z1 - z3) / dx + 10e-8;
                const double a2 = 0.5 * (z4 - z2) / dx + 10e-8;
                const double a3 = 0.5 * (z1 + z3 - 2. * z0) / (dx * dx) + 10e-8;
                const double a4 = 0.5 * (z2 + z4 - 2. * z0) / (dx * dx) + 10e-8;
                const double a5 = 0.5 * (z5 - z6) / dx + 10e-8;
                const double a6 = 0.5 * (z5 + z6 - 2. * z0) / (dx * dx) + 10e-8;
                const double delta_x = -a1 / (2. * a3);
                const double delta_y = -a2 / (2. * a4);
                const double delta_z = -a5 / (2. * a6);
                if (num_atoms < cap) {
                    double *o = out4 + 4L * num_atoms;
                    o[0] = (xtemp + 1) * dx + delta_x;
                    o[1] = (ytemp + 1) * dx + delta_y;
                    o[2] = (ztemp + 1) * dx + delta_z;
                    o[3] = a0 - 0.25 * a1 * a1 / a3 - 0.25 * a2 * a2 / a4 - 0.25 * a5 * a5 / a6;
                }
                num_atoms++;
            }
    free(buf);
    return num_atoms;
}

/* min3 (COM:241-244). */
static float min3f(float a, float b, float c) {
    float aa = fabsf(a), bb = fabsf(b), cc = fabsf(c);
    return ((aa < bb ? aa : bb) < cc) ? (aa < bb ? aa : bb) : cc;
}

/* ------------------------------------------------------------------------- */
/* elastic3D (ELA:3586-3729).                                                 */
/* ------------------------------------------------------------------------- */
void orc_elastic3d(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                   float benchel, double *strain, uint32_t *nb) {
    const int CNmax = 16;
    const double kels = 1.0;
    const float frame_x = (float)L * dx, frame_y = (float)M * dx, frame_z = (float)N * dx;
    for (int i = 0; i < n; i++) {
        unsigned Nb = 0;
        double sx = 0, sy = 0, sz = 0;
        float rjx = 0, rjy = 0, rjz = 0;
        for (int j = 0; j < n; j++) {
            if (i == j) continue;
            float r3[9];
            r3[0] = (float)(x[i] - x[j]);
            r3[1] = (float)(y[i] - y[j]);
            r3[2] = (float)(z[i] - z[j]);
            r3[3] = r3[0] + frame_x;
            r3[4] = r3[1] + frame_y;
            r3[5] = r3[2] + frame_z;
            r3[6] = r3[0] - frame_x;
            r3[7] = r3[1] - frame_y;
            r3[8] = r3[2] - frame_z;
            const float drx = min3f(fabsf(r3[0]), fabsf(r3[3]), fabsf(r3[6]));
            const float dry = min3f(fabsf(r3[1]), fabsf(r3[4]), fabsf(r3[7]));
            const float drz = min3f(fabsf(r3[2]), fabsf(r3[5]), fabsf(r3[8]));
            const float rr = sqrtf(drx * drx + dry * dry + drz * drz);
            if (!(rr < benchel && rr > 0.7)) continue;
            Nb = Nb + 1;
            if (!(Nb <= (unsigned)CNmax && Nb > 0)) continue;
            const double rij = rr;
            for (int ii = 0; ii < 7; ii += 3)
                if (fabsf(fabsf(r3[ii]) - drx) < 1e-3) rjx = (float)(x[i] - r3[ii]);
            for (int ii = 1; ii < 8; ii += 3)
                if (fabsf(fabsf(r3[ii]) - dry) < 1e-3) rjy = (float)(y[i] - r3[ii]);
            for (int ii = 2; ii < 9; ii += 3)
                if (fabsf(fabsf(r3[ii]) - drz) < 1e-3) rjz = (float)(z[i] - r3[ii]);
            const double cos_near = ((double)rjx - x[i]) / rij;
            const double sin_near = ((double)rjy - y[i]) / rij;
            const double tha_near = ((double)rjz - z[i]) / rij;
            double snx = 0.0, sny = 0.0, snz = 0.0; /* uninitialised in the reference when rij >= 1.3 */
            if (rij < 1.3) snx = kels * (rij - 1) * cos_near;
            sx = sx + snx;
            if (rij < 1.3) sny = kels * (rij - 1) * sin_near;
            sy = sy + sny;
            if (rij < 1.3) snz = kels * (rij - 1) * tha_near;
            sz = sz + snz;
        }
        strain[i] = sqrt(sx * sx + sy * sy + sz * sz);
        nb[i] = Nb;
    }
}

/* ------------------------------------------------------------------------- */
/* Spherical harmonics (COM:274-343), float arithmetic.                       */
/* ------------------------------------------------------------------------- */
static unsigned long facto(int h) {
    int g = 1;
    for (int i = 1; i <= h; i++) g = g * i;
    return (unsigned long)g;
}

static float lg_poly(int l, float x) {
    float plm2 = 1, plm1 = x, pl = 0;
    if (l == 0) return 1;
    if (l == 1) return x;
    for (int i = 2; i <= l; i++) {
        pl = ((2 * i - 1) * x * (float)(plm1) - (i - 1) * plm2) / (float)(i);
        plm2 = plm1;
        plm1 = pl;
    }
    return pl;
}

static float plgndr(int l, int m, float x) {
    float fact, pll = 0, pmm, pmmp1, somx2;
    if (m < 0) m = -m;
    if (m == 0) return lg_poly(l, x);
    pmm = 1.0f;
    if (m > 0) {
        somx2 = (float)sqrt((1.0 - x) * (1.0 + x));
        fact = 1.0f;
        for (int i = 1; i <= m; i++) {
            pmm *= -fact * somx2;
            fact = (float)(fact + 2.0);
        }
    }
    if (l == m) return pmm;
    pmmp1 = x * (2 * m + 1) * pmm;
    if (l == (m + 1)) return pmmp1;
    for (int ll = m + 2; ll <= l; ll++) {
        pll = (x * (2 * ll - 1) * pmmp1 - (ll + m - 1) * pmm) / (ll - m);
        pmm = pmmp1;
        pmmp1 = pll;
    }
    return pll;
}

static float ylm_r(int l, int m, float theta, float fai) {
    if (m < 0) m = -m;
    const float fnorm = (float)(pow(-1.0, m) * sqrt((2 * l + 1) / 4. / PI_REF) *
                                (double)sqrtf((float)(facto(l - m)) / (float)(facto(l + m))));
    const float plm = plgndr(l, m, cosf(theta));
    const float comp_m = cosf(m * fai);
    return fnorm * plm * comp_m;
}

static float ylm_c(int l, int m, float theta, float fai) {
    float fnorm, plm, comp_m;
    if (m < 0) {
        m = -m;
        fnorm = (float)(pow(-1.0, m + m) * sqrt((2 * l + 1) / 4. / PI_REF) *
                        (double)sqrtf((float)(facto(l - m)) / (float)(facto(l + m))));
        plm = plgndr(l, m, cosf(theta));
        comp_m = -sinf(m * fai);
    } else {
        fnorm = (float)(pow(-1.0, m) * sqrt((2 * l + 1) / 4. / PI_REF) *
                        (double)sqrtf((float)(facto(l - m)) / (float)(facto(l + m))));
        plm = plgndr(l, m, cosf(theta));
        comp_m = sinf(m * fai);
    }
    return fnorm * plm * comp_m;
}

/* ------------------------------------------------------------------------- */
/* cryst_order (ELA:3013-3319).  Both passes use l = 6 (ELA:3155 and 3238) and the */
/* per-atom accumulator is not reset between them, as in the reference.        */
/* ------------------------------------------------------------------------- */
void orc_cryst_order(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                     double *q4, double *q6) {
    const int CNmax = 16;
    const float bench100_h = 1.2f;
    const float frame_x = (float)L * dx, frame_y = (float)M * dx, frame_z = (float)N * dx;
    unsigned *Nb = (unsigned *)calloc((size_t)n + 1, sizeof(unsigned));
    double *theta = (double *)calloc((size_t)n * CNmax + 1, sizeof(double));
    double *fai = (double *)calloc((size_t)n * CNmax + 1, sizeof(double));
    int *nb_index = (int *)calloc((size_t)n * CNmax + 1, sizeof(int));
    for (int i = 0; i < n; i++) {
        float rjx = 0, rjy = 0, rjz = 0;
        for (int j = 0; j < n; j++) {
            if (i == j) continue;
            float r3[9];
            r3[0] = (float)(x[i] - x[j]);
            r3[1] = (float)(y[i] - y[j]);
            r3[2] = (float)(z[i] - z[j]);
            r3[3] = r3[0] + frame_x;
            r3[4] = r3[1] + frame_y;
            r3[5] = r3[2] + frame_z;
            r3[6] = r3[0] - frame_x;
            r3[7] = r3[1] - frame_y;
            r3[8] = r3[2] - frame_z;
            const float drx = min3f(fabsf(r3[0]), fabsf(r3[3]), fabsf(r3[6]));
            const float dry = min3f(fabsf(r3[1]), fabsf(r3[4]), fabsf(r3[7]));
            const float drz = min3f(fabsf(r3[2]), fabsf(r3[5]), fabsf(r3[8]));
            const float rr = sqrtf(drx * drx + dry * dry + drz * drz);
            if (!(rr < bench100_h)) continue;
            Nb[i] = Nb[i] + 1;
            if (!(Nb[i] <= (unsigned)CNmax && Nb[i] > 0)) continue;
            const long k = Nb[i] - 1 + (long)CNmax * i;
            const double rij = rr;
            for (int ii = 0; ii < 7; ii += 3)
                if (fabsf(fabsf(r3[ii]) - drx) < 1e-3) rjx = (float)(x[i] - r3[ii]);
            for (int ii = 1; ii < 8; ii += 3)
                if (fabsf(fabsf(r3[ii]) - dry) < 1e-3) rjy = (float)(y[i] - r3[ii]);
            for (int ii = 2; ii < 9; ii += 3)
                if (fabsf(fabsf(r3[ii]) - drz) < 1e-3) rjz = (float)(z[i] - r3[ii]);
            const double CoX = rjx, CoY = rjy, CoZ = rjz;
            theta[k] = acos((CoZ - z[i]) / (rij + 1.e-4));
            fai[k] = atan((CoY - y[i]) / (CoX - x[i] + 1.e-4));
            if ((CoX - x[i]) < 0.) fai[k] = fai[k] + PI_REF;
            nb_index[k] = j;
        }
    }
    double *qlmb = (double *)calloc(2 * (size_t)n + 2, sizeof(double));
    double *qlmbar = (double *)calloc(2 * (size_t)n + 2, sizeof(double));
    double *qlmb_m = (double *)calloc((size_t)n + 1, sizeof(double));
    for (int pass = 0; pass < 2; ++pass) {
        const int LL = 6;
        for (int m = -LL; m <= LL; m++) {
            for (int ii = 0; ii < n; ii++) qlmb[2 * ii] = qlmb[2 * ii + 1] = qlmbar[2 * ii] = qlmbar[2 * ii + 1] = 0.;
            for (int i = 0; i < n; i++) {
                if (!(Nb[i] > 0 && Nb[i] <= (unsigned)CNmax)) continue;
                for (int j = 0; j < (int)Nb[i]; j++) {
                    const long k = j + (long)CNmax * i;
                    qlmb[2 * i] += ylm_r(LL, m, (float)theta[k], (float)fai[k]);
                    qlmb[2 * i + 1] += ylm_c(LL, m, (float)theta[k], (float)fai[k]);
                    if (j == (int)Nb[i] - 1) {
                        qlmb[2 * i] = qlmb[2 * i] / (float)(Nb[i]);
                        qlmb[2 * i + 1] = qlmb[2 * i + 1] / (float)(Nb[i]);
                    }
                }
            }
            for (int i = 0; i < n; i++) {
                if (!(Nb[i] > 0 && Nb[i] <= (unsigned)CNmax)) continue;
                for (int j = 0; j < (int)Nb[i]; j++) {
                    const int jj = nb_index[j + (long)CNmax * i];
                    qlmbar[2 * i] += qlmb[2 * jj];
                    qlmbar[2 * i + 1] += qlmb[2 * jj + 1];
                    if (j == (int)Nb[i] - 1) {
                        qlmbar[2 * i] = (qlmb[2 * i] + qlmbar[2 * i]) / (float)(Nb[i] + 1);
                        qlmbar[2 * i + 1] = (qlmb[2 * i + 1] + qlmbar[2 * i + 1]) / (float)(Nb[i] + 1);
                    }
                }
            }
            for (int i = 0; i < n; i++) qlmb_m[i] += qlmbar[2 * i] * qlmbar[2 * i] + qlmbar[2 * i + 1] * qlmbar[2 * i + 1];
        }
        const double xishu = 4 * PI_REF / (float)(2 * LL + 1);
        for (int i = 0; i < n; i++) {
            if (pass == 0)
                q4[i] = sqrt(xishu * qlmb_m[i]);
            else
                q6[i] = sqrt(xishu * qlmb_m[i]);
        }
    }
    free(qlmb);
    free(qlmbar);
    free(qlmb_m);
    free(Nb);
    free(theta);
    free(fai);
    free(nb_index);
}

/* ------------------------------------------------------------------------- */
/* CVD checkpoint analysis: atompositionCFGC2 (CVD:1067-1275), GR (CVD:1277-1347), */
/* Q6_GLO (CVD:1349-1520).  Single rank: the x halo planes are copies of the     */
/* first and last plane (the MPI_Sendrecv stub copies a rank's own plane,        */
/* COM:101-110); neighbours are taken at flat offsets +-1 (n), +-N (m) and       */
/* +-N*M (l) of the haloed buffer, without wrap, as the reference indexes them.  */
/* ------------------------------------------------------------------------- */
int orc_cvd_atoms(const float *phi, int L, int M, int N, float dx, float u0, float *phic_out, float *phimax_out,
                  float *out4, int cap) {
    const float phi_rat = 0.618f;
    const long P = (long)L * M * N, NM = (long)N * M;
    float phimax = -1.0f; /* phimm */
    for (long i = 0; i < P; i++)
        if (phi[i] > phimax) phimax = phi[i];
    const float t = (phimax - u0) * phi_rat;
    const float phic = u0 + t;
    *phic_out = phic;
    *phimax_out = phimax;
    float *buf = (float *)malloc(sizeof(float) * (size_t)(NM * (L + 2)));
    for (int lp = 0; lp < L + 2; lp++) {
        const int src = lp == 0 ? 0 : (lp == L + 1 ? L - 1 : lp - 1);
        memcpy(buf + lp * NM, phi + src * NM, sizeof(float) * (size_t)NM);
    }
    const float frame_x = (float)L * dx, frame_y = (float)M * dx, frame_z = (float)N * dx;
    int num = 0;
    for (int l = 1; l < L + 1; l++)
        for (int m = 0; m < M; m++)
            for (int n = 0; n < N; n++) {
                const long idx = n + (long)N * (m + (long)M * l);
                const float v = buf[idx];
                if (!(v >= phic)) continue;
                if (!(v >= buf[idx - NM] && v >= buf[idx + NM])) continue;
                if (!(v >= buf[idx - N] && v >= buf[idx + N])) continue;
                if (!(v >= buf[idx - 1] && v >= buf[idx + 1])) continue;
                if (num < cap) {
                    const float yd = (float)(m + 1) * dx, zd = (float)(n + 1) * dx, xd = (float)l * dx;
                    out4[4 * num] = yd / frame_y;
                    out4[4 * num + 1] = zd / frame_z;
                    out4[4 * num + 2] = xd / frame_x;
                    out4[4 * num + 3] = v;
                }
                num++;
            }
    free(buf);
    if (num == 0) {
        if (cap > 0) {
            out4[0] = -1.0f;
            out4[1] = -1.0f;
            out4[2] = -1.0f;
            out4[3] = 0.0f;
        }
        num = 1;
    }
    return num;
}

/* Pair geometry shared by GR and Q6_GLO (CVD:1297-1310): the minimum-image
 * components (each scaled by the reference's frame of that slot) and the distance
 * rr = sqrt(...) + 1e-6, the sum taken in double and stored to float. */
static float cvd_pair(const float *x, const float *y, const float *z, int i, int j, float fx, float fy, float fz,
                      float *r3, float *drx, float *dry, float *drz) {
    r3[0] = (x[i] - x[j]) * fx;
    r3[1] = (y[i] - y[j]) * fy;
    r3[2] = (z[i] - z[j]) * fz;
    r3[3] = r3[0] + fx;
    r3[4] = r3[1] + fy;
    r3[5] = r3[2] + fz;
    r3[6] = r3[0] - fx;
    r3[7] = r3[1] - fy;
    r3[8] = r3[2] - fz;
    *drx = min3f(r3[0], r3[3], r3[6]);
    *dry = min3f(r3[1], r3[4], r3[7]);
    *drz = min3f(r3[2], r3[5], r3[8]);
    const float s = *drx * *drx + *dry * *dry + *drz * *drz;
    return (float)((double)sqrtf(s) + 1e-6);
}

int orc_cvd_gr_hist(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx,
                    unsigned *hist, int cap) {
    const float a_lattice = 1.0f;
    const float delr = (float)(a_lattice / 25.);
    const int maxbin = (int)(((float)L * dx) / delr);
    /* the reference scales x by L*dx, y by M*dx, z by N*dx although the records hold
     * (y, z, x) fractions (CVD:1297-1299); reproduced */
    const float fx = (float)L * dx, fy = (float)M * dx, fz = (float)N * dx;
    for (int b = 0; b < maxbin && b < cap; b++) hist[b] = 0;
    for (int i = 0; i < n - 1; i++)
        for (int j = i + 1; j < n; j++) {
            float r3[9], drx, dry, drz;
            const float rr = cvd_pair(x, y, z, i, j, fx, fy, fz, r3, &drx, &dry, &drz);
            const unsigned bin = (unsigned)(int)(rr / delr);
            if ((double)rr > (double)a_lattice / sqrt(2.) * 0.5 && bin < (unsigned)maxbin && (int)bin < cap)
                hist[bin] = hist[bin] + 2;
        }
    return maxbin;
}

void orc_cvd_q6(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, unsigned *Nb,
                float *ql_out, float *ql_global, unsigned *histq) {
    const int CNmax = 24, l = 6;
    const float a_lattice = 1.0f;
    const float fx = (float)L * dx, fy = (float)M * dx, fz = (float)N * dx;
    float *rij = (float *)calloc((size_t)n * CNmax + 1, sizeof(float));
    float *CoX = (float *)calloc((size_t)n * CNmax + 1, sizeof(float));
    float *CoY = (float *)calloc((size_t)n * CNmax + 1, sizeof(float));
    float *CoZ = (float *)calloc((size_t)n * CNmax + 1, sizeof(float));
    float *theta = (float *)calloc((size_t)n * CNmax + 1, sizeof(float));
    float *fai = (float *)calloc((size_t)n * CNmax + 1, sizeof(float));
    const double rhi = (double)a_lattice * sqrt(3.) / 2. * 1.2 + 1e-3;
    const double rlo = (double)a_lattice * sqrt(3.) / 2. * 0.9 - 1e-3;
    float rjx = 0, rjy = 0, rjz = 0;
    for (int i = 0; i < n; i++) {
        Nb[i] = 0;
        for (int j = 0; j < n; j++) {
            if (i == j) continue;
            float r3[9], drx, dry, drz;
            const float rr = cvd_pair(x, y, z, i, j, fx, fy, fz, r3, &drx, &dry, &drz);
            if (!((double)rr <= rhi && (double)rr >= rlo)) continue;
            Nb[i] = Nb[i] + 1;
            if (Nb[i] > (unsigned)CNmax) continue;
            rij[Nb[i] - 1 + CNmax * i] = rr;
            for (int ii = 0; ii < 7; ii += 3)
                if ((double)(fabsf(r3[ii]) - drx) < 1e-5) rjx = x[i] * fx - r3[ii];
            for (int ii = 1; ii < 8; ii += 3)
                if ((double)(fabsf(r3[ii]) - dry) < 1e-5) rjy = y[i] * fy - r3[ii];
            for (int ii = 2; ii < 9; ii += 3)
                if ((double)(fabsf(r3[ii]) - drz) < 1e-5) rjz = z[i] * fz - r3[ii];
            CoX[Nb[i] - 1 + CNmax * i] = rjx;
            CoY[Nb[i] - 1 + CNmax * i] = rjy;
            CoZ[Nb[i] - 1 + CNmax * i] = rjz;
        }
    }
    for (int i = 0; i < n; i++) {
        if (!(Nb[i] > 0 && Nb[i] <= (unsigned)CNmax)) continue;
        for (int j = 0; j < (int)Nb[i]; j++) {
            const int k = j + CNmax * i;
            theta[k] = acosf((CoZ[k] - z[i] * fz) / rij[k]);
            const float dyv = CoY[k] - y[i] * fy;
            if (dyv == 0.) fai[k] = 0.f;
            else fai[k] = atanf(dyv / (CoX[k] - x[i] * fx));
        }
    }
    float *qlmb_m = (float *)calloc((size_t)n + 1, sizeof(float));
    double *qre = (double *)calloc((size_t)n + 1, sizeof(double)), *qim = (double *)calloc((size_t)n + 1, sizeof(double));
    float Qlm_m = 0.f;
    for (int m = -l; m <= l; m++) {
        for (int i = 0; i < n; i++) {
            double ar = 0.0, ai = 0.0;
            qre[i] = 0.0;
            qim[i] = 0.0;
            if (Nb[i] > 0 && Nb[i] <= (unsigned)CNmax)
                for (int j = 0; j < (int)Nb[i]; j++) {
                    ar += (double)ylm_r(l, m, theta[j + CNmax * i], fai[j + CNmax * i]);
                    ai += (double)ylm_c(l, m, theta[j + CNmax * i], fai[j + CNmax * i]);
                    if (j == (int)Nb[i] - 1) {
                        qre[i] = ar / (double)(float)Nb[i];
                        qim[i] = ai / (double)(float)Nb[i];
                    }
                }
        }
        float SumNb = 0.f, Qlm_r = 0.f, Qlm_c = 0.f;
        for (int i = 0; i < n; i++) {
            qlmb_m[i] = (float)((double)qlmb_m[i] + (qre[i] * qre[i] + qim[i] * qim[i]));
            Qlm_r = (float)((double)Qlm_r + (double)Nb[i] * qre[i]);
            Qlm_c = (float)((double)Qlm_c + (double)Nb[i] * qim[i]);
            SumNb = SumNb + (float)Nb[i];
        }
        Qlm_r /= SumNb;
        Qlm_c /= SumNb;
        Qlm_m += (Qlm_r * Qlm_r + Qlm_c * Qlm_c);
    }
    const float delq = 0.05f;
    const float xishu = (float)(4 * PI_REF / (double)(float)(2 * l + 1));
    *ql_global = sqrtf(xishu * Qlm_m);
    for (int b = 0; b < 30; b++) histq[b] = 0;
    for (int i = 0; i < n; i++) {
        ql_out[i] = sqrtf(xishu * qlmb_m[i]);
        const unsigned bin = (unsigned)(int)(ql_out[i] / delq);
        if (bin < 30) histq[bin] = histq[bin] + 1;
    }
    free(rij);
    free(CoX);
    free(CoY);
    free(CoZ);
    free(theta);
    free(fai);
    free(qlmb_m);
    free(qre);
    free(qim);
}
