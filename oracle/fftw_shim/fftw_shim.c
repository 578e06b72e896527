/*
 * fftw_shim.c -- implementation of the five-symbol FFTW-3 API shim declared in
 * fftw3.h (oracle / test infrastructure only; never part of the product).
 *
 * Algorithm: a separable 3-D DFT.  Each axis is transformed line by line; a
 * line is gathered into a contiguous buffer, transformed, and scattered back.
 * Power-of-two lengths use an iterative radix-2 decimation-in-time
 * Cooley-Tukey FFT (bit-reversal permutation followed by log2(n) butterfly
 * levels) with twiddles exp(sign*2*pi*i*k/n) evaluated directly with cos/sin
 * for every k (no recurrences), so the transform is accurate to a few ulp of
 * double.  Other lengths fall back to the direct O(n^2) DFT with the twiddle
 * index reduced mod n.  Axis order is n2 (fastest), then n1, then n0.
 *
 * Conventions follow FFTW: FFTW_FORWARD = -1 uses exp(-2 pi i jk/n), the
 * backward sign +1; no normalisation; row-major layout with n2 fastest.
 */
#define _POSIX_C_SOURCE 200809L
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct fftw_plan_s {
    int n0, n1, n2;
    int sign;
    fftw_complex *in;
    fftw_complex *out;
};

typedef struct {
    int n;
    int sign;
    int log2n;
    double *wr; /* n/2 twiddle real parts (power-of-two case) or n (generic) */
    double *wi;
    int *rev;   /* bit reversal permutation (power-of-two case) */
} line_plan;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void line_plan_init(line_plan *lp, int n, int sign) {
    const double two_pi = 6.283185307179586476925286766559;
    lp->n = n;
    lp->sign = sign;
    lp->log2n = 0;
    lp->rev = NULL;
    if (is_pow2(n)) {
        while ((1 << lp->log2n) < n) lp->log2n++;
        int half = n / 2 > 0 ? n / 2 : 1;
        lp->wr = (double *)malloc(sizeof(double) * half);
        lp->wi = (double *)malloc(sizeof(double) * half);
        for (int k = 0; k < half; ++k) {
            double a = two_pi * (double)k / (double)n;
            lp->wr[k] = cos(a);
            lp->wi[k] = (double)sign * sin(a);
        }
        lp->rev = (int *)malloc(sizeof(int) * n);
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < lp->log2n; ++b)
                if (i & (1 << b)) r |= 1 << (lp->log2n - 1 - b);
            lp->rev[i] = r;
        }
    } else {
        lp->wr = (double *)malloc(sizeof(double) * n);
        lp->wi = (double *)malloc(sizeof(double) * n);
        for (int k = 0; k < n; ++k) {
            double a = two_pi * (double)k / (double)n;
            lp->wr[k] = cos(a);
            lp->wi[k] = (double)sign * sin(a);
        }
    }
}

static void line_plan_free(line_plan *lp) {
    free(lp->wr);
    free(lp->wi);
    free(lp->rev);
}

/* In-place transform of one contiguous line x[0..n) (scratch: tmp[0..n)). */
static void line_exec(const line_plan *lp, double *x, double *tmp) {
    const int n = lp->n;
    if (n == 1) return;
    if (lp->rev) {
        for (int i = 0; i < n; ++i) {
            tmp[2 * lp->rev[i]] = x[2 * i];
            tmp[2 * lp->rev[i] + 1] = x[2 * i + 1];
        }
        memcpy(x, tmp, sizeof(double) * 2 * n);
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1;
            const int step = n / len;
            for (int s = 0; s < n; s += len) {
                for (int j = 0; j < half; ++j) {
                    const double wr = lp->wr[j * step];
                    const double wi = lp->wi[j * step];
                    double *a = x + 2 * (s + j);
                    double *b = x + 2 * (s + j + half);
                    const double tr = b[0] * wr - b[1] * wi;
                    const double ti = b[0] * wi + b[1] * wr;
                    b[0] = a[0] - tr;
                    b[1] = a[1] - ti;
                    a[0] = a[0] + tr;
                    a[1] = a[1] + ti;
                }
            }
        }
    } else {
        for (int k = 0; k < n; ++k) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < n; ++j) {
                const int idx = (int)(((long long)j * k) % n);
                const double wr = lp->wr[idx], wi = lp->wi[idx];
                sr += x[2 * j] * wr - x[2 * j + 1] * wi;
                si += x[2 * j] * wi + x[2 * j + 1] * wr;
            }
            tmp[2 * k] = sr;
            tmp[2 * k + 1] = si;
        }
        memcpy(x, tmp, sizeof(double) * 2 * n);
    }
}

/* Transform every line along one axis of a (count x n x stride) array. */
static void axis_exec(double *data, int n, long outer, long stride, int sign) {
    if (n <= 1) return;
    line_plan lp;
    line_plan_init(&lp, n, sign);
    double *line = (double *)malloc(sizeof(double) * 2 * n);
    double *tmp = (double *)malloc(sizeof(double) * 2 * n);
    for (long o = 0; o < outer; ++o) {
        double *base = data + 2 * (o * (long)n * stride);
        for (long s = 0; s < stride; ++s) {
            for (int i = 0; i < n; ++i) {
                line[2 * i] = base[2 * (s + (long)i * stride)];
                line[2 * i + 1] = base[2 * (s + (long)i * stride) + 1];
            }
            line_exec(&lp, line, tmp);
            for (int i = 0; i < n; ++i) {
                base[2 * (s + (long)i * stride)] = line[2 * i];
                base[2 * (s + (long)i * stride) + 1] = line[2 * i + 1];
            }
        }
    }
    free(line);
    free(tmp);
    line_plan_free(&lp);
}

void pfc_shim_dft_3d(int n0, int n1, int n2, const fftw_complex *in, fftw_complex *out, int sign) {
    const long total = (long)n0 * n1 * n2;
    if ((const void *)in != (const void *)out) memmove(out, in, sizeof(fftw_complex) * total);
    double *d = (double *)out;
    axis_exec(d, n2, (long)n0 * n1, 1, sign);
    axis_exec(d, n1, n0, n2, sign);
    axis_exec(d, n0, 1, (long)n1 * n2, sign);
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags) {
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(struct fftw_plan_s));
    p->n0 = n0;
    p->n1 = n1;
    p->n2 = n2;
    p->sign = sign;
    p->in = in;
    p->out = out;
    return p;
}

void fftw_execute(const fftw_plan p) { pfc_shim_dft_3d(p->n0, p->n1, p->n2, p->in, p->out, p->sign); }

void fftw_destroy_plan(fftw_plan p) { free(p); }

void *fftw_malloc(size_t n) {
    void *ptr = NULL;
    if (posix_memalign(&ptr, 64, n ? n : 1) != 0) return NULL;
    return ptr;
}

void fftw_free(void *p) { free(p); }
