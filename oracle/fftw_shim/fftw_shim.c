/*
 * FP64 FFT behind the FFTW-API subset declared in fftw3.h.
 * Test infrastructure only: it lets the reference's sfac.cpp and the oracle
 * restatement (spme_oracle.c) run without FFTW installed.
 *
 * Algorithm: recursive mixed-radix decimation-in-time Cooley-Tukey
 * (radix 4, 2, 3, 5 butterflies written out; any other prime factor uses a
 * direct O(p^2) DFT butterfly), twiddles from one FP64 table per length.
 * Multi-dimensional r2c/c2r transforms are done axis by axis in FFTW's order
 * (row r2c on the last axis, then complex transforms on axes 1 and 0; the
 * inverse runs in reverse) and real rows are transformed two at a time by
 * packing them as the real and imaginary parts of one complex row.
 * Single-threaded, like the reference's un-threaded `-lfftw3` link
 * (Makefile:4).
 */
#include "fftw3.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double re, im;
} cplx;

typedef struct {
    int n;
    int nfac;
    int fac[64];
    cplx *tw; /* tw[j] = exp(-2 pi i j / n) */
    cplx *buf; /* scratch: 2n */
} fft1;

static void fft1_init(fft1 *P, int n) {
    P->n = n;
    P->nfac = 0;
    int m = n;
    /* Radix order: 4s first, then 2, 3, 5, then the remaining primes. */
    while (m % 4 == 0) { P->fac[P->nfac++] = 4; m /= 4; }
    while (m % 2 == 0) { P->fac[P->nfac++] = 2; m /= 2; }
    for (int p = 3; m > 1; p += 2) {
        while (m % p == 0) { P->fac[P->nfac++] = p; m /= p; }
        if ((long)p * p > m && m > 1) { P->fac[P->nfac++] = m; m = 1; }
    }
    if (P->nfac == 0) P->fac[P->nfac++] = 1;
    P->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    P->buf = (cplx *)malloc(sizeof(cplx) * (size_t)n * 2);
    for (int j = 0; j < n; j++) {
        /* Angle reduced to [-pi, pi] to keep sin/cos arguments small. */
        long jj = (2L * j <= n) ? j : j - (long)n;
        double a = -2.0 * M_PI * (double)jj / (double)n;
        P->tw[j].re = cos(a);
        P->tw[j].im = sin(a);
    }
}

static void fft1_free(fft1 *P) {
    free(P->tw);
    free(P->buf);
}

static inline cplx cmul(cplx a, cplx b) {
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}

/* w_N^(k) with sign: sign<0 -> table value, sign>0 -> conjugate. */
static inline cplx twid(const fft1 *P, long k, int sign) {
    cplx w = P->tw[k % P->n];
    if (sign > 0) w.im = -w.im;
    return w;
}

/* out[k] = sum_j in[j*is] w^(sign j k), length n = N / tws (N = P->n). */
static void fft_rec(cplx *out, const cplx *in, long is, int n,
                    const int *fac, const fft1 *P, long tws, int sign) {
    const int p = fac[0];
    const int m = n / p;
    if (m == 1) {
        for (int q = 0; q < p; q++) out[q] = in[(long)q * is];
    } else {
        for (int r = 0; r < p; r++)
            fft_rec(out + (long)r * m, in + (long)r * is, is * p, m, fac + 1,
                    P, tws * p, sign);
    }
    if (p == 1) return;
    const double s = (double)sign;
    for (int k = 0; k < m; k++) {
        if (p == 2) {
            cplx a = out[k];
            cplx b = cmul(out[k + m], twid(P, (long)k * tws, sign));
            out[k].re = a.re + b.re; out[k].im = a.im + b.im;
            out[k + m].re = a.re - b.re; out[k + m].im = a.im - b.im;
        } else if (p == 4) {
            cplx a0 = out[k];
            cplx a1 = cmul(out[k + m], twid(P, (long)k * tws, sign));
            cplx a2 = cmul(out[k + 2 * m], twid(P, 2L * k * tws, sign));
            cplx a3 = cmul(out[k + 3 * m], twid(P, 3L * k * tws, sign));
            cplx t0 = {a0.re + a2.re, a0.im + a2.im};
            cplx t1 = {a0.re - a2.re, a0.im - a2.im};
            cplx t2 = {a1.re + a3.re, a1.im + a3.im};
            cplx t3 = {a1.re - a3.re, a1.im - a3.im};
            /* multiply t3 by sign*i: forward (-i), backward (+i) */
            cplx t3r = {-s * t3.im, s * t3.re};
            out[k].re = t0.re + t2.re; out[k].im = t0.im + t2.im;
            out[k + 2 * m].re = t0.re - t2.re; out[k + 2 * m].im = t0.im - t2.im;
            out[k + m].re = t1.re + t3r.re; out[k + m].im = t1.im + t3r.im;
            out[k + 3 * m].re = t1.re - t3r.re; out[k + 3 * m].im = t1.im - t3r.im;
        } else if (p == 3) {
            const double c = -0.5, sn = s * 0.86602540378443864676;
            cplx a0 = out[k];
            cplx a1 = cmul(out[k + m], twid(P, (long)k * tws, sign));
            cplx a2 = cmul(out[k + 2 * m], twid(P, 2L * k * tws, sign));
            cplx t = {a1.re + a2.re, a1.im + a2.im};
            cplx d = {a1.re - a2.re, a1.im - a2.im};
            cplx mid = {a0.re + c * t.re, a0.im + c * t.im};
            /* sn * i * d */
            cplx rot = {-sn * d.im, sn * d.re};
            out[k].re = a0.re + t.re; out[k].im = a0.im + t.im;
            out[k + m].re = mid.re + rot.re; out[k + m].im = mid.im + rot.im;
            out[k + 2 * m].re = mid.re - rot.re; out[k + 2 * m].im = mid.im - rot.im;
        } else {
            /* Generic radix (5 and other primes): direct p-point DFT. */
            cplx y[64];
            cplx *yy = (p <= 64) ? y : (cplx *)malloc(sizeof(cplx) * (size_t)p);
            for (int r = 0; r < p; r++)
                yy[r] = (r == 0) ? out[k]
                                 : cmul(out[k + (long)r * m],
                                        twid(P, (long)r * k * tws, sign));
            const long wp = (long)m * tws; /* w_p = w_N^(m tws) */
            for (int q = 0; q < p; q++) {
                cplx acc = yy[0];
                for (int r = 1; r < p; r++) {
                    cplx w = twid(P, ((long)r * q % p) * wp, sign);
                    cplx t = cmul(yy[r], w);
                    acc.re += t.re;
                    acc.im += t.im;
                }
                out[k + (long)q * m] = acc;
            }
            if (yy != y) free(yy);
        }
    }
}

static void fft1_exec(const fft1 *P, const cplx *in, long is, cplx *out,
                      int sign) {
    fft_rec(out, in, is, P->n, P->fac, P, 1, sign);
}

void shim_fft1d(int n, const double *in, double *out, int sign) {
    fft1 P;
    fft1_init(&P, n);
    fft1_exec(&P, (const cplx *)in, 1, (cplx *)out, sign);
    fft1_free(&P);
}

/* ------------------------------------------------------------------ */

struct shim_fftw_plan_s {
    int kind; /* 0: r2c, 1: c2r */
    int n0, n1, n2, nh;
    long rpitch; /* real row pitch in doubles */
    double *real;
    cplx *cpx;
    fft1 p0, p1, p2;
};

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}

void fftw_free(void *p) { free(p); }

static fftw_plan mkplan(int kind, int n0, int n1, int n2, double *real,
                        cplx *cpx) {
    fftw_plan P = (fftw_plan)calloc(1, sizeof(*P));
    P->kind = kind;
    P->n0 = n0;
    P->n1 = n1;
    P->n2 = n2;
    P->nh = n2 / 2 + 1;
    P->real = real;
    P->cpx = cpx;
    /* In-place transforms use FFTW's padded real rows. */
    P->rpitch = ((void *)real == (void *)cpx) ? 2L * P->nh : n2;
    fft1_init(&P->p0, n0);
    fft1_init(&P->p1, n1);
    fft1_init(&P->p2, n2);
    return P;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags) {
    (void)flags;
    return mkplan(0, n0, n1, n2, in, (cplx *)out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags) {
    (void)flags;
    return mkplan(1, n0, n1, n2, out, (cplx *)in);
}

void fftw_destroy_plan(fftw_plan P) {
    if (!P) return;
    fft1_free(&P->p0);
    fft1_free(&P->p1);
    fft1_free(&P->p2);
    free(P);
}

void fftw_cleanup(void) {}

/* Complex transform of every line along axis 0 (len n0, stride n1*nh) or
 * axis 1 (len n1, stride nh) of the half-complex array. */
static void axis_c2c(fftw_plan P, int axis, int sign) {
    const int n0 = P->n0, n1 = P->n1, nh = P->nh;
    const int len = axis == 0 ? n0 : n1;
    const long stride = axis == 0 ? (long)n1 * nh : nh;
    const fft1 *F = axis == 0 ? &P->p0 : &P->p1;
    cplx *line = (cplx *)malloc(sizeof(cplx) * (size_t)len * 2);
    cplx *res = line + len;
    const long nlines = axis == 0 ? (long)n1 * nh : (long)n0 * nh;
    for (long l = 0; l < nlines; l++) {
        long base;
        if (axis == 0) {
            base = l; /* (y, kz) */
        } else {
            long x = l / nh, kz = l % nh;
            base = x * (long)n1 * nh + kz;
        }
        for (int j = 0; j < len; j++) line[j] = P->cpx[base + j * stride];
        fft1_exec(F, line, 1, res, sign);
        for (int j = 0; j < len; j++) P->cpx[base + j * stride] = res[j];
    }
    free(line);
}

static void rows_r2c(fftw_plan P) {
    const int n2 = P->n2, nh = P->nh;
    const long nrows = (long)P->n0 * P->n1;
    cplx *z = (cplx *)malloc(sizeof(cplx) * (size_t)n2 * 2);
    cplx *Z = z + n2;
    for (long r = 0; r < nrows; r += 2) {
        const int two = (r + 1 < nrows);
        const double *a = P->real + r * P->rpitch;
        const double *b = two ? P->real + (r + 1) * P->rpitch : NULL;
        for (int k = 0; k < n2; k++) {
            z[k].re = a[k];
            z[k].im = two ? b[k] : 0.0;
        }
        fft1_exec(&P->p2, z, 1, Z, -1);
        cplx *oa = P->cpx + r * nh;
        cplx *ob = two ? P->cpx + (r + 1) * nh : NULL;
        for (int k = 0; k < nh; k++) {
            cplx u = Z[k];
            cplx v = Z[(n2 - k) % n2];
            /* A = (u + conj v)/2 ; B = (u - conj v)/(2i) */
            cplx A = {0.5 * (u.re + v.re), 0.5 * (u.im - v.im)};
            cplx B = {0.5 * (u.im + v.im), -0.5 * (u.re - v.re)};
            oa[k] = A;
            if (two) ob[k] = B;
        }
    }
    free(z);
}

static void rows_c2r(fftw_plan P) {
    const int n2 = P->n2, nh = P->nh;
    const long nrows = (long)P->n0 * P->n1;
    cplx *z = (cplx *)malloc(sizeof(cplx) * (size_t)n2 * 2);
    cplx *Z = z + n2;
    for (long r = 0; r < nrows; r += 2) {
        const int two = (r + 1 < nrows);
        const cplx *ia = P->cpx + r * nh;
        const cplx *ib = two ? P->cpx + (r + 1) * nh : NULL;
        for (int k = 0; k < n2; k++) {
            cplx A, B = {0.0, 0.0};
            if (k < nh) {
                A = ia[k];
                if (two) B = ib[k];
            } else {
                A = ia[n2 - k];
                A.im = -A.im;
                if (two) {
                    B = ib[n2 - k];
                    B.im = -B.im;
                }
            }
            /* Self-conjugate bins contribute their real part only. */
            if (k == 0 || 2 * k == n2) {
                A.im = 0.0;
                B.im = 0.0;
            }
            /* z = A + i B */
            z[k].re = A.re - B.im;
            z[k].im = A.im + B.re;
        }
        fft1_exec(&P->p2, z, 1, Z, +1);
        double *oa = P->real + r * P->rpitch;
        double *ob = two ? P->real + (r + 1) * P->rpitch : NULL;
        for (int k = 0; k < n2; k++) {
            oa[k] = Z[k].re;
            if (two) ob[k] = Z[k].im;
        }
    }
    free(z);
}

void fftw_execute(const fftw_plan P) {
    if (P->kind == 0) {
        rows_r2c(P);
        axis_c2c(P, 1, -1);
        axis_c2c(P, 0, -1);
    } else {
        axis_c2c(P, 0, +1);
        axis_c2c(P, 1, +1);
        rows_c2r(P);
    }
}
