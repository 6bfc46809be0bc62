/*
 * CPU ORACLE for the SPME reciprocal-space path -- test infrastructure only.
 *
 * A plain-C FP64 restatement of the reference's algorithm (sfac.hpp and
 * sfac.cpp of frobnitzem/EwaldCorrel).  Only tests, the smoke check and the
 * CPU-baseline leg of the benchmark may load it, and only as a checker: the
 * product (libsfac.so) never calls into it.
 *
 * Each function names the reference lines it follows.  The FFT is the FP64
 * shim in fftw_shim/ (FFTW is not installed here); it follows FFTW's
 * conventions for rank-3 r2c/c2r transforms.
 *
 * Pinned against: test.log.ref (energy, gradient, virial of test.py's
 * fixture), the analytic cubic B-spline values printed by test.cpp, and the
 * reference's own sfac.cpp compiled against the same shim (oracle/_ref).
 *
 * Deliberate deviations from the reference (both also made by the GPU path):
 *  - Cell::wrap can return exactly 1.0 for tiny negative inputs
 *    (sfac.hpp:53-55); the reference then forms cell index K and an
 *    out-of-range or aliased key (sfac.cpp:100-106).  Here such a coordinate
 *    is treated as 0 (cell 0, fraction 0), i.e. its periodic image.
 *  - Neighbour-cell indices use a non-negative modulus, so K < order/2 is
 *    handled (the reference's `(i0+i)%K` can go negative there,
 *    sfac.cpp:144-154).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

typedef double (*orc_rad_fn)(double r2, double *dA, void *info);

typedef struct {
    double L[3][3];
    double iL[3][3];
    double iV;
} orc_cell;

typedef struct {
    int order;
    int K[3];
    int ldim;
    int state; /* -1 nothing, 0 structure factor, 1 potential grid */
    orc_cell cell;
    double *M;     /* order*order B-spline polynomial table */
    double *iB[3]; /* inverse B-spline moduli */
    double *Q;     /* padded in-place grid, 2*ldim*K1*K0 doubles */
    double *A;     /* K0*K1*ldim, followed by dA (6 per mode) */
    double *dA;
    double *spread; /* copy of the spread grid before the FFT (K0*K1*K2) */
    fftw_plan fwd, bwd;
} orc_sfac;

static int imod(int a, int b) { return ((a % b) + b) % b; }

/* Cell(L) -- sfac.hpp:37-52.  L6 = [ax, by, cz, bx, cx, cy]. */
static void cell_init(orc_cell *c, const double L6[6]) {
    memset(c, 0, sizeof(*c));
    c->L[0][0] = L6[0];
    c->L[1][1] = L6[1];
    c->L[2][2] = L6[2];
    c->L[1][0] = L6[3];
    c->L[2][0] = L6[4];
    c->L[2][1] = L6[5];
    c->iV = 1. / (L6[0] * L6[1] * L6[2]);
    c->iL[0][0] = 1. / L6[0];
    c->iL[1][1] = 1. / L6[1];
    c->iL[2][2] = 1. / L6[2];
    c->iL[1][0] = -L6[3] * L6[2] * c->iV;
    c->iL[2][0] = (L6[3] * L6[5] - L6[1] * L6[4]) * c->iV;
    c->iL[2][1] = -L6[0] * L6[5] * c->iV;
}

/* Cell::wrap -- sfac.hpp:53-55 */
static double wrap01(double x) { return x - floor(x); }

/* Cell::scale -- sfac.hpp:56-62: s = iL^T x, each component wrapped. */
static void cell_scale(const orc_cell *c, const double *x, double s[3]) {
    s[0] = wrap01(x[0] * c->iL[0][0] + x[1] * c->iL[1][0] + x[2] * c->iL[2][0]);
    s[1] = wrap01(x[1] * c->iL[1][1] + x[2] * c->iL[2][1]);
    s[2] = wrap01(x[2] * c->iL[2][2]);
}

/* BSpline::mk_bspl_coeffs -- sfac.hpp:81-109.
 * M[j*n+i] is the coefficient of t^(n-1-i) of M_n(t+j), t in [0,1):
 *   C(n-1,i)/(n-1)! * sum_{k<=j} (-1)^k C(n,k) (j-k)^i. */
static void bspline_table(int n, double *M) {
    for (int i = 0; i < n * n; i++) M[i] = 0.0;
    double den = 1.0;
    for (int k = 2; k < n; k++) den *= k;
    double f = 1.0;
    for (int k = 0; k < n; k++) {
        if (k > 0) {
            f *= k - n - 1;
            den *= k;
        }
        for (int j = k; j < n; j++) {
            double p = f / den;
            for (int i = 0; i < n; i++) {
                M[j * n + i] += p;
                p *= j - k;
            }
        }
    }
    double p = 1.0;
    for (int i = 1; i < n - 1; i++) {
        p *= (n - i) / (double)i;
        for (int j = 0; j < n; j++) M[j * n + i] *= p;
    }
}

/* BSpline::bspl_coef -- sfac.hpp:124-131 (Horner). */
static double bspl(const double *M, int n, double x, int j) {
    double b = M[n * j];
    for (int i = 1; i < n; i++) b = b * x + M[n * j + i];
    return b;
}

/* BSpline::dbspl_coef -- sfac.hpp:146-157 (value and derivative). */
static void dbspl(const double *M, int n, double x, int j, double *bp,
                  double *dbp) {
    double db = M[j * n];
    double b = M[j * n] * x + M[j * n + 1];
    for (int i = 2; i < n; i++) {
        db = db * x + b;
        b = b * x + M[j * n + i];
    }
    *bp = b;
    *dbp = db;
}

/* bspl_dft -- sfac.cpp:21-35: iB[i] = 1 / sum_{j=1}^{order-1}
 * cos(-2 pi i (j - order/2) / n) M_order(j). */
static void bspline_moduli(int n, int order, const double *M, double *out) {
    const int j0 = order / 2;
    const double *c = M + (order - 1); /* constant terms: M_order(j) */
    for (int i = 0; i < n; i++) {
        double om = -(2.0 * M_PI * i) / n;
        double x = 0.0;
        for (int j = 1; j < order; j++) x += cos(om * (j - j0)) * c[order * j];
        out[i] = 1.0 / x;
    }
}

/* SFac::SFac -- sfac.cpp:39-82.  Returns NULL (not an exception) on an odd
 * order, K < 1 or allocation failure. */
void *orc_ctor(const double L[6], const int K[3], int order) {
    if (order % 2 != 0 || order < 2) {
        printf("Bad order: %d (must be even)\n", order);
        return NULL;
    }
    if (K[0] < 1 || K[1] < 1 || K[2] < 1) {
        printf("Bad K: %d %d %d\n", K[0], K[1], K[2]);
        return NULL;
    }
    orc_sfac *h = (orc_sfac *)calloc(1, sizeof(orc_sfac));
    h->order = order;
    for (int d = 0; d < 3; d++) h->K[d] = K[d];
    h->ldim = K[2] / 2 + 1;
    h->state = -1;
    cell_init(&h->cell, L);
    h->M = (double *)malloc(sizeof(double) * order * order);
    bspline_table(order, h->M);
    for (int d = 0; d < 3; d++) {
        h->iB[d] = (double *)malloc(sizeof(double) * K[d]);
        bspline_moduli(K[d], order, h->M, h->iB[d]);
    }
    size_t n = 2 * (size_t)h->ldim * K[1] * K[0];
    h->Q = (double *)fftw_malloc(sizeof(double) * n);
    h->spread = (double *)malloc(sizeof(double) * (size_t)K[0] * K[1] * K[2]);
    if (!h->Q || !h->spread) return NULL;
    memset(h->Q, 0, sizeof(double) * n);
    h->fwd = fftw_plan_dft_r2c_3d(K[0], K[1], K[2], h->Q, (fftw_complex *)h->Q,
                                  FFTW_PATIENT);
    h->bwd = fftw_plan_dft_c2r_3d(K[0], K[1], K[2], (fftw_complex *)h->Q, h->Q,
                                  FFTW_PATIENT);
    return h;
}

/* SFac::~SFac -- sfac.cpp:170-176 */
void orc_dtor(void *vh) {
    orc_sfac *h = (orc_sfac *)vh;
    if (!h) return;
    fftw_destroy_plan(h->fwd);
    fftw_destroy_plan(h->bwd);
    fftw_free(h->Q);
    free(h->A);
    free(h->M);
    free(h->spread);
    for (int d = 0; d < 3; d++) free(h->iB[d]);
    free(h);
}

/* Cell index and in-cell fraction of one point -- sfac.cpp:97-106.
 * Returns the key cid = (n0*K1 + n1)*K2 + n2. */
static int cell_of(const orc_sfac *h, const double *x, double u[3]) {
    double s[3];
    int nn[3];
    cell_scale(&h->cell, x, s);
    for (int i = 0; i < 3; i++) {
        u[i] = s[i] * h->K[i];
        nn[i] = (int)u[i];
        u[i] -= nn[i];
        if (nn[i] >= h->K[i]) { /* wrap() returned 1.0: periodic image */
            nn[i] = 0;
            u[i] = 0.0;
        }
    }
    return (nn[0] * h->K[1] + nn[1]) * h->K[2] + nn[2];
}

typedef struct {
    int key;
    int idx;
} keyidx;

static int cmp_keyidx(const void *a, const void *b) {
    const keyidx *p = (const keyidx *)a, *q = (const keyidx *)b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return p->idx < q->idx ? -1 : (p->idx > q->idx);
}

/* SFac::sort -- sfac.cpp:92-111.  std::multimap keeps equal keys in
 * insertion order, so the result is the stable sort of the atoms by cid.
 * keys_out[r] / perm_out[r] give the key and original index of rank r. */
int orc_sort(void *vh, int n, const double *x, int *keys_out, int *perm_out,
             double *frac_out) {
    orc_sfac *h = (orc_sfac *)vh;
    keyidx *ki = (keyidx *)malloc(sizeof(keyidx) * (n > 0 ? n : 1));
    double *u = (double *)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
    for (int a = 0; a < n; a++) {
        ki[a].key = cell_of(h, x + 3 * a, u + 3 * a);
        ki[a].idx = a;
    }
    qsort(ki, (size_t)n, sizeof(keyidx), cmp_keyidx);
    for (int r = 0; r < n; r++) {
        if (keys_out) keys_out[r] = ki[r].key;
        if (perm_out) perm_out[r] = ki[r].idx;
        if (frac_out)
            for (int d = 0; d < 3; d++) frac_out[3 * r + d] = u[3 * ki[r].idx + d];
    }
    free(ki);
    free(u);
    return 0;
}

/* SFac::operator() + accum_spline -- sfac.cpp:113-168.
 * Owner-computes spreading: every grid point sums over the atoms of the
 * order^3 neighbouring cells (in sorted order), so no two writers share a
 * point.  Then the forward r2c FFT (sfac.cpp:125) and division by the
 * B-spline moduli (sfac.cpp:128-138). */
void orc_sfac_run(void *vh, int n, const double *w, const double *x) {
    orc_sfac *h = (orc_sfac *)vh;
    const int K0 = h->K[0], K1 = h->K[1], K2 = h->K[2], p = h->order;
    const int ldim = h->ldim;
    const long ncell = (long)K0 * K1 * K2;
    memset(h->Q, 0, sizeof(double) * (size_t)K0 * K1 * ldim * 2);

    int *keys = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int *perm = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    double *frac = (double *)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
    orc_sort(h, n, x, keys, perm, frac);
    int *start = (int *)malloc(sizeof(int) * (ncell + 1));
    {
        long r = 0;
        for (long c = 0; c <= ncell; c++) {
            while (r < n && keys[r] < c) r++;
            start[c] = (int)r;
        }
    }

#pragma omp parallel for collapse(3) schedule(static)
    for (int i1 = 0; i1 < K0; i1++)
        for (int j1 = 0; j1 < K1; j1++)
            for (int k1 = 0; k1 < K2; k1++) {
                double ans = 0.0;
                for (int i = 0; i < p; i++) {
                    int xid = imod(i1 - p / 2 + i, K0) * K1;
                    for (int j = 0; j < p; j++) {
                        int yid = (xid + imod(j1 - p / 2 + j, K1)) * K2;
                        for (int k = 0; k < p; k++) {
                            int cid = yid + imod(k1 - p / 2 + k, K2);
                            for (int r = start[cid]; r < start[cid + 1]; r++) {
                                const double *uu = frac + 3 * r;
                                ans += bspl(h->M, p, uu[0], i) *
                                       bspl(h->M, p, uu[1], j) *
                                       bspl(h->M, p, uu[2], k) * w[perm[r]];
                            }
                        }
                    }
                }
                long NN = ((long)i1 * K1 + j1) * ldim * 2 + k1;
                h->Q[NN] += ans;
                h->spread[((long)i1 * K1 + j1) * K2 + k1] = ans;
            }
    free(keys);
    free(perm);
    free(frac);
    free(start);

    fftw_execute(h->fwd);
    h->state = 0;

    const long nm = (long)K0 * K1 * ldim;
    for (long cid = 0; cid < nm; cid++) {
        double t = h->iB[0][cid / ((long)ldim * K1)] *
                   h->iB[1][(cid / ldim) % K1] * h->iB[2][cid % ldim];
        h->Q[2 * cid] *= t;
        h->Q[2 * cid + 1] *= t;
    }
}

/* get_S -- sfac.cpp:194-197 */
double *orc_get_S(void *vh) { return ((orc_sfac *)vh)->Q; }

/* The real grid produced by the last spread, before the FFT. */
double *orc_get_spread(void *vh) { return ((orc_sfac *)vh)->spread; }

/* set_L -- sfac.cpp:199-202: replaces the cell only; A is not recomputed. */
void orc_set_L(void *vh, const double L[6]) {
    cell_init(&((orc_sfac *)vh)->cell, L);
}

/* set_A -- sfac.cpp:213-292.  Visits every m = iL n with |m| < max_m
 * (aliases beyond Nyquist included), folds n onto the stored half space and
 * accumulates A += f(m^2)/2 and dA += f'(m^2) m_a m_b. */
int orc_set_A(void *vh, orc_rad_fn f, double max_m, void *info) {
    orc_sfac *h = (orc_sfac *)vh;
    const orc_cell *c = &h->cell;
    const int K0 = h->K[0], K1 = h->K[1], K2 = h->K[2], ldim = h->ldim;
    const double R2 = max_m * max_m;
    const int i0 = (int)(max_m / c->iL[0][0]);
    const long nm = (long)K0 * K1 * ldim;
    if (!h->A) {
        h->A = (double *)malloc(sizeof(double) * nm * 7);
        if (!h->A) return 2;
        h->dA = h->A + nm;
    }
    memset(h->A, 0, sizeof(double) * nm * 7);

    for (int i = -i0; i <= i0; i++) {
        const double mx = i * c->iL[0][0];
        const double m20 = mx * mx;
        const double dy = sqrt(R2 - m20);
        const double my0 = i * c->iL[1][0];
        const int j0 = (int)ceil((-dy - my0) / c->iL[1][1]);
        const int j1 = (int)floor((dy - my0) / c->iL[1][1]);
        const long rx = (long)imod(i, K0) * K1; /* row offset of +n */
        for (int j = j0; j <= j1; j++) {
            const double my = my0 + j * c->iL[1][1];
            const double m21 = m20 + my * my;
            const double dz = sqrt(R2 - m21);
            const double mz0 = i * c->iL[2][0] + j * c->iL[2][1];
            const int k0 = (int)ceil((-dz - mz0) / c->iL[2][2]);
            const int k1 = (int)floor((dz - mz0) / c->iL[2][2]);
            const long ry = (imod(j, K1) + rx) * ldim;
            for (int k = k0; k <= k1; k++) {
                const double mz = mz0 + k * c->iL[2][2];
                const double m2 = m21 + mz * mz;
                long idx;
                int kz = imod(k, K2);
                if (kz >= ldim) {
                    /* stored as the conjugate partner -n */
                    long nx = (long)imod(-i, K0), ny = imod(-j, K1);
                    idx = (nx * K1 + ny) * ldim + (K2 - kz);
                } else {
                    idx = ry + kz;
                }
                double s;
                h->A[idx] += 0.5 * f(m2, &s, info);
                double *d = h->dA + 6 * idx;
                d[0] += s * mx * mx;
                d[1] += s * my * my;
                d[2] += s * mz * mz;
                d[3] += s * my * mx;
                d[4] += s * mz * mx;
                d[5] += s * mz * my;
            }
        }
    }
    return 0;
}

/* A and dA as computed by the last set_A (7 * K0*K1*ldim doubles). */
double *orc_get_A(void *vh) { return ((orc_sfac *)vh)->A; }

/* en -- sfac.cpp:304-325 */
double orc_en(void *vh) {
    orc_sfac *h = (orc_sfac *)vh;
    if (h->state != 0) {
        printf("Error: You must call sfac before this routine.\n");
        return 0.0;
    }
    if (!h->A) {
        printf("Error: No convolution kernel has been set.\n");
        return 0.0;
    }
    const long nm = (long)h->K[0] * h->K[1] * h->ldim;
    double e = 0.0;
    for (long i = 0; i < nm; i++)
        e += h->A[i] * (h->Q[2 * i] * h->Q[2 * i] + h->Q[2 * i + 1] * h->Q[2 * i + 1]);
    return e * h->cell.iV;
}

/* de1 -- sfac.cpp:339-396: energy, virial, FQ *= A iB (x2 on the kz=0 and
 * even-K2 Nyquist planes), inverse c2r FFT into the potential grid. */
double orc_de1(void *vh, double vir[6]) {
    orc_sfac *h = (orc_sfac *)vh;
    if (h->state != 0) {
        printf("Error: You must call sfac before this routine.\n");
        return 0.0;
    }
    if (!h->A) {
        printf("Error: No convolution kernel has been set.\n");
        return 0.0;
    }
    const int K1 = h->K[1], ldim = h->ldim;
    const long nm = (long)h->K[0] * K1 * ldim;
    const int even = (h->K[2] + 1) % 2;
    double e = 0, v00 = 0, v11 = 0, v22 = 0, v10 = 0, v20 = 0, v21 = 0;
    for (long i = 0; i < nm; i++) {
        double *q = h->Q + 2 * i;
        double s = q[0] * q[0] + q[1] * q[1];
        const double *d = h->dA + 6 * i;
        double t = h->A[i] * h->iB[0][i / ((long)ldim * K1)] *
                   h->iB[1][(i / ldim) % K1] * h->iB[2][i % ldim];
        if (i % ldim == 0 || (even && (i + 1) % ldim == 0)) t *= 2.0;
        q[0] *= t;
        q[1] *= t;
        e += s * h->A[i];
        v00 += s * d[0];
        v11 += s * d[1];
        v22 += s * d[2];
        v10 += s * d[3];
        v20 += s * d[4];
        v21 += s * d[5];
    }
    const double fac = h->cell.iV * h->cell.iV;
    vir[0] = (v00 + e) * fac;
    vir[1] = (v11 + e) * fac;
    vir[2] = (v22 + e) * fac;
    vir[3] = v10 * fac;
    vir[4] = v20 * fac;
    vir[5] = v21 * fac;
    fftw_execute(h->bwd);
    h->state = 1;
    return e * h->cell.iV;
}

/* Stencil origin of a gather point -- sfac.cpp:428-439. */
static void gather_origin(const orc_sfac *h, const double *x, double u[3],
                          int k1[3], int k0[3]) {
    double s[3];
    cell_scale(&h->cell, x, s);
    for (int d = 0; d < 3; d++) {
        u[d] = s[d] * h->K[d];
        k1[d] = (int)ceil(u[d]);
        k0[d] = imod(k1[d] - h->order / 2, h->K[d]);
    }
}

/* de2 -- sfac.cpp:409-483: dE/dx of each point (gradient; force = -dx). */
void orc_de2(void *vh, int n, const double *w, const double *x, double *dx0) {
    orc_sfac *h = (orc_sfac *)vh;
    if (h->state != 1) {
        printf("Error: You must call de1 before this routine.\n");
        return;
    }
    const int p = h->order, K0 = h->K[0], K1 = h->K[1], K2 = h->K[2];
    const long pitch = 2L * h->ldim;
    for (int a = 0; a < n; a++) {
        double u[3];
        int k1[3], k0[3];
        double g[3] = {0., 0., 0.};
        gather_origin(h, x + 3 * a, u, k1, k0);
        for (int i = 0; i < p; i++) {
            long ni = (long)((k0[0] + i) % K0) * K1;
            double mpx, dmpx;
            dbspl(h->M, p, k1[0] - u[0], i, &mpx, &dmpx);
            for (int j = 0; j < p; j++) {
                double mpy, dmpy;
                dbspl(h->M, p, k1[1] - u[1], j, &mpy, &dmpy);
                double fj0 = dmpx * mpy;
                double fj1 = mpx * dmpy;
                double fj2 = mpx * mpy;
                long nj = (ni + (k0[1] + j) % K1) * pitch;
                for (int k = 0; k < p; k++) {
                    double mpz, dmpz;
                    dbspl(h->M, p, k1[2] - u[2], k, &mpz, &dmpz);
                    long nk = nj + (k0[2] + k) % K2;
                    double fk = mpz * h->Q[nk];
                    g[0] += fj0 * fk;
                    g[1] += fj1 * fk;
                    g[2] += fj2 * dmpz * h->Q[nk];
                }
            }
        }
        const orc_cell *c = &h->cell;
        g[0] *= (-w[a] * c->iV) * K0;
        g[1] *= (-w[a] * c->iV) * K1;
        g[2] *= (-w[a] * c->iV) * K2;
        dx0[3 * a + 0] = c->iL[0][0] * g[0];
        dx0[3 * a + 1] = c->iL[1][0] * g[0] + c->iL[1][1] * g[1];
        dx0[3 * a + 2] = c->iL[2][0] * g[0] + c->iL[2][1] * g[1] + c->iL[2][2] * g[2];
    }
}

/* potl -- sfac.cpp:497-545: potential phi_a = dE/dw_a. */
void orc_potl(void *vh, int n, const double *x, double *phi) {
    orc_sfac *h = (orc_sfac *)vh;
    if (h->state != 1) {
        printf("Error: You must call de1 before this routine.\n");
        return;
    }
    const int p = h->order, K0 = h->K[0], K1 = h->K[1], K2 = h->K[2];
    const long pitch = 2L * h->ldim;
    for (int a = 0; a < n; a++) {
        double u[3];
        int k1[3], k0[3];
        double pot = 0.0;
        gather_origin(h, x + 3 * a, u, k1, k0);
        for (int i = 0; i < p; i++) {
            long ni = (long)((k0[0] + i) % K0) * K1;
            double s1 = 0.0;
            for (int j = 0; j < p; j++) {
                double mpy = bspl(h->M, p, k1[1] - u[1], j);
                long nj = (ni + (k0[1] + j) % K1) * pitch;
                for (int k = 0; k < p; k++) {
                    double mpz = bspl(h->M, p, k1[2] - u[2], k);
                    long nk = nj + (k0[2] + k) % K2;
                    s1 += mpy * mpz * h->Q[nk];
                }
            }
            double mpx = bspl(h->M, p, k1[0] - u[0], i);
            pot += mpx * s1;
        }
        phi[a] = pot * h->cell.iV;
    }
}

/* Ewald influence function, the C twin of ewald.py:124-132:
 * f(r2) = exp(-pi^2 r2 / eta^2) / (pi r2), f' = (-pi^2/eta^2 - 1/r2) f.
 * info points to eta (double). */
double orc_ewald_rad(double r2, double *dA, void *info) {
    const double eta = *(const double *)info;
    const double fac = -pow(M_PI / eta, 2.0);
    if (r2 < 1e-10) {
        *dA = 0.0;
        return 0.0;
    }
    double f = exp(r2 * fac) / (r2 * M_PI);
    *dA = (fac - 1. / r2) * f;
    return f;
}

/* Small helpers for the oracle's self-tests. */
double orc_bspl_value(int order, double x, int j) {
    double M[64];
    if (order < 2 || order > 8) return NAN;
    bspline_table(order, M);
    return bspl(M, order, x, j);
}

void orc_bspline_table(int order, double *M) { bspline_table(order, M); }

void orc_bspline_moduli(int n, int order, double *out) {
    double M[64];
    bspline_table(order, M);
    bspline_moduli(n, order, M, out);
}

void orc_cell_consts(const double L[6], double *iL9, double *iV) {
    orc_cell c;
    cell_init(&c, L);
    memcpy(iL9, c.iL, sizeof(double) * 9);
    *iV = c.iV;
}
