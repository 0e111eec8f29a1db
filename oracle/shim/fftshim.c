/*
 * Real 1-D DFTs behind the FFTW plan API (test infrastructure, see fftw3.h).
 *
 * Even n: the real sequence x is packed as z[m] = x[2m] + i x[2m+1] and one
 * complex radix-2 FFT of length n/2 is run (textbook decimation in time with
 * a bit-reversal permutation); the n/2+1 output bins follow from
 *     X[k] = E[k] + W^k O[k],  E = (Z[k] + conj Z[n/2-k]) / 2,
 *                              O = (Z[k] - conj Z[n/2-k]) / (2i),
 * with W = exp(-2 pi i / n).  The inverse runs the same identities backwards.
 * Lengths that are not powers of two fall back to a direct O(n^2) sum.
 * Twiddles are computed in long double and rounded once.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct oracle_fftw_plan {
    int n;          /* real length */
    int dir;        /* -1: r2c, +1: c2r */
    double *rbuf;   /* real side */
    fftw_complex *cbuf; /* complex side (n/2+1 bins) */
    int m;          /* complex FFT length n/2 (even n) */
    int pow2;       /* m is a power of two */
    double *wm;     /* exp(-2 pi i k / m), k < m: interleaved re, im */
    double *wn;     /* exp(-2 pi i k / n), k <= n/2 */
    int *rev;       /* bit reversal of length m */
    double *work;   /* 2*m doubles */
    double *zbuf;   /* 2*m doubles: the packed sequence */
};

static const long double TWO_PI_L = 6.283185307179586476925286766559005768L;

void *fftw_malloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}

void fftw_free(void *p) { free(p); }

static fftw_plan make_plan(int n, int dir, double *r, fftw_complex *c)
{
    fftw_plan p = (fftw_plan)calloc(1, sizeof *p);
    p->n = n;
    p->dir = dir;
    p->rbuf = r;
    p->cbuf = c;
    if (n % 2 == 0) {
        int m = n / 2;
        p->m = m;
        p->pow2 = (m & (m - 1)) == 0;
        p->wm = (double *)malloc(sizeof(double) * 2 * (size_t)m);
        for (int k = 0; k < m; k++) {
            long double a = -TWO_PI_L * (long double)k / (long double)m;
            p->wm[2 * k] = (double)cosl(a);
            p->wm[2 * k + 1] = (double)sinl(a);
        }
        p->wn = (double *)malloc(sizeof(double) * 2 * (size_t)(m + 1));
        for (int k = 0; k <= m; k++) {
            long double a = -TWO_PI_L * (long double)k / (long double)n;
            p->wn[2 * k] = (double)cosl(a);
            p->wn[2 * k + 1] = (double)sinl(a);
        }
        p->work = (double *)malloc(sizeof(double) * 2 * (size_t)m);
        p->zbuf = (double *)malloc(sizeof(double) * 2 * (size_t)m);
        if (p->pow2) {
            int bits = 0;
            while ((1 << bits) < m) bits++;
            p->rev = (int *)malloc(sizeof(int) * (size_t)m);
            for (int k = 0; k < m; k++) {
                int r = 0;
                for (int b = 0; b < bits; b++) r |= ((k >> b) & 1) << (bits - 1 - b);
                p->rev[k] = r;
            }
        }
    }
    return p;
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags)
{
    (void)flags;
    return make_plan(n, -1, in, out);
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags)
{
    (void)flags;
    return make_plan(n, +1, out, in);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    free(p->wm);
    free(p->wn);
    free(p->rev);
    free(p->work);
    free(p->zbuf);
    free(p);
}

/* complex DFT of length m on interleaved data z, sign -1 (forward) or +1 */
static void cfft(const struct oracle_fftw_plan *p, double *z, int sign)
{
    int m = p->m;
    if (p->pow2) {
        double *t = p->work;
        for (int k = 0; k < m; k++) {
            t[2 * p->rev[k]] = z[2 * k];
            t[2 * p->rev[k] + 1] = z[2 * k + 1];
        }
        for (int len = 2; len <= m; len <<= 1) {
            int half = len / 2, step = m / len;
            for (int s = 0; s < m; s += len) {
                for (int k = 0; k < half; k++) {
                    double wr = p->wm[2 * k * step];
                    double wi = -sign * p->wm[2 * k * step + 1]; /* wm holds exp(-i...) */
                    double *a = t + 2 * (s + k), *b = t + 2 * (s + k + half);
                    double br = b[0] * wr - b[1] * wi;
                    double bi = b[0] * wi + b[1] * wr;
                    b[0] = a[0] - br;
                    b[1] = a[1] - bi;
                    a[0] = a[0] + br;
                    a[1] = a[1] + bi;
                }
            }
        }
        memcpy(z, t, sizeof(double) * 2 * (size_t)m);
    } else {
        double *t = p->work;
        for (int k = 0; k < m; k++) {
            double sr = 0, si = 0;
            for (int j = 0; j < m; j++) {
                long idx = ((long)j * k) % m;
                double wr = p->wm[2 * idx], wi = -sign * p->wm[2 * idx + 1];
                sr += z[2 * j] * wr - z[2 * j + 1] * wi;
                si += z[2 * j] * wi + z[2 * j + 1] * wr;
            }
            t[2 * k] = sr;
            t[2 * k + 1] = si;
        }
        memcpy(z, t, sizeof(double) * 2 * (size_t)m);
    }
}

static void direct_r2c(int n, const double *x, fftw_complex *X)
{
    for (int k = 0; k <= n / 2; k++) {
        long double sr = 0, si = 0;
        for (int j = 0; j < n; j++) {
            long double a = -TWO_PI_L * (long double)(((long)j * k) % n) / n;
            sr += x[j] * cosl(a);
            si += x[j] * sinl(a);
        }
        X[k][0] = (double)sr;
        X[k][1] = (double)si;
    }
    X[0][1] = 0.0;
}

static void direct_c2r(int n, const fftw_complex *X, double *x)
{
    for (int j = 0; j < n; j++) {
        long double s = X[0][0];
        for (int k = 1; k <= (n - 1) / 2; k++) {
            long double a = TWO_PI_L * (long double)(((long)j * k) % n) / n;
            s += 2.0L * (X[k][0] * cosl(a) - X[k][1] * sinl(a));
        }
        x[j] = (double)s;
    }
}

void fftw_execute(const fftw_plan p)
{
    int n = p->n;
    if (n % 2 != 0) {
        if (p->dir < 0) direct_r2c(n, p->rbuf, p->cbuf);
        else direct_c2r(n, p->cbuf, p->rbuf);
        return;
    }
    int m = p->m;
    double *z = p->zbuf;
    if (p->dir < 0) {
        const double *x = p->rbuf;
        for (int k = 0; k < m; k++) {
            z[2 * k] = x[2 * k];
            z[2 * k + 1] = x[2 * k + 1];
        }
        cfft(p, z, -1);
        fftw_complex *X = p->cbuf;
        for (int k = 0; k <= m; k++) {
            int k1 = k % m, k2 = (m - k) % m;
            double zr = z[2 * k1], zi = z[2 * k1 + 1];
            double cr = z[2 * k2], ci = -z[2 * k2 + 1]; /* conj Z[m-k] */
            double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
            /* O = (Z - conj Z') / (2i) */
            double dr = zr - cr, di = zi - ci;
            double orr = 0.5 * di, oi = -0.5 * dr;
            double wr = p->wn[2 * k], wi = p->wn[2 * k + 1];
            X[k][0] = er + (wr * orr - wi * oi);
            X[k][1] = ei + (wr * oi + wi * orr);
        }
        X[0][1] = 0.0;
        X[m][1] = 0.0;
    } else {
        const fftw_complex *X = p->cbuf;
        for (int k = 0; k < m; k++) {
            double ar = X[k][0], ai = (k == 0) ? 0.0 : X[k][1];
            int k2 = m - k;
            double br = X[k2][0], bi = (k2 == m || k2 == 0) ? 0.0 : X[k2][1];
            bi = -bi; /* conj X[m-k] */
            double er = ar + br, ei = ai + bi;      /* 2E */
            double dr = ar - br, di = ai - bi;      /* 2 W^k O */
            double wr = p->wn[2 * k], wi = -p->wn[2 * k + 1]; /* W^-k */
            double orr = dr * wr - di * wi, oi = dr * wi + di * wr; /* 2O */
            z[2 * k] = er - oi;   /* 2E + i 2O */
            z[2 * k + 1] = ei + orr;
        }
        cfft(p, z, +1);
        double *x = p->rbuf;
        for (int k = 0; k < m; k++) {
            x[2 * k] = z[2 * k];
            x[2 * k + 1] = z[2 * k + 1];
        }
    }
}
