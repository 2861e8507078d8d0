/*
 * A working stand-in for the subset of the <fftw3.h> API that the reference's
 * weakly non-linear waveform mode calls (geoac.eqset.*.cpp wnl_wvfrm,
 * waveforms.cpp), so that the unmodified reference can be compiled here as
 * the waveform oracle.  Test infrastructure only: nothing here is linked into
 * the product library.  FFTW itself is not installed in this image; no FFTW
 * code is contained or reproduced here.
 *
 * Conventions are FFTW's published ones for the two plans used:
 *   r2c, size n:  X[k] = sum_{j<n} x[j] exp(-2 pi i j k / n), k = 0..n/2
 *   c2r, size n:  x[j] = sum_{k<n} X[k] exp(+2 pi i j k / n), unnormalised,
 *                 X[n-k] = conj(X[k]) implied; the imaginary parts of X[0]
 *                 and (even n) X[n/2] do not contribute (the result is the
 *                 real part of the Hermitian-extended sum).
 * The transforms are an iterative radix-2 Cooley-Tukey FFT for power-of-two
 * n (twiddles from cos/sin of the exact angle index) and a direct O(n^2)
 * sum for any other n.
 */
#ifndef IGA_ORACLE_FFTW3_SHIM_H_
#define IGA_ORACLE_FFTW3_SHIM_H_

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double fftw_complex[2];

struct iga_shim_plan {
    int n;
    int dir;            /* -1: r2c, +1: c2r */
    double* r;          /* the real array of the plan */
    fftw_complex* c;    /* the half-spectrum of the plan */
    double* wre;        /* twiddles exp(-2 pi i k / n), k < n/2 (power of two n) */
    double* wim;
    double* bre;        /* complex work array of length n */
    double* bim;
};
typedef struct iga_shim_plan* fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

static inline void* fftw_malloc(size_t bytes) { return malloc(bytes); }
static inline void fftw_free(void* p) { free(p); }

static inline int iga_shim_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static inline fftw_plan iga_shim_make(int n, int dir, double* r, fftw_complex* c) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(struct iga_shim_plan));
    p->n = n; p->dir = dir; p->r = r; p->c = c;
    p->bre = (double*)malloc(sizeof(double) * (size_t)n);
    p->bim = (double*)malloc(sizeof(double) * (size_t)n);
    if (iga_shim_pow2(n) && n >= 2) {
        p->wre = (double*)malloc(sizeof(double) * (size_t)(n / 2));
        p->wim = (double*)malloc(sizeof(double) * (size_t)(n / 2));
        const double two_pi = 6.283185307179586476925286766559;
        for (int k = 0; k < n / 2; k++) {
            p->wre[k] = cos(two_pi * (double)k / (double)n);
            p->wim[k] = -sin(two_pi * (double)k / (double)n);
        }
    }
    return p;
}

static inline fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned) {
    return iga_shim_make(n, -1, in, out);
}
static inline fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned) {
    return iga_shim_make(n, +1, out, in);
}

/* In-place complex transform of (re, im), length n, sign s (-1 forward). */
static inline void iga_shim_cfft(fftw_plan p, double* re, double* im, int s) {
    const int n = p->n;
    if (p->wre) {
        for (int i = 1, j = 0; i < n; i++) {          /* bit-reversal permutation */
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double t = re[i]; re[i] = re[j]; re[j] = t;
                t = im[i]; im[i] = im[j]; im[j] = t;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1, step = n / len;
            for (int b = 0; b < n; b += len) {
                for (int k = 0; k < half; k++) {
                    const double wr = p->wre[k * step], wi = s < 0 ? p->wim[k * step] : -p->wim[k * step];
                    const int i0 = b + k, i1 = b + k + half;
                    const double xr = re[i1] * wr - im[i1] * wi;
                    const double xi = re[i1] * wi + im[i1] * wr;
                    re[i1] = re[i0] - xr; im[i1] = im[i0] - xi;
                    re[i0] += xr; im[i0] += xi;
                }
            }
        }
    } else {
        const double two_pi = 6.283185307179586476925286766559;
        double* tr = (double*)malloc(sizeof(double) * (size_t)n);
        double* ti = (double*)malloc(sizeof(double) * (size_t)n);
        for (int k = 0; k < n; k++) {
            double ar = 0.0, ai = 0.0;
            for (int j = 0; j < n; j++) {
                const long long m = ((long long)j * k) % n;
                const double ang = two_pi * (double)m / (double)n;
                const double c = cos(ang), sn = s * sin(ang);
                ar += re[j] * c - im[j] * sn;
                ai += re[j] * sn + im[j] * c;
            }
            tr[k] = ar; ti[k] = ai;
        }
        memcpy(re, tr, sizeof(double) * (size_t)n);
        memcpy(im, ti, sizeof(double) * (size_t)n);
        free(tr); free(ti);
    }
}

static inline void fftw_execute(const fftw_plan p) {
    const int n = p->n, h = n / 2;
    double* re = p->bre;
    double* im = p->bim;
    if (p->dir < 0) {
        for (int j = 0; j < n; j++) { re[j] = p->r[j]; im[j] = 0.0; }
        iga_shim_cfft(p, re, im, -1);
        for (int k = 0; k <= h; k++) { p->c[k][0] = re[k]; p->c[k][1] = im[k]; }
    } else {
        for (int k = 0; k <= h; k++) { re[k] = p->c[k][0]; im[k] = p->c[k][1]; }
        im[0] = 0.0;
        if (n % 2 == 0) im[h] = 0.0;
        for (int k = h + 1; k < n; k++) { re[k] = re[n - k]; im[k] = -im[n - k]; }
        iga_shim_cfft(p, re, im, +1);
        for (int j = 0; j < n; j++) p->r[j] = re[j];
    }
}

static inline void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->wre); free(p->wim); free(p->bre); free(p->bim);
    free(p);
}

#endif
