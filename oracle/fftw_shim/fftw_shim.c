/*
 * fftw_shim.c -- CPU mixed-radix FFT behind the FFTW3 API subset in fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  The reference calls FFTW3 for every
 * spectral transform (OP_FFT.cpp:26,54; OP_iFFT.cpp:26,57; operations.cpp:230,260);
 * FFTW3 is absent here, so this file restates the discrete Fourier transform
 * that FFTW computes, with FFTW's documented conventions:
 *   r2c 3-D: X[i][j][k] = sum_{a,b,c} x[a][b][c] e^{-2 pi i (ia/n0 + jb/n1 + kc/n2)},
 *            k = 0..n2/2 (half spectrum, last dimension);
 *   c2r 3-D: the Hermitian inverse with sign +1, unnormalised.
 * The 1-D kernel is a Stockham autosort FFT (decimation in time) with radix
 * 4/2 butterflies and a generic small-prime DFT for the other factors
 * (published algorithm: Stockham autosort as formulated in Van Loan,
 * "Computational Frameworks for the FFT", 1992).  Twiddles come from a
 * table computed in long double.
 *
 * Real transforms along the last dimension pack two real rows as one complex
 * row (z = a + i b) and separate the spectra afterwards; on the inverse the
 * imaginary parts of the k=0 and k=n2/2 bins are ignored, as a Hermitian
 * c2r transform does.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef KFS_THREADS
#include <pthread.h>
#include <unistd.h>
#endif

/* ------------------------------------------------------------ host threads */
int kfs_nthreads(void) {
#ifdef KFS_THREADS
    static int nt = 0;
    if (!nt) {
        const char *e = getenv("KF_ORACLE_THREADS");
        long v = e ? strtol(e, NULL, 10) : sysconf(_SC_NPROCESSORS_ONLN);
        nt = v < 1 ? 1 : (v > 256 ? 256 : (int)v);
    }
    return nt;
#else
    return 1;
#endif
}

#ifdef KFS_THREADS
typedef struct {
    kfs_range_fn fn;
    void *ctx;
    long b, e;
} kfs_piece;

static void *kfs_piece_run(void *a) {
    kfs_piece *p = (kfs_piece *)a;
    p->fn(p->b, p->e, p->ctx);
    return NULL;
}
#endif

void kfs_parallel(long n, long min_items, kfs_range_fn fn, void *ctx) {
    if (n <= 0) return;
    long T = kfs_nthreads();
    if (min_items < 1) min_items = 1;
    if (T > n / min_items) T = n / min_items;
#ifdef KFS_THREADS
    if (T > 1) {
        pthread_t th[256];
        kfs_piece pc[256];
        int started[256];
        for (long t = 0; t < T; ++t) {
            pc[t].fn = fn;
            pc[t].ctx = ctx;
            pc[t].b = n * t / T;
            pc[t].e = n * (t + 1) / T;
            started[t] = t > 0 && pthread_create(&th[t], NULL, kfs_piece_run, &pc[t]) == 0;
        }
        for (long t = 0; t < T; ++t)
            if (!started[t]) kfs_piece_run(&pc[t]); /* piece 0, or a thread that could not start */
        for (long t = 1; t < T; ++t)
            if (started[t]) pthread_join(th[t], NULL);
        return;
    }
#endif
    fn(0, n, ctx);
}

#define KFS_MAXF 40

typedef struct {
    int n;
    int nf;
    int fac[KFS_MAXF];
    double *tw; /* e^{-2 pi i m / n}, m = 0..n-1, interleaved */
} kfs_plan1d;

static void kfs_plan1d_init(kfs_plan1d *p, int n) {
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    for (int r = 3; m > 1; r += 2) {
        while (m % r == 0) { p->fac[p->nf++] = r; m /= r; }
    }
    for (int s = 0; s < p->nf; ++s)
        if (p->fac[s] > 64) abort(); /* radix beyond the butterfly buffers */
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int i = 0; i < n; ++i) {
        long double ang = twopi * (long double)i / (long double)n;
        p->tw[2 * i] = (double)cosl(ang);
        p->tw[2 * i + 1] = (double)(-sinl(ang));
    }
}

static void kfs_plan1d_free(kfs_plan1d *p) { free(p->tw); p->tw = NULL; }

/* One Stockham stage on B interleaved lines: x[(t*B+b)], complex. */
static void kfs_stage(const kfs_plan1d *p, int R, int Ns, int B, int sign,
                      const double *x, double *y) {
    const int n = p->n;
    const int nR = n / R;
    const int tstep = n / (Ns * R); /* twiddle index multiplier */
    const double *tw = p->tw;
    double ar[64], ai[64];
    double br[64], bi[64];
    for (int j = 0; j < nR; ++j) {
        const int k = j % Ns;
        const int idxD = (j / Ns) * Ns * R + k;
        for (int b = 0; b < B; ++b) {
            for (int t = 0; t < R; ++t) {
                const double *src = x + 2 * ((size_t)(j + t * nR) * B + b);
                double re = src[0], im = src[1];
                if (t && k) {
                    int m = (t * k * tstep) % n;
                    double wr = tw[2 * m], wi = sign < 0 ? tw[2 * m + 1] : -tw[2 * m + 1];
                    double tr = re * wr - im * wi;
                    im = re * wi + im * wr;
                    re = tr;
                }
                ar[t] = re;
                ai[t] = im;
            }
            if (R == 4) {
                double s0r = ar[0] + ar[2], s0i = ai[0] + ai[2];
                double d0r = ar[0] - ar[2], d0i = ai[0] - ai[2];
                double s1r = ar[1] + ar[3], s1i = ai[1] + ai[3];
                double d1r = ar[1] - ar[3], d1i = ai[1] - ai[3];
                /* w = sign * i ; w*(x+iy) = sign*(-y + i x) */
                double wdr = sign < 0 ? d1i : -d1i;
                double wdi = sign < 0 ? -d1r : d1r;
                br[0] = s0r + s1r; bi[0] = s0i + s1i;
                br[1] = d0r + wdr; bi[1] = d0i + wdi;
                br[2] = s0r - s1r; bi[2] = s0i - s1i;
                br[3] = d0r - wdr; bi[3] = d0i - wdi;
            } else if (R == 2) {
                br[0] = ar[0] + ar[1]; bi[0] = ai[0] + ai[1];
                br[1] = ar[0] - ar[1]; bi[1] = ai[0] - ai[1];
            } else {
                const int tq = n / R;
                for (int q = 0; q < R; ++q) {
                    double sr = ar[0], si = ai[0];
                    for (int t = 1; t < R; ++t) {
                        int m = ((t * q) % R) * tq;
                        double wr = tw[2 * m], wi = sign < 0 ? tw[2 * m + 1] : -tw[2 * m + 1];
                        sr += ar[t] * wr - ai[t] * wi;
                        si += ar[t] * wi + ai[t] * wr;
                    }
                    br[q] = sr;
                    bi[q] = si;
                }
            }
            for (int t = 0; t < R; ++t) {
                double *dst = y + 2 * ((size_t)(idxD + t * Ns) * B + b);
                dst[0] = br[t];
                dst[1] = bi[t];
            }
        }
    }
}

/* FFT of B interleaved lines in place (buf), scratch of the same size. */
static void kfs_exec1d(const kfs_plan1d *p, int B, int sign, double *buf, double *scratch) {
    double *x = buf, *y = scratch;
    int Ns = 1;
    for (int s = 0; s < p->nf; ++s) {
        int R = p->fac[s];
        kfs_stage(p, R, Ns, B, sign, x, y);
        double *t = x; x = y; y = t;
        Ns *= R;
    }
    if (x != buf) memcpy(buf, x, sizeof(double) * 2 * (size_t)p->n * B);
}

#define KFS_B 8

/* Complex FFT along a strided axis of an interleaved complex array:
 * lines are data[off + t*stride] for t < n, with the line start offsets
 * given by  outer * ostride + c  for outer < nouter, c < ninner (contiguous). */
typedef struct {
    const kfs_plan1d *p;
    double *data;
    long nblk;
    size_t ostride, stride;
    int ninner, sign;
} kfs_axis_job;

/* line blocks [b, e) of an axis pass; scratch per piece */
static void kfs_axis_range(long b, long e, void *ctx) {
    const kfs_axis_job *J = (const kfs_axis_job *)ctx;
    const int n = J->p->n;
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)n * KFS_B);
    double *scr = (double *)malloc(sizeof(double) * 2 * (size_t)n * KFS_B);
    for (long w = b; w < e; ++w) {
        const int o = (int)(w / J->nblk), c0 = (int)(w % J->nblk) * KFS_B;
        int B = J->ninner - c0 < KFS_B ? J->ninner - c0 : KFS_B;
        for (int t = 0; t < n; ++t) {
            const double *src = J->data + 2 * (o * J->ostride + (size_t)t * J->stride + c0);
            memcpy(buf + 2 * (size_t)t * B, src, sizeof(double) * 2 * B);
        }
        kfs_exec1d(J->p, B, J->sign, buf, scr);
        for (int t = 0; t < n; ++t) {
            double *dst = J->data + 2 * (o * J->ostride + (size_t)t * J->stride + c0);
            memcpy(dst, buf + 2 * (size_t)t * B, sizeof(double) * 2 * B);
        }
    }
    free(buf);
    free(scr);
}

/* Complex FFT along a strided axis of an interleaved complex array:
 * lines are data[off + t*stride] for t < n, with the line start offsets
 * given by  outer * ostride + c  for outer < nouter, c < ninner (contiguous).
 * Blocks of KFS_B lines are independent, and a line's arithmetic does not
 * depend on its block. */
static void kfs_axis_pass(const kfs_plan1d *p, double *data, int nouter, size_t ostride,
                          int ninner, size_t stride, int sign) {
    kfs_axis_job J = {p, data, (ninner + KFS_B - 1) / KFS_B, ostride, stride, ninner, sign};
    kfs_parallel((long)nouter * J.nblk, 4, kfs_axis_range, &J);
}

typedef struct {
    const kfs_plan1d *p;
    const double *in;
    double *out;
    size_t rows;
    int n2, nzc;
} kfs_z_job;

/* z pass of an r2c: row pairs [b, e) packed as one complex line each */
static void kfs_r2c_z_range(long b, long e, void *ctx) {
    const kfs_z_job *J = (const kfs_z_job *)ctx;
    const int n2 = J->n2, nzc = J->nzc;
    double *z = (double *)malloc(sizeof(double) * 2 * n2);
    double *s = (double *)malloc(sizeof(double) * 2 * n2);
    for (long r2 = b; r2 < e; ++r2) {
        const size_t r = 2 * (size_t)r2;
        const double *a = J->in + r * n2;
        const double *bb = (r + 1 < J->rows) ? J->in + (r + 1) * n2 : NULL;
        for (int t = 0; t < n2; ++t) {
            z[2 * t] = a[t];
            z[2 * t + 1] = bb ? bb[t] : 0.0;
        }
        kfs_exec1d(J->p, 1, -1, z, s);
        double *oa = J->out + 2 * r * nzc;
        double *ob = bb ? J->out + 2 * (r + 1) * nzc : NULL;
        for (int k = 0; k < nzc; ++k) {
            int km = (n2 - k) % n2;
            double zr = z[2 * k], zi = z[2 * k + 1];
            double cr = z[2 * km], ci = -z[2 * km + 1]; /* conj(Z[n-k]) */
            oa[2 * k] = 0.5 * (zr + cr);
            oa[2 * k + 1] = 0.5 * (zi + ci);
            if (ob) { /* (Z - conj Z[n-k]) / (2i) */
                ob[2 * k] = 0.5 * (zi - ci);
                ob[2 * k + 1] = -0.5 * (zr - cr);
            }
        }
    }
    free(z);
    free(s);
}

void kfs_r2c_3d(int n0, int n1, int n2, const double *in, double *out) {
    const int nzc = n2 / 2 + 1;
    const size_t rows = (size_t)n0 * n1;
    kfs_plan1d pz, py, px;
    kfs_plan1d_init(&pz, n2);
    kfs_z_job J = {&pz, in, out, rows, n2, nzc};
    kfs_parallel((long)((rows + 1) / 2), 8, kfs_r2c_z_range, &J);
    kfs_plan1d_free(&pz);
    kfs_plan1d_init(&py, n1);
    kfs_axis_pass(&py, out, n0, (size_t)n1 * nzc, nzc, (size_t)nzc, -1);
    kfs_plan1d_free(&py);
    kfs_plan1d_init(&px, n0);
    kfs_axis_pass(&px, out, 1, 0, n1 * nzc, (size_t)n1 * nzc, -1);
    kfs_plan1d_free(&px);
}

/* z pass of a c2r: row pairs [b, e) from the Hermitian half spectra */
static void kfs_c2r_z_range(long b, long e, void *ctx) {
    const kfs_z_job *J = (const kfs_z_job *)ctx;
    const int n2 = J->n2, nzc = J->nzc;
    double *z = (double *)malloc(sizeof(double) * 2 * n2);
    double *s = (double *)malloc(sizeof(double) * 2 * n2);
    for (long r2 = b; r2 < e; ++r2) {
        const size_t r = 2 * (size_t)r2;
        const double *A = J->in + 2 * r * nzc;
        const double *Bv = (r + 1 < J->rows) ? J->in + 2 * (r + 1) * nzc : NULL;
        for (int k = 0; k < n2; ++k) {
            double ar, ai, br = 0.0, bi = 0.0;
            if (k < nzc) {
                ar = A[2 * k];
                ai = A[2 * k + 1];
                if (Bv) { br = Bv[2 * k]; bi = Bv[2 * k + 1]; }
                if (k == 0 || 2 * k == n2) { ai = 0.0; bi = 0.0; }
            } else {
                int km = n2 - k;
                ar = A[2 * km];
                ai = -A[2 * km + 1];
                if (Bv) { br = Bv[2 * km]; bi = -Bv[2 * km + 1]; }
            }
            /* Z = A + i B */
            z[2 * k] = ar - bi;
            z[2 * k + 1] = ai + br;
        }
        kfs_exec1d(J->p, 1, +1, z, s);
        double *oa = J->out + r * n2;
        double *ob = Bv ? J->out + (r + 1) * n2 : NULL;
        for (int t = 0; t < n2; ++t) {
            oa[t] = z[2 * t];
            if (ob) ob[t] = z[2 * t + 1];
        }
    }
    free(z);
    free(s);
}

void kfs_c2r_3d(int n0, int n1, int n2, const double *in, double *out) {
    const int nzc = n2 / 2 + 1;
    const size_t rows = (size_t)n0 * n1;
    double *w = (double *)malloc(sizeof(double) * 2 * rows * nzc);
    memcpy(w, in, sizeof(double) * 2 * rows * nzc);
    kfs_plan1d px, py, pz;
    kfs_plan1d_init(&px, n0);
    kfs_axis_pass(&px, w, 1, 0, n1 * nzc, (size_t)n1 * nzc, +1);
    kfs_plan1d_free(&px);
    kfs_plan1d_init(&py, n1);
    kfs_axis_pass(&py, w, n0, (size_t)n1 * nzc, nzc, (size_t)nzc, +1);
    kfs_plan1d_free(&py);
    kfs_plan1d_init(&pz, n2);
    kfs_z_job J = {&pz, w, out, rows, n2, nzc};
    kfs_parallel((long)((rows + 1) / 2), 8, kfs_c2r_z_range, &J);
    kfs_plan1d_free(&pz);
    free(w);
}

void kfs_fft_1d(int n, int sign, double *data) {
    kfs_plan1d p;
    kfs_plan1d_init(&p, n);
    double *s = (double *)malloc(sizeof(double) * 2 * n);
    kfs_exec1d(&p, 1, sign < 0 ? -1 : 1, data, s);
    free(s);
    kfs_plan1d_free(&p);
}

/* ---------------------------------------------------------------- FFTW API */

struct kfs_plan_s {
    int kind; /* 0 = r2c, 1 = c2r */
    int n0, n1, n2;
    double *rin;
    double *cio;
};

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    return p;
}

void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out,
                               unsigned flags) {
    (void)flags;
    struct kfs_plan_s *p = (struct kfs_plan_s *)calloc(1, sizeof(*p));
    p->kind = 0;
    p->n0 = n0; p->n1 = n1; p->n2 = n2;
    p->rin = in;
    p->cio = (double *)out;
    return p;
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out,
                               unsigned flags) {
    (void)flags;
    struct kfs_plan_s *p = (struct kfs_plan_s *)calloc(1, sizeof(*p));
    p->kind = 1;
    p->n0 = n0; p->n1 = n1; p->n2 = n2;
    p->rin = out;
    p->cio = (double *)in;
    return p;
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if (p->kind == 0)
        kfs_r2c_3d(p->n0, p->n1, p->n2, p->rin, p->cio);
    else
        kfs_c2r_3d(p->n0, p->n1, p->n2, p->cio, p->rin);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
