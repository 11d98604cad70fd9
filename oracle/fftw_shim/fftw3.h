/*
 * fftw3.h -- a minimal FFTW3-API shim used only by the CPU oracle.
 *
 * TEST INFRASTRUCTURE: this header and fftw_shim.c exist so that the
 * reference's own FFT call sites (OP_FFT.cpp:26,54, OP_iFFT.cpp:26,57,
 * operations.cpp:230-232,260-262) and the oracle restatement can be compiled
 * without FFTW3, which is neither vendored by the reference (its makefile:46
 * links -lfftw3 -lfftw3_threads, no version pinned) nor installed here.
 * Nothing in the product (kielflow_b200/) links it.
 *
 * Only the subset of the FFTW3 API that the reference's hot path calls is
 * declared: fftw_malloc/fftw_free, fftw_plan_dft_r2c_3d / fftw_plan_dft_c2r_3d,
 * fftw_execute, fftw_destroy_plan and the fftw_complex type.  Conventions
 * follow FFTW's documented ones: row-major n0 x n1 x n2 real array, half
 * spectrum n0 x n1 x (n2/2+1) complex, forward sign -1 unnormalised, backward
 * sign +1 unnormalised.  The transform itself is a mixed-radix Stockham FFT
 * written from the DFT definition (see fftw_shim.c); it is NOT FFTW code.
 */
#ifndef KF_FFTW_SHIM_H_
#define KF_FFTW_SHIM_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct kfs_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_EXHAUSTIVE (1U << 3)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Direct entry points (no plan object) used by the Python tests to pin the
 * shim against numpy.fft.  Unnormalised in both directions, like FFTW. */
void kfs_r2c_3d(int n0, int n1, int n2, const double *in, double *out_interleaved);
void kfs_c2r_3d(int n0, int n1, int n2, const double *in_interleaved, double *out);
void kfs_fft_1d(int n, int sign, double *data_interleaved);

/* Runs fn(begin, end, ctx) over contiguous pieces of [0, n) on the host's
 * cores (threads only when built with KFS_THREADS, the oracle's build; the
 * reference's build stays single-threaded, as FFTW_ESTIMATE plans without
 * fftw_plan_with_nthreads are).  Pieces of fewer than min_items items are not
 * split off.  Callers give each item work whose result does not depend on the
 * other items, so the number of threads changes no result. */
typedef void (*kfs_range_fn)(long begin, long end, void *ctx);
void kfs_parallel(long n, long min_items, kfs_range_fn fn, void *ctx);
/* threads kfs_parallel uses: KF_ORACLE_THREADS, else the online cores (1
 * without KFS_THREADS) */
int kfs_nthreads(void);

#ifdef __cplusplus
}
#endif

#endif
