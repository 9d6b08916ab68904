/*
 * fftw3.h -- the subset of the FFTW3 C interface that the reference's
 * order-4 executor paper/order4/cpp/gl_eta44_fftw.cpp calls (lines 32-69:
 * fftw_malloc, fftw_init_threads, fftw_plan_with_nthreads,
 * fftw_plan_dft_2d, fftw_execute, fftw_destroy_plan, fftw_cleanup_threads,
 * fftw_free), with FFTW's published names, types and sign convention, so
 * that executor builds from its own source without the FFTW library.
 *
 * Test infrastructure only (oracle/Makefile links it into oracle/_ref/):
 * the engine never links or runs it.  The transforms are this project's own
 * (fftw3_shim.c); they agree with FFTW to roundoff, not bit for bit.
 */
#ifndef GL_FFTW3_SHIM_H
#define GL_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct gl_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t bytes);
void fftw_free(void* p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
/* Unnormalised 2-D DFT of an n0 x n1 row-major array:
 * out[k0][k1] = sum in[j0][j1] exp(sign 2 pi i (j0 k0 / n0 + j1 k1 / n1)). */
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

#ifdef __cplusplus
}
#endif

#endif /* GL_FFTW3_SHIM_H */
