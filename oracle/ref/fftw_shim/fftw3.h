/* Test-infrastructure stand-in for the part of FFTW 3's interface that the
 * reference's blocked Cowan reference calls (src/blocked_cowan_reference.cpp:
 * PlaneDST): a two-dimensional real-to-real plan of kind FFTW_RODFT00 along
 * both axes, executed in place and destroyed.  FFTW is not in this image.
 * RODFT00 is FFTW's documented type-I discrete sine transform,
 *   Y_k = 2 * sum_{j=0}^{n-1} X_j sin(pi (j+1)(k+1) / (n+1)),
 * applied along each axis of the row-major n0 x n1 array (unnormalised,
 * like FFTW's).  The stand-in evaluates the sums directly, so its results
 * agree with FFTW's to rounding, not bit for bit.  Built only into
 * oracle/_ref; nothing in the product links it. */
#ifndef APRL_ORACLE_FFTW_SHIM_H
#define APRL_ORACLE_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { FFTW_RODFT00 = 8 } fftw_r2r_kind;
#define FFTW_ESTIMATE (1U << 6)

typedef struct aprl_fftw_plan_s* fftw_plan;

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double* in, double* out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

#ifdef __cplusplus
}
#endif
#endif
