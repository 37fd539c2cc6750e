/* Minimal FFTW3-compatible interface for the oracle build of the reference
 * (test infrastructure only).  The reference uses exactly one FFTW feature:
 * an in-place, unnormalised 3-D complex DFT on a (2P)^3 grid
 * (src/wave3d_setup.cpp:81-95, src/wave3d_eval.cpp:631,651).
 * Forward sign is -1 (exp(-2 pi i jk/n)), backward +1, as in FFTW. */
#ifndef DDFMM_ORACLE_FFTW3_STUB_H
#define DDFMM_ORACLE_FFTW3_STUB_H
#include <stdio.h>
#include <stdlib.h>
#include <math.h>

typedef double fftw_complex[2];
typedef struct ddfmm_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

#ifdef __cplusplus
extern "C" {
#endif
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
#endif
