/*
 * Project-written stand-in for the small part of the FFTW3 single-precision
 * API that the reference gridding C code calls.  TEST INFRASTRUCTURE ONLY:
 * it exists so that the reference's gridrec_v4_forwproj.c / _backproj.c /
 * filters.c compile into oracle/_ref/ when FFTW3 itself is not installed.
 *
 * Conventions follow FFTW's published definition of the DFT:
 *   out[k] = sum_j in[j] * exp(sign * 2*pi*i * j*k / n),  unnormalised,
 *   FFTW_FORWARD = -1, FFTW_BACKWARD = +1, 2-D transforms row-major.
 * Arithmetic is done in double precision (fftw_standin.c), then rounded to
 * float, so the stand-in is at least as accurate as FFTW's float transforms.
 *
 * Call sites covered (reference, file:line):
 *   gridrec_v4_forwproj.c:101-105,146,170,256-259,267,390,426-437
 *   gridrec_v4_backproj.c:134-138,165,235,241-243,301,413,427-430,502-503
 *   gridrec_v4_backproj.c:516-543 (wisdom helper), filters.c:164-176
 */
#ifndef TOMO_FFTW3_STANDIN_H
#define TOMO_FFTW3_STANDIN_H

#include <stdio.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)

void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in,
                             fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
int fftwf_import_wisdom_from_file(FILE *f);
void fftwf_export_wisdom_to_file(FILE *f);

#ifdef __cplusplus
}
#endif

#endif
