/*
 * Oracle test infrastructure: the subset of FFTW 3's single-precision API that
 * the reference calls (lenia.cpp:193-194, 259, 488, 1043; reintegration.cpp:76,
 * 124, 128, 141, 153).  FFTW itself is absent here; fftw_shim.c implements the
 * unnormalised DFT that FFTW documents, using the project's LFFT engine.
 */
#ifndef LENIA_REFSHIM_FFTW3_H
#define LENIA_REFSHIM_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct lenia_fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
#endif
