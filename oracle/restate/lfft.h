/*
 * Oracle test infrastructure: CPU implementation of the project's FFT
 * specification ("LFFT"), used by
 *   - the FFTW stand-in that the reference build links against
 *     (fftwf_plan_dft_3d / fftwf_execute_dft, lenia.cpp:193-194, 259, 488,
 *     1043; reintegration.cpp:76, 124, 128, 141, 153), and
 *   - the C restatement of the simulation step (lenia_oracle.c).
 *
 * FFTW 3 (single precision, version unpinned: the reference ships no build
 * files) is absent from this machine.  Its published contract is the
 * unnormalised DFT  X[k] = sum_j x[j] exp(sign * 2 pi i j k / n)  with
 * sign = -1 (FFTW_FORWARD) and +1 (FFTW_BACKWARD).  LFFT computes that
 * transform; its exact float operation order is the one the CUDA library
 * uses, so CPU and GPU results agree bit for bit.  The order is:
 *
 *   radix plan: greedy 8s, then 4, then 2, then 3s, 5s, 7s, 11s;
 *   Stockham autosort stages Ns = 1, R1, R1*R2, ...: for j in [0, n/R)
 *     v[r] = x[j + r*n/R];  if (j % Ns) v[r] *= tw[r*(j%Ns)*(n/(Ns*R))] (r>=1)
 *     v = DFT_R(v);  y[(j/Ns)*Ns*R + j%Ns + r*Ns] = v[r]
 *   tw[t] = (cos(2 pi t/n), sign*sin(2 pi t/n)) evaluated in double, stored
 *   as float; complex products (a*c - b*d, a*d + b*c) without fused
 *   multiply-add; DFT_R butterflies as written in lfft.c.
 */
#ifndef LENIA_ORACLE_LFFT_H
#define LENIA_ORACLE_LFFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } lcf;

#define LFFT_MAX_STAGES 16

typedef struct {
    int n;
    int nstages;
    int radix[LFFT_MAX_STAGES];
    lcf *tw_fwd; /* n entries: (cos, -sin) */
    lcf *tw_inv; /* n entries: (cos, +sin) */
} lfft_plan;

/* Radix plan for length n; returns number of stages or -1 if n has a prime
 * factor outside {2,3,5,7,11}. */
int lfft_factor(int n, int *radix);

int lfft_plan_init(lfft_plan *p, int n);
void lfft_plan_free(lfft_plan *p);

/* In-place 1D transform of n elements spaced `stride` apart.  `work` must hold
 * 2*n elements.  sign = -1 forward, +1 inverse (unnormalised). */
void lfft_1d(const lfft_plan *p, lcf *x, long stride, int sign, lcf *work);

/* In-place 3D complex transform of an array laid out [d][h][w] (w fastest):
 * 1D transforms along w, then h, then d. */
void lfft_3d_c2c(lcf *x, int w, int h, int d, int sign);

#ifdef __cplusplus
}
#endif
#endif
