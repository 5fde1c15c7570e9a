/*
 * Oracle test infrastructure: FFTW stand-in.  A plan records the 3D extents
 * (n0 slowest, n2 fastest, as fftwf_plan_dft_3d documents) and the sign; an
 * execution copies `in` to `out` and transforms `out` in place with LFFT.
 */
#include "fftw3.h"

#include <stdlib.h>
#include <string.h>

#include "../restate/lfft.h"

struct lenia_fftwf_plan_s {
    int n0, n1, n2, sign;
};

fftwf_plan fftwf_plan_dft_3d(int n0, int n1, int n2, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags)
{
    (void)in; (void)out; (void)flags;
    fftwf_plan p = (fftwf_plan)malloc(sizeof(*p));
    p->n0 = n0; p->n1 = n1; p->n2 = n2; p->sign = sign;
    return p;
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out)
{
    size_t n = (size_t)p->n0 * p->n1 * p->n2;
    if (in != out) memmove(out, in, n * sizeof(fftwf_complex));
    lfft_3d_c2c((lcf *)out, p->n2, p->n1, p->n0, p->sign);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
