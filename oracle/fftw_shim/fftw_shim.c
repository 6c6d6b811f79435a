/*
 * Plain complex DFT behind the FFTW3 API subset declared in fftw3.h (test infrastructure).
 *
 * Accumulates in double with exact-index twiddles (j*k mod n), then rounds once to float,
 * so it is at least as accurate as FFTW's own single-precision transforms. Execution is
 * re-entrant: the reference calls fftwf_execute_dft from inside OpenMP regions with one
 * shared plan (prop3DAcoIsoDenQ_DEO2_FDTD.h:691-737).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

struct wfd_shim_plan {
    int n;
    int sign;
    double *cosv; /* cos(2*pi*m/n), m = 0..n-1 */
    double *sinv; /* sin(2*pi*m/n) */
};

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags) {
    (void)in;
    (void)out;
    (void)flags;
    struct wfd_shim_plan *p = (struct wfd_shim_plan *)calloc(1, sizeof(*p));
    p->n = n;
    p->sign = sign;
    p->cosv = (double *)malloc(sizeof(double) * (size_t)n);
    p->sinv = (double *)malloc(sizeof(double) * (size_t)n);
    const double twopi = 6.283185307179586476925286766559;
    for (int m = 0; m < n; m++) {
        p->cosv[m] = cos(twopi * (double)m / (double)n);
        p->sinv[m] = sin(twopi * (double)m / (double)n);
    }
    return p;
}

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out) {
    const int n = p->n;
    double *acc = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int k = 0; k < n; k++) {
        double re = 0.0, im = 0.0;
        long m = 0;
        for (int j = 0; j < n; j++) {
            const double c = p->cosv[m];
            const double s = p->sign * p->sinv[m];
            const double xr = in[j][0], xi = in[j][1];
            re += xr * c - xi * s;
            im += xr * s + xi * c;
            m += k;
            if (m >= n) m -= n;
        }
        acc[2 * k] = re;
        acc[2 * k + 1] = im;
    }
    for (int k = 0; k < n; k++) {
        out[k][0] = (float)acc[2 * k];
        out[k][1] = (float)acc[2 * k + 1];
    }
    free(acc);
}

void fftwf_destroy_plan(fftwf_plan p) {
    if (!p) return;
    free(p->cosv);
    free(p->sinv);
    free(p);
}
