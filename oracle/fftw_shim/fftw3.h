/*
 * Minimal FFTW3-compatible declarations, written for this project.
 *
 * Test infrastructure only. The reference propagators (WaveFD src/prop*.h) call
 * fftwf_plan_dft_1d / fftwf_execute_dft / fftwf_destroy_plan for the wavefield-separation
 * imaging condition (e.g. prop3DAcoIsoDenQ_DEO2_FDTD.h:673-765). FFTW is not installed in
 * this image, so the reference is compiled against these declarations and the plain DFT in
 * fftw_shim.c, which follows FFTW's published conventions: unnormalised transform,
 * out[k] = sum_j in[j] * exp(sign * 2*pi*i*j*k/n), sign -1 called "forward" by FFTW.
 */
#ifndef WAVEFD_ORACLE_FFTW_SHIM_H
#define WAVEFD_ORACLE_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct wfd_shim_plan *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif

#endif
