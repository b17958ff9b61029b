// Abort stubs for the FFTW and SEPlib entry points declared in fftw3.h and
// seplib.h.  None is reachable from the propagation functions the oracle
// build exercises.
#include <cstdio>
#include <cstdlib>
#include "fftw3.h"
#include "seplib.h"

[[noreturn]] static void off_path(const char *what)
{
    std::fprintf(stderr, "oracle reference build: %s is not available\n", what);
    std::abort();
}
extern "C" {
void *fftw_malloc(size_t) { off_path("fftw_malloc"); }
void fftw_free(void *) { off_path("fftw_free"); }
void fftw_execute(const fftw_plan) { off_path("fftw_execute"); }
void fftw_destroy_plan(fftw_plan) { off_path("fftw_destroy_plan"); }
void fftw_cleanup(void) { off_path("fftw_cleanup"); }
fftw_plan fftw_plan_dft_1d(int, fftw_complex *, fftw_complex *, int, unsigned) { off_path("fftw_plan"); }
fftw_plan fftw_plan_dft_2d(int, int, fftw_complex *, fftw_complex *, int, unsigned) { off_path("fftw_plan"); }
fftw_plan fftw_plan_dft_r2c_1d(int, double *, fftw_complex *, unsigned) { off_path("fftw_plan"); }
fftw_plan fftw_plan_dft_r2c_2d(int, int, double *, fftw_complex *, unsigned) { off_path("fftw_plan"); }
fftw_plan fftw_plan_dft_c2r_1d(int, fftw_complex *, double *, unsigned) { off_path("fftw_plan"); }
fftw_plan fftw_plan_dft_c2r_2d(int, int, fftw_complex *, double *, unsigned) { off_path("fftw_plan"); }
void *fftwf_malloc(size_t) { off_path("fftwf_malloc"); }
void fftwf_free(void *) { off_path("fftwf_free"); }
void fftwf_execute(const fftwf_plan) { off_path("fftwf_execute"); }
void fftwf_destroy_plan(fftwf_plan) { off_path("fftwf_destroy_plan"); }
void fftwf_cleanup(void) { off_path("fftwf_cleanup"); }
fftwf_plan fftwf_plan_dft_1d(int, fftwf_complex *, fftwf_complex *, int, unsigned) { off_path("fftwf_plan"); }
fftwf_plan fftwf_plan_dft_2d(int, int, fftwf_complex *, fftwf_complex *, int, unsigned) { off_path("fftwf_plan"); }
fftwf_plan fftwf_plan_dft_r2c_1d(int, float *, fftwf_complex *, unsigned) { off_path("fftwf_plan"); }
fftwf_plan fftwf_plan_dft_r2c_2d(int, int, float *, fftwf_complex *, unsigned) { off_path("fftwf_plan"); }
fftwf_plan fftwf_plan_dft_c2r_1d(int, fftwf_complex *, float *, unsigned) { off_path("fftwf_plan"); }
fftwf_plan fftwf_plan_dft_c2r_2d(int, int, fftwf_complex *, float *, unsigned) { off_path("fftwf_plan"); }
int putch(const char *, const char *, const void *) { off_path("putch"); }
int auxputch(const char *, const char *, const void *, const char *) { off_path("auxputch"); }
int hetch(const char *, const char *, void *) { off_path("hetch"); }
int auxpar(const char *, const char *, void *, const char *) { off_path("auxpar"); }
long long sreed_big(const char *, void *, long long) { off_path("sreed_big"); }
long long srite_big(const char *, void *, long long) { off_path("srite_big"); }
void initpar(int, char **) { off_path("initpar"); }
}
