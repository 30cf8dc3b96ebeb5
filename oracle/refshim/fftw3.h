/* Declarations only, for the reference's FFT Poynting sensor, which the
 * oracle driver never instantiates; the stubs in refstubs.cpp abort if called. */
#ifndef AEORACLE_FFTW_SHIM
#define AEORACLE_FFTW_SHIM
typedef double fftw_complex[2];
typedef struct aeoracle_fftw_plan_s *fftw_plan;
#define FFTW_BACKWARD (+1)
#define FFTW_FORWARD (-1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
void *fftw_malloc(unsigned long n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#endif
