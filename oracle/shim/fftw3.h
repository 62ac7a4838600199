/* Build shim for compiling the reference with cuFFTW in place of FFTW3,
 * which is not installed on these machines: cuFFTW exports the FFTW3 API
 * (fftw_plan_dft_1d, fftw_execute, fftw_malloc, ...). */
#include <cufftw.h>
