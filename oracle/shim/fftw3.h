/* The reference includes <fftw3.h> (src/admin/admin.hpp:10) for the wavelet
 * filter of set_wavelet (src/modeling/modeling.cu:50-88).  FFTW3 is not
 * installed in this image; cuFFTW provides the same fftw_* API on the GPU. */
#include <cufftw.h>
