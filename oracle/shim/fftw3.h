/* fftw3.h (oracle shim, TEST INFRASTRUCTURE): box.h:31 includes FFTW
 * unconditionally, but every FFTW use sits behind USE_FFTW, which the reference
 * build does not define (CMakeLists.txt:52 defines USE_MKL).  Nothing to declare. */
