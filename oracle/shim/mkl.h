/* mkl.h (oracle shim, TEST INFRASTRUCTURE): the reference includes it
 * (grainhdl.cpp:42) only for the DFTI declarations. */
#include "mkl_dfti.h"
