/*
 * mkl_dfti.h (oracle shim, TEST INFRASTRUCTURE) -- the subset of the DFTI
 * interface that the reference's convolution calls (box.cpp:685-795), declared
 * here so that the reference compiles without Intel MKL.  The transforms behind
 * it are the specified DFT of oracle/gg_dft.c; only the configuration the
 * reference uses (3D, real, double, not-in-place, CCE storage, x-contiguous
 * cubic strides) is accepted -- anything else returns an error status.
 */
#ifndef GG_SHIM_MKL_DFTI_H
#define GG_SHIM_MKL_DFTI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef long MKL_LONG;
typedef struct { double real; double imag; } MKL_Complex16;

typedef enum {
    DFTI_PRECISION = 3, DFTI_FORWARD_DOMAIN = 0, DFTI_DIMENSION = 1, DFTI_LENGTHS = 2,
    DFTI_PLACEMENT = 11, DFTI_INPUT_STRIDES = 12, DFTI_OUTPUT_STRIDES = 13,
    DFTI_CONJUGATE_EVEN_STORAGE = 18, DFTI_INPUT_DISTANCE = 14, DFTI_OUTPUT_DISTANCE = 15
} DFTI_CONFIG_PARAM;

typedef enum {
    DFTI_COMMITTED = 30, DFTI_UNCOMMITTED = 31, DFTI_COMPLEX = 32, DFTI_REAL = 33,
    DFTI_SINGLE = 35, DFTI_DOUBLE = 36, DFTI_COMPLEX_COMPLEX = 39, DFTI_COMPLEX_REAL = 40,
    DFTI_INPLACE = 43, DFTI_NOT_INPLACE = 44
} DFTI_CONFIG_VALUE;

struct gg_dfti_desc;
typedef struct gg_dfti_desc* DFTI_DESCRIPTOR_HANDLE;

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, DFTI_CONFIG_VALUE precision,
                              DFTI_CONFIG_VALUE domain, MKL_LONG dimension, ...);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, DFTI_CONFIG_PARAM param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void* in, ...);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void* in, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h);

#ifdef __cplusplus
}
#endif
#endif
