/*
 * dfti_shim.c (oracle shim, TEST INFRASTRUCTURE) -- DFTI entry points on top of
 * the specified DFT (oracle/gg_dft.c).  Accepts exactly the descriptors the
 * reference builds at box.cpp:699-718 (forward) and box.cpp:775-792 (backward):
 * 3D, real domain, double precision, not in place, CCE storage, cubic lengths
 * {n,n,n}, real strides {0,n,n*n,1}, complex strides {0,n/2+1,(n/2+1)*n,1}.
 */
#include "mkl_dfti.h"
#include "../gg_dft.h"

#include <stdarg.h>
#include <stdlib.h>

struct gg_dfti_desc {
    long n;
    long in_strides[4];
    long out_strides[4];
    int precision, domain, placement, storage, have_in, have_out;
};

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, DFTI_CONFIG_VALUE precision,
                              DFTI_CONFIG_VALUE domain, MKL_LONG dimension, ...) {
    if (!h || dimension != 3) return 1;
    va_list ap;
    va_start(ap, dimension);
    const MKL_LONG* lengths = va_arg(ap, const MKL_LONG*);
    va_end(ap);
    if (!lengths || lengths[0] != lengths[1] || lengths[0] != lengths[2] || lengths[0] < 1) return 2;
    struct gg_dfti_desc* d = (struct gg_dfti_desc*)calloc(1, sizeof(*d));
    d->n = lengths[0];
    d->precision = precision;
    d->domain = domain;
    *h = d;
    return 0;
}

MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE d, DFTI_CONFIG_PARAM param, ...) {
    if (!d) return 1;
    va_list ap;
    va_start(ap, param);
    MKL_LONG rc = 0;
    switch (param) {
    case DFTI_PLACEMENT: d->placement = va_arg(ap, int); break;
    case DFTI_CONJUGATE_EVEN_STORAGE: d->storage = va_arg(ap, int); break;
    case DFTI_INPUT_STRIDES: {
        const MKL_LONG* s = va_arg(ap, const MKL_LONG*);
        for (int i = 0; i < 4; i++) d->in_strides[i] = s[i];
        d->have_in = 1;
        break;
    }
    case DFTI_OUTPUT_STRIDES: {
        const MKL_LONG* s = va_arg(ap, const MKL_LONG*);
        for (int i = 0; i < 4; i++) d->out_strides[i] = s[i];
        d->have_out = 1;
        break;
    }
    default: rc = 3;
    }
    va_end(ap);
    return rc;
}

static int strides_are(const long* s, long n, long inner) {
    return s[0] == 0 && s[1] == inner && s[2] == inner * n && s[3] == 1;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE d) {
    if (!d) return 1;
    if (d->precision != DFTI_DOUBLE || d->domain != DFTI_REAL || d->placement != DFTI_NOT_INPLACE ||
        d->storage != DFTI_COMPLEX_COMPLEX || !d->have_in || !d->have_out)
        return 4;
    long n = d->n, h = n / 2 + 1;
    /* forward descriptor: real in, complex out; backward: the reverse */
    int fwd = strides_are(d->in_strides, n, n) && strides_are(d->out_strides, n, h);
    int bwd = strides_are(d->in_strides, n, h) && strides_are(d->out_strides, n, n);
    return (fwd || bwd) ? 0 : 5;
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE d, void* in, ...) {
    va_list ap;
    va_start(ap, in);
    void* out = va_arg(ap, void*);
    va_end(ap);
    if (!d || !in || !out) return 1;
    ggdft_forward_r2c_3d((int)d->n, (const double*)in, (double*)out);
    return 0;
}

MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE d, void* in, ...) {
    va_list ap;
    va_start(ap, in);
    void* out = va_arg(ap, void*);
    va_end(ap);
    if (!d || !in || !out) return 1;
    ggdft_backward_c2r_3d((int)d->n, (const double*)in, (double*)out);
    return 0;
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h) {
    if (h && *h) { free(*h); *h = 0; }
    return 0;
}
