// 2DIR family (calc_2DIR.c:22-629) on the device.
#include "common.cuh"
#include "engine.h"
#include "nise_internal.h"

extern "C" int nise_2dir(nise_ctx *c, double *R, int *sample_count) {
    (void)R;
    (void)sample_count;
    return nise_fail(c, NISE_ERR_UNSUPPORTED, "2DIR not available yet");
}

extern "C" int nise_propagate_doubles(nise_ctx *c, const float *H, void *re, void *im, int nvec, const float *anh) {
    (void)H; (void)re; (void)im; (void)nvec; (void)anh;
    return nise_fail(c, NISE_ERR_UNSUPPORTED, "doubles propagation not available yet");
}
