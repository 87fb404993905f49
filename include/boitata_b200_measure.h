/* boitata_b200 measurement hooks: bench and profiling tooling, not part of
 * the kriging call surface (no counterpart in the reference). They take a
 * context of include/boitata_b200.h.
 *
 * btk_set_timing records CUDA events around the phases of every prediction
 * on this context; btk_phase_ms waits for the last one and gives its search,
 * solve and FP64 re-solve times in milliseconds. btk_peak_flops runs a
 * CUDA-core FMA loop and returns the FLOP/s reached (fp64 != 0: double, else
 * float), the denominator of the solve kernels' roofline. */
#ifndef BOITATA_B200_MEASURE_H
#define BOITATA_B200_MEASURE_H

#include <stdint.h>

#include "boitata_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

int btk_set_timing(btk_ctx* ctx, int32_t on);
int btk_phase_ms(btk_ctx* ctx, float* out3);
double btk_peak_flops(btk_ctx* ctx, int32_t fp64);

#ifdef __cplusplus
}
#endif
#endif /* BOITATA_B200_MEASURE_H */
