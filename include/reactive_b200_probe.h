/* Measurement helper exported by libreactive_b200.so (no reference counterpart:
 * the reference records no FP64 peak). Launches a kernel of independent FP64
 * FMA chains on `stream` (not synchronised); flopsPerLaunch receives its FLOP
 * count so the caller can time it with CUDA events. scratch: >= blocks doubles. */
#ifndef REACTIVE_B200_PROBE_H
#define REACTIVE_B200_PROBE_H
#ifdef __cplusplus
extern "C" {
#endif
int rb200_probe_fp64_fma_v1(int blocks, int threads, int iterations, double* scratch, void* stream,
                            double* flopsPerLaunch);
#ifdef __cplusplus
}
#endif
#endif
