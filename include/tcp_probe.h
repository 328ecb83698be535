/*
 * tcp_probe.h -- measured arithmetic ceilings for the roofline of the MVP
 * kernels in `libtcpmvp.so`.
 *
 * The MVP kernels are bound by FP64 (complex128) or FP32 (complex64) FMA
 * issue and shared-memory operand delivery, not by HBM, so their roofline
 * needs the device's own FMA rate.  The probe runs independent FMA chains on
 * every SM (no memory traffic in the timed loop) and reports the best of
 * `repeats` timed launches.
 */
#ifndef TCP_PROBE_H
#define TCP_PROBE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* dtype: TCP_DTYPE_C128 (FP64 FMA) or TCP_DTYPE_C64 (FP32 FMA).  Writes the
 * achieved rate in flop/s (one FMA = 2 flops) and the best launch time. */
int tcp_probe_fma_rate(int dtype, uint32_t repeats, double *out_flops_per_s, double *out_ms);

#ifdef __cplusplus
}
#endif

#endif /* TCP_PROBE_H */
