/*
 * tcp_probe.h -- measured arithmetic ceilings for the roofline of the MVP
 * kernels in `libtcpmvp.so`.
 *
 * The MVP kernels are bound by shared-memory operand delivery and FP64
 * (complex128) or FP32 (complex64) FMA issue, not by HBM, so their roofline
 * needs the device's own shared-memory and FMA rates.  Each probe runs on
 * every SM with no global-memory traffic in its timed loop and reports the
 * best of `repeats` timed launches.
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

/* Shared-memory operand rate of the device: one CTA of 512 threads per SM
 * reads 16-byte values of a 64 KiB shared tile in the access pattern of the
 * tiled MVP kernels (XOR-permuted rows inside aligned 32-row blocks, 8 rows
 * per thread).  Writes bytes/s delivered to registers and the best launch
 * time out of `repeats`. */
int tcp_probe_smem_rate(uint32_t repeats, double *out_bytes_per_s, double *out_ms);

#ifdef __cplusplus
}
#endif

#endif /* TCP_PROBE_H */
