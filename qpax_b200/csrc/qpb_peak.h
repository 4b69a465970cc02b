/*
 * qpb_peak.h -- measurement helper of libqpb_peak.so, a library of its own
 * that only the benchmark loads (no counterpart in qpax: it puts the solver's
 * FP32/FP64 arithmetic next to the throughput the GPU can deliver).
 */
#ifndef QPB_PEAK_H_
#define QPB_PEAK_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Runs a fused-multiply-add throughput kernel (independent FMA chains in
 * every thread of a full grid) on `stream` and returns the achieved
 * TFLOP/s (FMA = 2 FLOPs), or a negative value on a CUDA error.
 * precision 0 = FP32, 1 = FP64.  `scratch` is a device buffer of at least
 * 4 MiB that receives the chain results.  Synchronizes the stream. */
double qpb_bench_fma_peak(int precision, void* scratch, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QPB_PEAK_H_ */
