/*
 * tb_probe.h -- C ABI of libtb_probe.so, measurement and test helpers that
 * are not part of libtraceon_b200.so.  No reference counterpart.
 */
#ifndef TB_PROBE_H
#define TB_PROBE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *tb_probe_stream_t;

/* `blocks` x 256 threads each run `iters` x 8 independent FP64 FMAs (16
 * flops per thread-iteration): the FP64 pipe peak that the FP64-bound
 * kernels are compared against.  Returns 0 on success. */
int tb_probe_fp64_fma(int blocks, int64_t iters, double *out, tb_probe_stream_t stream);

/* out[i] = f(x[i]) on the device for the branch-free functions of the
 * ring-pair loops (fn 0: 1/x, 1: 1/sqrt(x), 2: log x) and, for comparison,
 * the CUDA library forms (fn 10, 11, 12).  Returns 0 on success. */
int tb_probe_math(const double *x, int64_t n, int fn, double *out, tb_probe_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* TB_PROBE_H */
