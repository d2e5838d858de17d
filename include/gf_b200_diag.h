/*
 * gf_b200_diag.h -- diagnostic entry points of libgfb200.so (not part of the
 * filtering API; no reference counterpart).
 */
#ifndef GF_B200_DIAG_H
#define GF_B200_DIAG_H
#ifdef __cplusplus
extern "C" {
#endif
/* D = A * B^T for one 128-row tile on the tcgen05 tensor cores (kind::tf32;
 * split3 != 0 uses the 3xTF32 split for FP32-level accuracy).  A [128 x K],
 * B [N x K], D [128 x N] row-major FP32 host arrays; K % 8 == 0, N % 16 == 0,
 * 16 <= N <= 256.  Returns 0 on success. */
int gfx_umma_selftest(const float* A, const float* B, float* D, int N, int K, int split3);
/* Runs one of the library's bounded device waits against a flag that is
 * published beforehand (publish != 0) or never set, polling at most `limit`
 * times: which = 0 is the decoupled lookback of the cumulative-weight scan
 * (tile 1 of two; tile 0's inclusive prefix is 5 when published, *excl_out
 * receives the exclusive prefix), which = 1 the tensor-core propagate's
 * mbarrier wait (one arrival expected).  *status_out receives GF_OK or
 * GF_ERR_TIMEOUT, the status the waiting kernel records.  Returns GF_OK when
 * the kernel ran. */
int gfx_wait_selftest(int which, int publish, long long limit, int* status_out,
                      unsigned long long* excl_out);
#ifdef __cplusplus
}
#endif
#endif
