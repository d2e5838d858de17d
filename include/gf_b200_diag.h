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
 * 16 <= N <= 256.  swap != 0 exchanges the descriptor's two stride fields (used
 * by tests to show the layout encoding is the one the hardware expects).
 * Returns 0 on success. */
int gfx_umma_selftest(const float* A, const float* B, float* D, int N, int K, int split3, int swap);
#ifdef __cplusplus
}
#endif
#endif
