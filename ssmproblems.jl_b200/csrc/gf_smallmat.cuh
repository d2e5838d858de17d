// gf_smallmat.cuh -- block-wide FP64 helpers on small dense matrices held in
// shared memory (column-major, column stride LD = 16, so dimensions up to 16):
// products, matrix-vector products, symmetrisation, and a Cholesky factor with
// the inverse.  Every helper is called by all threads of the block and ends
// with a barrier.
#pragma once
#include <cuda_runtime.h>

namespace gf {
namespace {

constexpr int SM_MAXD = 16;
constexpr int LD = SM_MAXD;  // column stride of every shared matrix

// C (m x n) = alpha op(A) op(B) + beta C on LD-strided shared matrices; C must
// not alias A or B.  Ends with a barrier.
__device__ void mm(double* C, const double* A, bool tA, const double* B, bool tB, int m, int k, int n,
                   double alpha, double beta) {
  for (int e = threadIdx.x; e < m * n; e += blockDim.x) {
    const int i = e % m, j = e / m;
    double s = 0.0;
    for (int p = 0; p < k; ++p) s += (tA ? A[p + i * LD] : A[i + p * LD]) * (tB ? B[j + p * LD] : B[p + j * LD]);
    C[i + j * LD] = alpha * s + (beta != 0.0 ? beta * C[i + j * LD] : 0.0);
  }
  __syncthreads();
}

// y (m) = op(A) x
__device__ void mv(double* y, const double* A, bool tA, const double* x, int m, int k) {
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < k; ++p) s += (tA ? A[p + i * LD] : A[i + p * LD]) * x[p];
    y[i] = s;
  }
  __syncthreads();
}

__device__ void symmetrize(double* M, int n) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    if (i < j) {
      const double v = 0.5 * (M[i + j * LD] + M[j + i * LD]);
      M[i + j * LD] = v;
      M[j + i * LD] = v;
    }
  }
  __syncthreads();
}

// Cholesky of S (n x n) into L, S^{-1} into Si and log det S; false if S is
// not positive definite.  Column by column: one thread takes the pivot, the
// block fills the column below it.
__device__ bool chol_inv(const double* S, double* L, double* Si, int n, double* logdet, int* s_ok) {
  if (threadIdx.x == 0) {
    *s_ok = 1;
    *logdet = 0.0;
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (threadIdx.x == 0) {
      double d = S[j + j * LD];
      for (int p = 0; p < j; ++p) d -= L[j + p * LD] * L[j + p * LD];
      if (d > 0.0) {
        L[j + j * LD] = sqrt(d);
        *logdet += log(d);
      } else {
        *s_ok = 0;
        L[j + j * LD] = 1.0;  // keeps the column fill finite; the result is discarded
      }
    }
    __syncthreads();
    const double ljj = L[j + j * LD];
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double s = S[i + j * LD];
      for (int p = 0; p < j; ++p) s -= L[i + p * LD] * L[j + p * LD];
      L[i + j * LD] = s / ljj;
    }
    __syncthreads();
  }
  if (!*s_ok) return false;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {  // column j of S^{-1}
    double w[SM_MAXD];
    for (int i = 0; i < n; ++i) {
      double s = i == j ? 1.0 : 0.0;
      for (int p = 0; p < i; ++p) s -= L[i + p * LD] * w[p];
      w[i] = s / L[i + i * LD];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = w[i];
      for (int p = i + 1; p < n; ++p) s -= L[p + i * LD] * w[p];
      w[i] = s / L[i + i * LD];
    }
    for (int i = 0; i < n; ++i) Si[i + j * LD] = w[i];
  }
  __syncthreads();
  return true;
}

}  // namespace
}  // namespace gf
