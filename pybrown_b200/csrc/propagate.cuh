// Launchers of the position-update kernels (propagate.cu).
#pragma once

#include "common.cuh"

namespace pbg {

int launch_gemv_scaled(const void* A, int ld, int n, int precision, const double* x, double c,
                       double* y, cudaStream_t st);
int launch_gemv_diff(const void* A, const void* A0, int ld, int n, int precision, const double* x,
                     double c, double* y, cudaStream_t st);
int launch_trmv_lower(const void* B, int ld, int n, int precision, const double* x, double* y,
                      cudaStream_t st);
int launch_scale2(const double* in, double s1, double s2, int n, double* out, cudaStream_t st);
int launch_translate(double* pos, const double* v, int n, bool negate, cudaStream_t st);
int launch_wrap(double* pos, int n3, double L, cudaStream_t st);
int launch_drift_combine(const double* Dy, const double* Bxi, const double* ddet, double c2, int n,
                         double* drift, cudaStream_t st);
// Solves B^T y = rhs (B lower, order ld, padded); invdiag are the inverted
// diagonal tiles left by the Cholesky workspace; rhs, r_work, y have ld entries.
int launch_trsv_upper(const void* B, int ld, int precision, const void* invdiag, const double* rhs,
                      double* r_work, double* y, cudaStream_t st);

}  // namespace pbg
