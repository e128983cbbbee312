// Shared definitions for the pybrown_b200 sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "pybrown_b200.h"

#define PBG_PI 3.14159265358979323846

// Record a CUDA error as a status code (no aborts, no device traps).
#define PBG_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      pbg_record_cuda_error(_e, #expr, __FILE__, __LINE__);                       \
      return PBG_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

// Every kernel launch of the library is followed by this check, which also
// counts the launch (pbg_launch_count()).
#define PBG_CHECK_LAUNCH()                                                        \
  do {                                                                            \
    cudaError_t _e = cudaGetLastError();                                          \
    if (_e != cudaSuccess) {                                                      \
      pbg_record_cuda_error(_e, "kernel launch", __FILE__, __LINE__);             \
      return PBG_ERR_CUDA;                                                        \
    }                                                                             \
    pbg_count_launch();                                                           \
  } while (0)

void pbg_record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void pbg_set_error_message(const char* fmt, ...);
void pbg_count_launch();
// Adds n launches (kernels replayed inside a CUDA graph; negative to take
// back the launches a stream capture counted without running them).
void pbg_count_launches(long long n);
// Adds n host launch calls (+1 per graph launch; negative to take back the
// kernel launches a stream capture counted).
void pbg_count_host_calls(long long n);

// Device-side error bits (written with atomicOr into a status word).
enum : unsigned {
  PBG_DEV_ERR_NONE = 0u,
  PBG_DEV_ERR_NOT_SPD = 1u,        // non-positive pivot in a Cholesky factorisation
  PBG_DEV_ERR_BARRIER = 2u,        // a bounded grid barrier gave up
  PBG_DEV_ERR_ATTEMPTS = 4u,       // max_move_attempts reached
  PBG_DEV_ERR_NOISE = 8u,          // the noise pool ran out
  PBG_DEV_ERR_NAN = 16u,           // non-finite value met
};

// Matrices are row-major with a padded leading dimension; the order is
// padded to a multiple of PBG_TILE and the padding is an identity block so
// that every tiled factorisation runs without bounds checks.
#ifndef PBG_TILE
#define PBG_TILE 64
#endif

static inline int pbg_round_up(int x, int m) { return (x + m - 1) / m * m; }

// Minimum-image shift with the reference's while-loop semantics
// (src/bdsim/clib/bead.c:44-73): pull down while x >= L/2, then push up while
// x <= -L/2.  A single subtraction/addition suffices for |x| < 1.5 L, which
// covers positions kept inside the box; larger inputs loop a bounded number
// of times (the bound only protects against non-finite input).
__host__ __device__ inline double pbg_min_image(double x, double L) {
  const double h = L / 2.0;
  int guard = 0;
  while (x >= h && guard < 64) { x -= L; ++guard; }
  while (x <= -h && guard < 128) { x += L; ++guard; }
  return x;
}

// keep_in_box (src/bdsim/pyBrown/bead.py:170-183): [-L/2, L/2).
__host__ __device__ inline double pbg_wrap(double x, double L) {
  int guard = 0;
  while (x < -L / 2 && guard < 64) { x += L; ++guard; }
  while (x >= L / 2 && guard < 128) { x -= L; ++guard; }
  return x;
}
