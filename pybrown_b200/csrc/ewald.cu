// RPY mobility tensors on sm_100a: free space (src/bdsim/clib/diff_tensor.c:73-166,
// :483-549) and under Smith's Ewald summation (diff_tensor.c:170-266, :553-1087).
//
// One CTA owns a 16 x 16 tile of bead pairs on or below the block diagonal.
// Bead coordinates, radii and the per-bead reciprocal-space phase factors of
// its two bead strips are staged in shared memory; each thread evaluates one
// pair block (real-space image sum + reciprocal sum) in registers, the 48 x 48
// value tile is assembled in shared memory and written out twice -- as tile
// (I, J) and as its transpose (J, I) -- with row-contiguous stores.
//
// Reciprocal space uses cos(2 pi n.(s_i - s_j)) = c_i c_j + s_i s_j with
// per-bead phase tables (c, s) = (cos, sin)(2 pi n.s_i), so the n-sum costs
// two FMAs per pair and n instead of one cosine, and the n <-> -n symmetry
// halves the n-set.  The minimum image does not enter the reciprocal part
// (the phase is periodic), only the real-space images.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace pbg {

namespace {

constexpr int TB = 16;           // beads per tile edge
constexpr int TV = 3 * TB;       // values per tile edge
constexpr int THREADS = TB * TB;

struct RpyArgs {
  PairSource src;
  const double* radii;
  const void* phase;    // [n_recip][n] of (c, s) pairs, T precision
  const double* real;   // [n_real][4]
  const double* recip;  // [n_recip][8]
  const float* recip_f;
  void* M;
  void* M_lower;        // or null: also receives the lower block triangle (tiles I >= J)
  double L, scale, alpha;
  double self_O[6], self_Q[6];
  int n, ld, smith, n_real, n_recip;
};

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

__device__ __forceinline__ double d_erfc(double x) { return erfc(x); }
__device__ __forceinline__ double d_exp(double x) { return exp(x); }
__device__ __forceinline__ double d_sqrt(double x) { return sqrt(x); }

// erfc(x) for x >= 0 in FP32 from e = exp(-x^2), by Abramowitz & Stegun,
// Handbook of Mathematical Functions, 7.1.26 (Hastings' rational
// approximation): erfc(x) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) e^{-x^2}
// with t = 1 / (1 + p x), absolute error below 1.5e-7 (a few FP32 ulps of
// erfc's values near 1).  The real-space Ewald sum needs exp(-x^2) anyway.
__device__ __forceinline__ float erfc_as(float x, float e) {
  const float t = __fdividef(1.0f, fmaf(0.3275911f, x, 1.0f));
  float p = 1.061405429f;
  p = fmaf(p, t, -1.453152027f);
  p = fmaf(p, t, 1.421413741f);
  p = fmaf(p, t, -0.284496736f);
  p = fmaf(p, t, 0.254829592f);
  return p * t * e;
}

// Free-space RPY pair block in FP64 (diff_tensor.c:490-549), three regimes.
__device__ void rpy_pair_fp64(double ai, double aj, double rx, double ry, double rz, double out[6]) {
  const double al = ai > aj ? ai : aj, as = ai > aj ? aj : ai;
  const double d2 = rx * rx + ry * ry + rz * rz, d = sqrt(d2), aij2 = ai * ai + aj * aj;
  double c1, cd, co;
  if (d > ai + aj) {
    c1 = 1.0 / (8 * PBG_PI * d);
    cd = 1.0 + aij2 / (3 * d2);
    co = (1.0 - aij2 / d2) / d2;
  } else if (d <= al - as) {
    c1 = 1.0 / (6 * PBG_PI * al);
    cd = 1.0;
    co = 0.0;
  } else {
    const double d3 = d2 * d;
    c1 = 1.0 / (6 * PBG_PI * ai * aj);
    double c3 = (ai - aj) * (ai - aj) + 3 * d2;
    c3 *= c3;
    cd = (16 * d3 * (ai + aj) - c3) / 32 / d3;
    double c5 = (ai - aj) * (ai - aj) - d2;
    c5 *= 3 * c5;
    co = c5 / (32 * d3) / d2;
  }
  out[0] = c1 * (cd + co * rx * rx);
  out[1] = c1 * (cd + co * ry * ry);
  out[2] = c1 * (cd + co * rz * rz);
  out[3] = c1 * co * rx * ry;
  out[4] = c1 * co * rx * rz;
  out[5] = c1 * co * ry * rz;
}

// Smith-Ewald pair block (diff_tensor.c:579-648) without the overlap fix:
// M = cO * O(sigma) + cQ * Q(sigma), cO = 1/(8 pi L), cQ = (ai^2+aj^2)/(24 pi L^3).
// Returns the 6 components as (outer_ab) + delta_ab * diag.
template <typename T>
__device__ __forceinline__ void smith_pair(T sx, T sy, T sz, T cO, T cQ, T alpha,
                                           const double* __restrict__ s_real, int n_real,
                                           const T* __restrict__ s_recip, int n_recip,
                                           const typename Vec2<T>::type* __restrict__ ph_i,
                                           const typename Vec2<T>::type* __restrict__ ph_j,
                                           int ph_stride, T acc[6], T& diag) {
  const T sqrt_pi = (T)1.7724538509055160273;
  const T alpha2 = alpha * alpha;
  const T o_real = (T)2 * alpha / sqrt_pi;
  const T q1 = (T)2 / sqrt_pi;
  const T q2 = (T)4 * alpha2 * alpha / sqrt_pi;
  T d = 0;
  // FP32: the image sum is compensated (Kahan): comp holds minus the
  // low-order bits lost so far; FP64 keeps the reference's plain summation.
  constexpr bool kahan = sizeof(T) == 4;
  T comp[7] = {0, 0, 0, 0, 0, 0, 0};
  auto add = [&](T& s, T& c, T v) {
    if constexpr (kahan) {
      const T yv = v - c;
      const T t = s + yv;
      c = (t - s) - yv;
      s = t;
    } else {
      s += v;
    }
  };
#pragma unroll 1
  for (int m = 0; m < n_real; ++m) {
    const T x = sx + (T)s_real[4 * m + 0];
    const T y = sy + (T)s_real[4 * m + 1];
    const T z = sz + (T)s_real[4 * m + 2];
    const T l2 = x * x + y * y + z * z;
    T l, il, ec, e, il2;
    if constexpr (sizeof(T) == 4) {
      // FP32: 1/l from the reciprocal square root, erfc from exp(-alpha^2 l^2)
      // (erfc_as), 1/l^2 = (1/l)^2
      asm("rsqrt.approx.f32 %0, %1;" : "=f"(il) : "f"(l2));
      l = l2 * il;
      e = __expf(-alpha2 * l2);
      ec = erfc_as(alpha * l, e);
      il2 = il * il;
    } else {
      l = d_sqrt(l2);
      il = (T)1 / l;
      ec = d_erfc(alpha * l);
      e = d_exp(-alpha2 * l2);
    }
    const T W = ec + q1 * alpha * l * e;
    const T il3 = il * il * il;
    add(d, comp[6], cO * ec * il + cQ * W * il3);
    const T num = cO * (ec * il + o_real * e) - cQ * ((T)3 * W * il3 + q2 * e);
    T oc;
    if constexpr (sizeof(T) == 4) oc = num * il2;
    else oc = num / l2;
    add(acc[0], comp[0], oc * x * x);
    add(acc[1], comp[1], oc * y * y);
    add(acc[2], comp[2], oc * z * z);
    add(acc[3], comp[3], oc * x * y);
    add(acc[4], comp[4], oc * x * z);
    add(acc[5], comp[5], oc * y * z);
  }
  if constexpr (kahan) {
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] -= comp[c];
    d -= comp[6];
  }
  T dr = 0;
#pragma unroll 2
  for (int k = 0; k < n_recip; ++k) {
    const T* r = s_recip + 8 * k;
    const typename Vec2<T>::type a = ph_i[k * ph_stride];
    const typename Vec2<T>::type b = ph_j[k * ph_stride];
    const T cs = a.x * b.x + a.y * b.y;
    dr += cs * r[3];
    const T g = cs * (cQ * r[5] - cO * r[4]);
    const T nx = r[0], ny = r[1], nz = r[2];
    acc[0] += g * nx * nx;
    acc[1] += g * ny * ny;
    acc[2] += g * nz * nz;
    acc[3] += g * nx * ny;
    acc[4] += g * nx * nz;
    acc[5] += g * ny * nz;
  }
  diag = d + cO * dr;
}

// One 16 x 16 bead tile (I, J), I >= J, of the tensor described by `a`.
template <typename T>
__device__ __forceinline__ void rpy_tile_body(const RpyArgs& a, int I, int J, void* M_lower) {
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // layout: out tile [TV][TV+1] T | recip table [n_recip][8] T | real [n_real][4] double |
  //         phases [n_recip][2*TB] V2
  T* s_out = reinterpret_cast<T*>(smem_raw);
  size_t off = sizeof(T) * TV * (TV + 1);
  off = (off + 15) & ~size_t(15);
  T* s_recip = reinterpret_cast<T*>(smem_raw + off);
  off += sizeof(T) * 8 * a.n_recip;
  off = (off + 15) & ~size_t(15);
  double* s_real = reinterpret_cast<double*>(smem_raw + off);
  off += sizeof(double) * 4 * a.n_real;
  off = (off + 15) & ~size_t(15);
  V2* s_ph = reinterpret_cast<V2*>(smem_raw + off);

  const int tid = threadIdx.x;
  const int ti = tid / TB, tj = tid % TB;
  const int i = I * TB + ti, j = J * TB + tj;
  const int n = a.n;

  if (a.smith) {
    const T* gsrc = sizeof(T) == 8 ? reinterpret_cast<const T*>(a.recip)
                                   : reinterpret_cast<const T*>(a.recip_f);
    for (int t = tid; t < 8 * a.n_recip; t += THREADS) s_recip[t] = gsrc[t];
    for (int t = tid; t < 4 * a.n_real; t += THREADS) s_real[t] = a.real[t];
    const V2* ph = reinterpret_cast<const V2*>(a.phase);
    for (int t = tid; t < a.n_recip * 2 * TB; t += THREADS) {
      const int k = t / (2 * TB), c = t % (2 * TB);
      const int bead = c < TB ? I * TB + c : J * TB + (c - TB);
      V2 v;
      v.x = 0; v.y = 0;
      if (bead < n) v = ph[(size_t)k * n + bead];
      s_ph[t] = v;
    }
  }
  __syncthreads();

  double blk[6] = {0, 0, 0, 0, 0, 0};
  bool active = (i < n) && (j < n) && !(I == J && ti < tj);
  if (active) {
    const double ai = a.radii[i], aj = a.radii[j];
    if (i == j) {
      // Self block (diff_tensor.c:553-575); the lattice sums are a-independent.
      const double c1 = 1.0 / (6 * PBG_PI * ai);
      if (a.smith) {
        const double sqrt_pi = 1.7724538509055160273;
        const double c2 = 3 * ai / (4 * a.L);
        const double c3 = ai * ai * ai / (2 * a.L * a.L * a.L);
        const double so = 1.5 * a.alpha * ai / (sqrt_pi * a.L);
        const double sq = a.alpha * a.alpha * a.alpha * ai * ai * ai / (a.L * a.L * a.L * 3.0 * sqrt_pi);
        for (int c = 0; c < 3; ++c)
          blk[c] = c1 * (1.0 + c2 * (a.self_O[c] - so) + c3 * (a.self_Q[c] - sq));
        for (int c = 3; c < 6; ++c) blk[c] = c1 * (c2 * a.self_O[c] + c3 * a.self_Q[c]);
      } else {
        blk[0] = blk[1] = blk[2] = c1;
      }
    } else {
      // Pair vector handed to the reference kernels: -minimg(r_i - r_j).
      double rx, ry, rz;
      get_pair_vector(a.src, i, j, rx, ry, rz);
      if (a.smith) {
        const double cO = 1.0 / (8 * PBG_PI * a.L);
        const double cQ = (ai * ai + aj * aj) / (24 * PBG_PI * a.L * a.L * a.L);
        T acc[6] = {0, 0, 0, 0, 0, 0};
        T dg;
        smith_pair<T>((T)(rx / a.L), (T)(ry / a.L), (T)(rz / a.L), (T)cO, (T)cQ, (T)a.alpha,
                      s_real, a.n_real, s_recip, a.n_recip, s_ph + ti, s_ph + TB + tj, 2 * TB,
                      acc, dg);
        for (int c = 0; c < 6; ++c) blk[c] = (double)acc[c];
        for (int c = 0; c < 3; ++c) blk[c] += (double)dg;
        const double d2 = rx * rx + ry * ry + rz * rz;
        if (d2 < (ai + aj) * (ai + aj)) {
          // Overlap fix (diff_tensor.c:614-643): swap far-field RPY for the
          // overlapping-regime RPY.
          double near[6], far[6];
          rpy_pair_fp64(ai, aj, rx, ry, rz, near);
          const double d = sqrt(d2), aij2 = ai * ai + aj * aj;
          const double f1 = 1.0 / (8 * PBG_PI * d), f2 = 1.0 + aij2 / (3 * d2);
          const double f3 = (1.0 - aij2 / d2) / d2;
          far[0] = f1 * (f2 + f3 * rx * rx);
          far[1] = f1 * (f2 + f3 * ry * ry);
          far[2] = f1 * (f2 + f3 * rz * rz);
          far[3] = f1 * f3 * rx * ry;
          far[4] = f1 * f3 * rx * rz;
          far[5] = f1 * f3 * ry * rz;
          for (int c = 0; c < 6; ++c) blk[c] += near[c] - far[c];
        }
      } else {
        rpy_pair_fp64(ai, aj, rx, ry, rz, blk);
      }
    }
    for (int c = 0; c < 6; ++c) blk[c] *= a.scale;
  }
  if (active) {
    const T v[6] = {(T)blk[0], (T)blk[1], (T)blk[2], (T)blk[3], (T)blk[4], (T)blk[5]};
    const int comp[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        s_out[(3 * ti + r) * (TV + 1) + 3 * tj + c] = v[comp[r][c]];
        if (I == J) s_out[(3 * tj + c) * (TV + 1) + 3 * ti + r] = v[comp[r][c]];
      }
  }
  __syncthreads();

  T* M = reinterpret_cast<T*>(a.M);
  const int n3 = 3 * n;
  const int row0 = 3 * I * TB, col0 = 3 * J * TB;
  T* ML = reinterpret_cast<T*>(M_lower);
  for (int t = tid; t < TV * TV; t += THREADS) {
    const int r = t / TV, c = t % TV;
    if (row0 + r < n3 && col0 + c < n3) {
      const T v = s_out[r * (TV + 1) + c];
      M[(size_t)(row0 + r) * a.ld + col0 + c] = v;
      if (ML) ML[(size_t)(row0 + r) * a.ld + col0 + c] = v;
    }
  }
  if (I != J) {
    for (int t = tid; t < TV * TV; t += THREADS) {
      const int r = t / TV, c = t % TV;  // output row col0 + r, column row0 + c
      if (col0 + r < n3 && row0 + c < n3) M[(size_t)(col0 + r) * a.ld + row0 + c] = s_out[c * (TV + 1) + r];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(THREADS) rpy_tile_kernel(RpyArgs a) {
  // Tile (I, J), I >= J, from the linear lower-triangle block index.
  const int b = blockIdx.x;
  int I = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= b) ++I;
  while (I * (I + 1) / 2 > b) --I;
  const int J = b - I * (I + 1) / 2;
  rpy_tile_body<T>(a, I, J, a.M_lower);
}

// Batched build: block b computes tile (work[b].y, work[b].z) of replica work[b].x;
// with fill_lower the lower block triangle also goes to the replica's M_lower.
template <typename T>
__global__ void __launch_bounds__(THREADS) rpy_batch_kernel(const RpyArgs* __restrict__ args,
                                                            const int4* __restrict__ work, int fill_lower) {
  const int4 w = work[blockIdx.x];
  rpy_tile_body<T>(args[w.x], w.y, w.z, fill_lower ? args[w.x].M_lower : nullptr);
}

__global__ void positions_from_pairs_kernel(const double* __restrict__ pairs, int n, double* __restrict__ pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i == 0) {
    pos[0] = pos[1] = pos[2] = 0.0;
    return;
  }
  const long long k = 3LL * (i - 1);  // pair (i, 0)
  pos[3 * i + 0] = -pairs[k];
  pos[3 * i + 1] = -pairs[k + 1];
  pos[3 * i + 2] = -pairs[k + 2];
}

// Per-bead phase factors (cos, sin)(2 pi n.s_i), s_i = r_i / L, layout [k][bead].
template <typename V2>
__global__ void phase_kernel(const double* __restrict__ pos, int n, double L,
                             const double* __restrict__ recip, int n_recip, V2* __restrict__ out) {
  const long long total = (long long)n * n_recip;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t / n), bead = (int)(t % n);
    const double* r = recip + 8 * k;
    const double ns = r[0] * (pos[3 * bead] / L) + r[1] * (pos[3 * bead + 1] / L) + r[2] * (pos[3 * bead + 2] / L);
    double s, c;
    sincospi(2.0 * ns, &s, &c);
    V2 v;
    v.x = c;
    v.y = s;
    out[(size_t)k * n + bead] = v;
  }
}

// Batched phase tables: blockIdx.y = replica, grid-stride over its (k, bead) entries.
template <typename V2>
__global__ void phase_batch_kernel(const RpyArgs* __restrict__ args, const double* __restrict__ recip,
                                   int n_recip) {
  const RpyArgs& a = args[blockIdx.y];
  const int n = a.n;
  const double L = a.L;
  const double* pos = a.src.pos;
  V2* out = reinterpret_cast<V2*>(const_cast<void*>(a.phase));
  const long long total = (long long)n * n_recip;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t / n), bead = (int)(t % n);
    const double* r = recip + 8 * k;
    const double ns = r[0] * (pos[3 * bead] / L) + r[1] * (pos[3 * bead + 1] / L) + r[2] * (pos[3 * bead + 2] / L);
    double sn, cs;
    sincospi(2.0 * ns, &sn, &cs);
    V2 v;
    v.x = cs;
    v.y = sn;
    out[(size_t)k * n + bead] = v;
  }
}

// ---------------------------------------------------------------- host side

// Self-block lattice sums (diff_tensor.c:652-849) without the a-dependent
// self terms, in the reference's loop order.
void host_self_sums(double alpha, int m_max, int n_max, double O[6], double Q[6]) {
  const double sqrt_pi = std::sqrt(PBG_PI), alpha2 = alpha * alpha, alpha3 = alpha * alpha2;
  const double kexp = -PBG_PI * PBG_PI / alpha2;
  for (int c = 0; c < 6; ++c) O[c] = Q[c] = 0.0;
  auto outer = [](double x, double y, double z, double v[6]) {
    v[0] = x * x; v[1] = y * y; v[2] = z * z; v[3] = x * y; v[4] = x * z; v[5] = y * z;
  };
  double mm[6];
  for (int mx = -m_max; mx <= m_max; ++mx)
    for (int my = -(m_max - std::abs(mx)); my <= m_max - std::abs(mx); ++my)
      for (int mz = -(m_max - std::abs(mx) - std::abs(my)); mz <= m_max - std::abs(mx) - std::abs(my); ++mz) {
        if (!mx && !my && !mz) continue;
        const double l2 = mx * mx + my * my + mz * mz, l = std::sqrt(l2), l3 = l2 * l;
        outer(mx, my, mz, mm);
        const double ec = std::erfc(alpha * l);
        const double e = std::exp(-alpha2 * l2);
        // O: erfc * O(m) + (2 alpha / sqrt(pi)) exp(-alpha^2 m^2) / m^2 * m m
        const double o_fn[6] = {(1 + mm[0] / l2) / l, (1 + mm[1] / l2) / l, (1 + mm[2] / l2) / l,
                                mm[3] / l3, mm[4] / l3, mm[5] / l3};
        const double w_o = 2 * alpha / sqrt_pi * e / l2;
        for (int c = 0; c < 6; ++c) O[c] += ec * o_fn[c] + w_o * mm[c];
        // Q: (erfc + 2/sqrt(pi) alpha m e) * Q(m) - 4 alpha^3/sqrt(pi) e / m^2 * m m
        const double am = alpha * l, l5 = l3 * l2;
        const double q_fn[6] = {(1 - 3 * mm[0] / l2) / l3, (1 - 3 * mm[1] / l2) / l3, (1 - 3 * mm[2] / l2) / l3,
                                -3 * mm[3] / l5, -3 * mm[4] / l5, -3 * mm[5] / l5};
        const double w_q1 = std::erfc(am) + 2 / sqrt_pi * am * e;
        const double w_q2 = 2 / sqrt_pi * 2 * alpha3 * e / l2;
        for (int c = 0; c < 6; ++c) Q[c] += w_q1 * q_fn[c] - w_q2 * mm[c];
      }
  for (int nx = -n_max; nx <= n_max; ++nx)
    for (int ny = -(n_max - std::abs(nx)); ny <= n_max - std::abs(nx); ++ny)
      for (int nz = -(n_max - std::abs(nx) - std::abs(ny)); nz <= n_max - std::abs(nx) - std::abs(ny); ++nz) {
        if (!nx && !ny && !nz) continue;
        const double nl2 = nx * nx + ny * ny + nz * nz;
        outer(nx, ny, nz, mm);
        const double w = 2.0 / PBG_PI / nl2 * std::exp(kexp * nl2);
        const double t = 1.0 / nl2 - kexp;
        for (int c = 0; c < 3; ++c) O[c] += w * (1.0 - t * mm[c]);
        for (int c = 3; c < 6; ++c) O[c] += w * (-t * mm[c]);
        const double wq = 4 * PBG_PI * std::exp(kexp * nl2) / nl2;
        for (int c = 0; c < 6; ++c) Q[c] += wq * mm[c];
      }
}

std::mutex g_tables_mu;
std::map<std::tuple<double, int, int>, EwaldTables*> g_tables;

}  // namespace

long long lattice_points_l1(int m) {
  // integer points with |x| + |y| + |z| <= m: (2m + 1)(2m^2 + 2m + 3) / 3
  const long long mm = m;
  return (2 * mm + 1) * (2 * mm * mm + 2 * mm + 3) / 3;
}

void build_lattice_tables(double alpha, int m_max, int n_max, std::vector<double>& real,
                          std::vector<double>& recip, double self_O[6], double self_Q[6]) {
  real.clear();
  recip.clear();
  for (int mx = -m_max; mx <= m_max; ++mx)
    for (int my = -(m_max - std::abs(mx)); my <= m_max - std::abs(mx); ++my)
      for (int mz = -(m_max - std::abs(mx) - std::abs(my)); mz <= m_max - std::abs(mx) - std::abs(my); ++mz) {
        real.push_back(mx); real.push_back(my); real.push_back(mz); real.push_back(0);
      }
  const double kk = PBG_PI * PBG_PI / (alpha * alpha);
  for (int nx = -n_max; nx <= n_max; ++nx)
    for (int ny = -(n_max - std::abs(nx)); ny <= n_max - std::abs(nx); ++ny)
      for (int nz = -(n_max - std::abs(nx) - std::abs(ny)); nz <= n_max - std::abs(nx) - std::abs(ny); ++nz) {
        // keep the half with the first non-zero component positive; weights x2
        const bool keep = nx > 0 || (nx == 0 && ny > 0) || (nx == 0 && ny == 0 && nz > 0);
        if (!keep) continue;
        const double nl2 = nx * nx + ny * ny + nz * nz;
        const double e = std::exp(-kk * nl2);
        const double P = 2.0 * (2.0 / PBG_PI) / nl2 * e;  // O weight
        const double R = P * (1.0 + kk * nl2) / nl2;       // O weight * t
        const double S = 2.0 * 4 * PBG_PI * e / nl2;       // Q weight
        const double row[8] = {(double)nx, (double)ny, (double)nz, P, R, S, 0, 0};
        recip.insert(recip.end(), row, row + 8);
      }
  host_self_sums(alpha, m_max, n_max, self_O, self_Q);
}

int get_ewald_tables(double alpha, int m_max, int n_max, const EwaldTables** out) {
  if (m_max < 0 || n_max < 0 || m_max > 16 || n_max > 16 || !(alpha > 0)) {
    pbg_set_error_message("invalid Ewald parameters alpha=%g m_max=%d n_max=%d", alpha, m_max, n_max);
    return PBG_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_tables_mu);
  auto key = std::make_tuple(alpha, m_max, n_max);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    *out = it->second;
    return PBG_OK;
  }
  auto* t = new EwaldTables();
  t->alpha = alpha;
  t->m_max = m_max;
  t->n_max = n_max;
  std::vector<double> real, recip;
  build_lattice_tables(alpha, m_max, n_max, real, recip, t->self_O, t->self_Q);
  t->n_real = (int)real.size() / 4;
  t->n_recip = (int)recip.size() / 8;
  std::vector<float> recip_f(recip.begin(), recip.end());
  if (cudaMalloc(&t->d_real, real.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&t->d_recip, std::max<size_t>(recip.size(), 8) * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&t->d_recip_f, std::max<size_t>(recip.size(), 8) * sizeof(float)) != cudaSuccess) {
    pbg_set_error_message("cudaMalloc failed for Ewald tables");
    return PBG_ERR_NOMEM;
  }
  PBG_CUDA_TRY(cudaMemcpy(t->d_real, real.data(), real.size() * sizeof(double), cudaMemcpyHostToDevice));
  if (!recip.empty()) {
    PBG_CUDA_TRY(cudaMemcpy(t->d_recip, recip.data(), recip.size() * sizeof(double), cudaMemcpyHostToDevice));
    PBG_CUDA_TRY(cudaMemcpy(t->d_recip_f, recip_f.data(), recip_f.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  g_tables[key] = t;
  *out = t;
  return PBG_OK;
}

int launch_positions_from_pairs(const double* pairs, int n, double* pos, cudaStream_t st) {
  if (n <= 0) return PBG_OK;
  positions_from_pairs_kernel<<<(n + 127) / 128, 128, 0, st>>>(pairs, n, pos);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

size_t phase_scratch_bytes(int n, const EwaldTables* t, int precision) {
  if (!t) return 0;
  const size_t elem = precision == PBG_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  return (size_t)n * t->n_recip * elem;
}

static size_t rpy_smem_bytes(const EwaldTables* t, int precision, bool smith) {
  const size_t ts = precision == PBG_PREC_FP64 ? 8 : 4;
  size_t off = ts * TV * (TV + 1);
  off = (off + 15) & ~size_t(15);
  if (!smith) return off;
  off += ts * 8 * t->n_recip;
  off = (off + 15) & ~size_t(15);
  off += sizeof(double) * 4 * t->n_real;
  off = (off + 15) & ~size_t(15);
  off += 2 * ts * (size_t)t->n_recip * 2 * TB;
  return off;
}

int launch_rpy_tensor(const PairSource& src, const double* pos, const double* radii, bool smith,
                      const EwaldTables* t, double scale, int precision, void* M, int ld,
                      void* phase, cudaStream_t st, void* M_lower) {
  const int n = src.n;
  const double L = src.L;
  if (n <= 0) return PBG_OK;
  if (smith && !t) return PBG_ERR_ARG;
  RpyArgs a{};
  a.src = src;
  a.radii = radii;
  a.M = M;
  a.M_lower = M_lower;
  a.L = L;
  a.scale = scale;
  a.n = n;
  a.ld = ld;
  a.smith = smith ? 1 : 0;
  if (smith) {
    a.alpha = t->alpha;
    a.real = t->d_real;
    a.recip = t->d_recip;
    a.recip_f = t->d_recip_f;
    a.n_real = t->n_real;
    a.n_recip = t->n_recip;
    for (int c = 0; c < 6; ++c) {
      a.self_O[c] = t->self_O[c];
      a.self_Q[c] = t->self_Q[c];
    }
    a.phase = phase;
    if (t->n_recip > 0) {
      const long long total = (long long)n * t->n_recip;
      const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
      if (precision == PBG_PREC_FP64)
        phase_kernel<double2><<<blocks, 256, 0, st>>>(pos, n, L, t->d_recip, t->n_recip, (double2*)phase);
      else
        phase_kernel<float2><<<blocks, 256, 0, st>>>(pos, n, L, t->d_recip, t->n_recip, (float2*)phase);
      PBG_CHECK_LAUNCH();
    }
  }
  const int tiles = (n + TB - 1) / TB;
  const int blocks = tiles * (tiles + 1) / 2;
  const size_t smem = rpy_smem_bytes(t, precision, smith);
  if (smem > 227 * 1024) {
    pbg_set_error_message("Ewald n-set too large for shared memory (%zu bytes)", smem);
    return PBG_ERR_ARG;
  }
  if (precision == PBG_PREC_FP64) {
    PBG_CUDA_TRY(cudaFuncSetAttribute(rpy_tile_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    rpy_tile_kernel<double><<<blocks, THREADS, smem, st>>>(a);
  } else {
    PBG_CUDA_TRY(cudaFuncSetAttribute(rpy_tile_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    rpy_tile_kernel<float><<<blocks, THREADS, smem, st>>>(a);
  }
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

size_t rpy_batch_arg_bytes() { return sizeof(RpyArgs); }

void rpy_batch_arg(const double* pos, const double* radii, int n, double L, bool smith, const EwaldTables* t,
                   double scale, void* M, void* M_lower, int ld, void* phase, void* dst) {
  RpyArgs a{};
  a.src.pos = pos;
  a.src.pairs = nullptr;
  a.src.n = n;
  a.src.L = L;
  a.radii = radii;
  a.M = M;
  a.M_lower = M_lower;
  a.L = L;
  a.scale = scale;
  a.n = n;
  a.ld = ld;
  a.smith = smith ? 1 : 0;
  if (smith && t) {
    a.alpha = t->alpha;
    a.real = t->d_real;
    a.recip = t->d_recip;
    a.recip_f = t->d_recip_f;
    a.n_real = t->n_real;
    a.n_recip = t->n_recip;
    for (int c = 0; c < 6; ++c) {
      a.self_O[c] = t->self_O[c];
      a.self_Q[c] = t->self_Q[c];
    }
    a.phase = phase;
  }
  std::memcpy(dst, &a, sizeof(a));
}

void rpy_batch_work(int replica, int n, std::vector<int4>& work) {
  const int tiles = (n + TB - 1) / TB;
  for (int I = 0; I < tiles; ++I)
    for (int J = 0; J <= I; ++J) work.push_back(make_int4(replica, I, J, 0));
}

// args: device array of the replicas' argument blocks (rpy_batch_arg);
// the phase tables are built first (one grid row per replica).  fill_lower:
// each replica's lower block triangle also goes to its M_lower (the matrix
// the step factors next).
int launch_rpy_batch(int precision, bool smith, const EwaldTables* t, const void* args, const int4* work,
                     int nwork, int n_replicas, bool fill_lower, cudaStream_t st) {
  if (nwork <= 0) return PBG_OK;
  const RpyArgs* a = static_cast<const RpyArgs*>(args);
  if (smith && t && t->n_recip > 0 && n_replicas > 0) {
    const dim3 grid(16, n_replicas);
    if (precision == PBG_PREC_FP64) phase_batch_kernel<double2><<<grid, 256, 0, st>>>(a, t->d_recip, t->n_recip);
    else phase_batch_kernel<float2><<<grid, 256, 0, st>>>(a, t->d_recip, t->n_recip);
    PBG_CHECK_LAUNCH();
  }
  const size_t smem = rpy_smem_bytes(t, precision, smith);
  if (smem > 227 * 1024) {
    pbg_set_error_message("Ewald n-set too large for shared memory (%zu bytes)", smem);
    return PBG_ERR_ARG;
  }
  if (precision == PBG_PREC_FP64) {
    PBG_CUDA_TRY(cudaFuncSetAttribute(rpy_batch_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    rpy_batch_kernel<double><<<nwork, THREADS, smem, st>>>(a, work, fill_lower ? 1 : 0);
  } else {
    PBG_CUDA_TRY(cudaFuncSetAttribute(rpy_batch_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    rpy_batch_kernel<float><<<nwork, THREADS, smem, st>>>(a, work, fill_lower ? 1 : 0);
  }
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
