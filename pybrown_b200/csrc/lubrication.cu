// Jeffrey-Onishi lubrication correction of the resistance matrix on sm_100a
// (src/bdsim/clib/diff_tensor.c:270-479, :1091-1625).
//
// For every pair with (r - ai - aj)/(ai + aj) <= cutoff the correction is
// P(R_JO) - P(R_RPY2B): the Jeffrey-Onishi two-body resistance minus the
// inverse of the two-bead free-space RPY mobility, P being the optional
// Cichocki projection.  Every 3x3 block involved has the form
// X r^r^ + Y (1 - r^r^), so all pair work is done on (X, Y) scalar pairs:
// the 6x6 LAPACK inverse of the reference (diff_tensor.c:1629-1641) becomes
// a closed-form 2x2 inverse per longitudinal/transverse direction.
//
// Scatter without atomics: the off-diagonal block (i, j) belongs to exactly
// one pair, so one thread per pair adds it; the diagonal block of bead b is
// summed by one warp per bead over its partners in increasing partner index,
// which is the addition order of the reference's double loop.
#include "common.cuh"
#include "kernels.cuh"

namespace pbg {

namespace {

// Jeffrey & Onishi (1984) f_m(l) coefficients by power of l (diff_tensor.c:1385-1545).
__constant__ double c_XF[12][11] = {
    {1},
    {0, 3},
    {0, 9},
    {0, -4, 27, -4},
    {0, -24, 81, 36},
    {0, 0, 72, 243, 72},
    {0, 16, 108, 281, 648, 144},
    {0, 0, 288, 1620, 1515, 1620, 288},
    {0, 0, 576, 4848, 5409, 4524, 3888, 576},
    {0, 0, 1152, 9072, 14752, 26163, 14752, 9072, 1152},
    {0, 0, 2304, 20736, 42804, 115849, 76176, 39264, 20736, 2304},
    {0, 0, 4608, 46656, 108912, 269100, 319899, 269100, 108912, 46656, 4608},
};
__constant__ double c_YF[12][11] = {
    {1},
    {0, 1.5},
    {0, 2.25},
    {0, 2, 3.375, 2},
    {0, 6, 5.0625, 18},
    {0, 0, 31.5, 7.59375, 31.5},
    {0, 4, 54, 19.390625, 81, 72},
    {0, 0, 144, 131.625, 149.0859375, 131.625, 144},
    {0, 0, 279, 532.625, 493.62890625, -14.625, 648, 288},
    {0, 0, 576, 1134, 1888.84375, 1496.443359375, 1888.84375, 1134, 576},
    {0, 0, 1152, 1964.25, 6155.4375, 10301.1650390625, 8452.125, -175.5, 3888, 1152},
    {0, 0, 2304, 7128, 11035.5, 21441.4453125, 46486.24755859375, 21441.4453125, 11035.5, 7128, 2304},
};

__device__ double poly11(const double* c, double l) {
  double s = 0.0, p = 1.0;
#pragma unroll
  for (int k = 0; k < 11; ++k) {
    s += c[k] * p;
    p *= l;
  }
  return s;
}

__device__ __forceinline__ double Xg(double l, int k) {
  const double l2 = l * l, p3 = (1 + l) * (1 + l) * (1 + l);
  if (k == 1) return 2 * l2 / p3;
  if (k == 2) return 0.2 * l * (1 + 7 * l + l2) / p3;
  return 1.0 / 42 * (1 + 18 * l - 29 * l2 + 18 * l2 * l + l2 * l2) / p3;
}

__device__ __forceinline__ double Yg(double l, int k) {
  const double l2 = l * l, p3 = (1 + l) * (1 + l) * (1 + l);
  if (k == 2) return 4.0 / 15 * l * (2 + l + 2 * l2) / p3;
  return 2.0 / 375 * (16 - 45 * l + 58 * l2 - 45 * l2 * l + 16 * l2 * l2) / p3;
}

// A11 (m even, diff_tensor.c:1190-1284) and A12 (m odd, :1288-1381) series.
// X selects the X (longitudinal) or Y (transverse) function family.
__device__ double A11(double s, double l, bool X) {
  const double s2 = 1.0 - 4.0 / (s * s), lg = log(s2);
  const double g1 = X ? Xg(l, 1) : 0.0, g2 = X ? Xg(l, 2) : Yg(l, 2), g3 = X ? Xg(l, 3) : Yg(l, 3);
  double v = 0.0;
  if (X) v += g1 / s2;
  v -= g2 * lg;
  v -= g3 * s2 * lg;
  v += 1.0 - g1;  // f_0 = 1
  const double q = 2.0 / s, ql = 1.0 / (2.0 * (1.0 + l));
  double w = 1.0, wl = 1.0;
  for (int m = 1; m <= 10; ++m) {
    w *= q;
    wl *= ql;
    if (m & 1) continue;
    const int m1 = (m == 2) ? -2 : m - 2;
    const double f = poly11(X ? c_XF[m] : c_YF[m], l);
    v += w * (wl * f - g1 - 2.0 / m * g2);
    v += w * (4.0 / (m * m1) * g3);
  }
  return v;
}

__device__ double A12(double s, double l, bool X) {
  const double s2 = 1.0 - 4.0 / (s * s), lg = log((s + 2) / (s - 2));
  const double g1 = X ? Xg(l, 1) : 0.0, g2 = X ? Xg(l, 2) : Yg(l, 2), g3 = X ? Xg(l, 3) : Yg(l, 3);
  double v = 0.0;
  if (X) v += 2.0 / s * g1 / s2;
  v += g2 * lg;
  v += g3 * s2 * lg;
  v += 4 * g3 / s;
  const double q = 2.0 / s, ql = 1.0 / (2.0 * (1.0 + l));
  double w = 1.0, wl = 1.0;
  for (int m = 1; m <= 11; ++m) {
    w *= q;
    wl *= ql;
    if (!(m & 1)) continue;
    const int m1 = m - 2;
    const double f = poly11(X ? c_XF[m] : c_YF[m], l);
    v += w * (wl * f - g1 - 2.0 / m * g2);
    v += w * (4.0 / (m * m1) * g3);
  }
  return -v;
}

// Scalars of a two-bead resistance in the (longitudinal, transverse) basis:
// blocks 11, 22 and 12 are each X r^r^ + Y (1 - r^r^).
struct TwoBody {
  double x11, y11, x22, y22, x12, y12;
};

// diff_tensor.c:270-342 with a = first bead, b = second bead.
__device__ TwoBody jo_two_body(double a, double b, double d) {
  const double s = 2 * d / (a + b), l = b / a, il = 1 / l;
  TwoBody t;
  t.x11 = A11(s, l, true);
  t.y11 = A11(s, l, false);
  t.x22 = l * A11(s, il, true);
  t.y22 = l * A11(s, il, false);
  t.x12 = A12(s, l, true);
  t.y12 = A12(s, l, false);
  const double mult = 6 * PBG_PI * a;
  t.x11 *= mult; t.y11 *= mult; t.x22 *= mult; t.y22 *= mult; t.x12 *= mult; t.y12 *= mult;
  return t;
}

// Inverse of [[I/(6 pi a), C], [C, I/(6 pi b)]] with C the RPY pair block
// (diff_tensor.c:1091-1162): closed-form per direction.
__device__ TwoBody rpy_two_body_resistance(double a, double b, double d) {
  const double al = a > b ? a : b, as = a > b ? b : a;
  const double d2 = d * d, aij2 = a * a + b * b;
  double cT, cL;
  if (d > a + b) {
    const double c1 = 1.0 / (8 * PBG_PI * d);
    const double c2 = 1.0 + aij2 / (3 * d2);
    const double c3 = (1.0 - aij2 / d2) / d2;
    cT = c1 * c2;
    cL = c1 * (c2 + c3 * d2);
  } else if (d <= al - as) {
    cT = cL = 1.0 / (6 * PBG_PI * al);
  } else {
    const double d3 = d2 * d;
    const double c1 = 1.0 / (6 * PBG_PI * a * b);
    double c3 = (a - b) * (a - b) + 3 * d2;
    c3 *= c3;
    const double c4 = (16 * d3 * (a + b) - c3) / 32 / d3;
    double c5 = (a - b) * (a - b) - d2;
    c5 *= 3 * c5;
    const double c6 = c5 / (32 * d3) / d2;
    cT = c1 * c4;
    cL = c1 * (c4 + c6 * d2);
  }
  const double ma = 1.0 / (6 * PBG_PI * a), mb = 1.0 / (6 * PBG_PI * b);
  const double detL = ma * mb - cL * cL, detT = ma * mb - cT * cT;
  TwoBody t;
  t.x11 = mb / detL; t.y11 = mb / detT;
  t.x22 = ma / detL; t.y22 = ma / detT;
  t.x12 = -cL / detL; t.y12 = -cT / detT;
  return t;
}

__device__ __forceinline__ TwoBody cichocki(const TwoBody& t) {
  // diff_tensor.c:1166-1186: every self block -> (R11 + R22 - 2 R12)/4,
  // the coupling block -> (2 R12 - R11 - R22)/4.
  TwoBody p;
  p.x11 = p.x22 = (t.x11 + t.x22 - 2 * t.x12) / 4;
  p.y11 = p.y22 = (t.y11 + t.y22 - 2 * t.y12) / 4;
  p.x12 = (2 * t.x12 - t.x11 - t.x22) / 4;
  p.y12 = (2 * t.y12 - t.y11 - t.y22) / 4;
  return p;
}

__device__ __forceinline__ void xy_block(double X, double Y, double rx, double ry, double rz,
                                         double d2, double out[6]) {
  out[0] = X * rx * rx / d2 + Y * (1 - rx * rx / d2);
  out[1] = X * ry * ry / d2 + Y * (1 - ry * ry / d2);
  out[2] = X * rz * rz / d2 + Y * (1 - rz * rz / d2);
  out[3] = (X - Y) * rx * ry / d2;
  out[4] = (X - Y) * rx * rz / d2;
  out[5] = (X - Y) * ry * rz / d2;
}

// Correction scalars of pair (first bead j, second bead i) at distance d.
__device__ TwoBody pair_correction(double aj, double ai, double d, int cich) {
  TwoBody nf = jo_two_body(aj, ai, d);
  TwoBody ff = rpy_two_body_resistance(aj, ai, d);
  if (cich) {
    nf = cichocki(nf);
    ff = cichocki(ff);
  }
  TwoBody r;
  r.x11 = nf.x11 - ff.x11; r.y11 = nf.y11 - ff.y11;
  r.x22 = nf.x22 - ff.x22; r.y22 = nf.y22 - ff.y22;
  r.x12 = nf.x12 - ff.x12; r.y12 = nf.y12 - ff.y12;
  return r;
}

__device__ __forceinline__ bool within_cutoff(double d, double ai, double aj, double cutoff) {
  return (d - aj - ai) / (aj + ai) <= cutoff;  // diff_tensor.c:388
}

__device__ __forceinline__ void add_block(double* M, int ld, int row0, int col0, const double b[6],
                                          double scale) {
  const int comp[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) M[(size_t)(row0 + r) * ld + col0 + c] += scale * b[comp[r][c]];
}

__global__ void lub_offdiag_kernel(PairSource src, const double* __restrict__ radii,
                                   double cutoff, int cich, double scale,
                                   double* __restrict__ M, int ld) {
  const int n = src.n;
  const long long npairs = (long long)n * (n - 1) / 2;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    int i, j;
    pair_from_linear(p, i, j);
    double rx, ry, rz;
    get_pair_vector(src, i, j, rx, ry, rz);
    const double d2 = rx * rx + ry * ry + rz * rz, d = sqrt(d2);
    if (!within_cutoff(d, radii[i], radii[j], cutoff)) continue;
    const TwoBody c = pair_correction(radii[j], radii[i], d, cich);
    double b[6];
    xy_block(c.x12, c.y12, rx, ry, rz, d2, b);
    add_block(M, ld, 3 * i, 3 * j, b, scale);
    add_block(M, ld, 3 * j, 3 * i, b, scale);
  }
}

// One warp per bead b: contributions from partners p in increasing order
// (p < b: b is the second bead, block 22; p > b: b is the first bead, block 11).
__global__ void lub_diag_kernel(PairSource src, const double* __restrict__ radii,
                                double cutoff, int cich, double scale,
                                double* __restrict__ M, int ld) {
  const int n = src.n;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int b = warp;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int base = 0; base < n; base += 32) {
    const int p = base + lane;
    double v[6] = {0, 0, 0, 0, 0, 0};
    bool hit = false;
    if (p < n && p != b) {
      const int i = p > b ? p : b, j = p > b ? b : p;
      double rx, ry, rz;
      get_pair_vector(src, i, j, rx, ry, rz);
      const double d2 = rx * rx + ry * ry + rz * rz, d = sqrt(d2);
      if (within_cutoff(d, radii[i], radii[j], cutoff)) {
        const TwoBody c = pair_correction(radii[j], radii[i], d, cich);
        if (p > b) xy_block(c.x11, c.y11, rx, ry, rz, d2, v);  // b == j, first bead
        else xy_block(c.x22, c.y22, rx, ry, rz, d2, v);        // b == i, second bead
        hit = true;
      }
    }
    unsigned mask = __ballot_sync(0xffffffffu, hit);
    while (mask) {  // ordered accumulation over the hits of this chunk
      const int src = __ffs(mask) - 1;
      mask &= mask - 1;
      for (int c = 0; c < 6; ++c) acc[c] += __shfl_sync(0xffffffffu, v[c], src);
    }
  }
  if (lane == 0) add_block(M, ld, 3 * b, 3 * b, acc, scale);
}

__global__ void jo_pair_kernel(double ai, double aj, double rx, double ry, double rz, double* out) {
  const double d2 = rx * rx + ry * ry + rz * rz, d = sqrt(d2);
  const TwoBody t = jo_two_body(ai, aj, d);
  xy_block(t.x11, t.y11, rx, ry, rz, d2, out);
  xy_block(t.x22, t.y22, rx, ry, rz, d2, out + 6);
  xy_block(t.x12, t.y12, rx, ry, rz, d2, out + 12);
}

}  // namespace

int launch_lubrication_add(const PairSource& src, const double* radii, double cutoff,
                           int cichocki_correction, double scale, double* M, int ld, cudaStream_t st) {
  const int n = src.n;
  if (n < 2) return PBG_OK;
  const long long npairs = (long long)n * (n - 1) / 2;
  const int blocks = (int)std::min<long long>((npairs + 255) / 256, 148LL * 16);
  lub_offdiag_kernel<<<blocks, 256, 0, st>>>(src, radii, cutoff, cichocki_correction, scale, M, ld);
  PBG_CHECK_LAUNCH();
  lub_diag_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(src, radii, cutoff, cichocki_correction, scale, M, ld);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int launch_jo_pair(double ai, double aj, double rx, double ry, double rz, double* out18, cudaStream_t st) {
  jo_pair_kernel<<<1, 1, 0, st>>>(ai, aj, rx, ry, rz, out18);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
