// Internal (C++) interfaces between the pybrown_b200 translation units.
#pragma once

#include <vector>

#include "common.cuh"

namespace pbg {

// Pair index p in [0, n(n-1)/2) -> (i, j) with i > j, p = i(i-1)/2 + j.
__device__ __forceinline__ void pair_from_linear(long long p, int& i, int& j) {
  int ii = (int)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
  while ((long long)ii * (ii - 1) / 2 > p) --ii;
  while ((long long)(ii + 1) * ii / 2 <= p) ++ii;
  i = ii;
  j = (int)(p - (long long)ii * (ii - 1) / 2);
}

// Where pair vectors come from: device positions (minimum image in L) or,
// for the reference ABI, the packed upper-triangle pair vectors the Python
// wrappers build (diffusion.py:40,70,155): 3 doubles per pair i > j at
// 3*((i-1) + j*(n-1) - j*(j+1)/2), value r_j - r_i.
struct PairSource {
  const double* pos;    // N x 3, or null
  const double* pairs;  // packed pair vectors, or null
  int n;
  double L;
};

// Returns the vector the reference kernels see for pair (i > j): r_j - r_i
// after the minimum image.
__device__ __forceinline__ void get_pair_vector(const PairSource& s, int i, int j, double& rx,
                                                double& ry, double& rz) {
  if (s.pairs) {
    const long long k = 3LL * ((i - 1) + (long long)j * (s.n - 1) - (long long)j * (j + 1) / 2);
    rx = s.pairs[k];
    ry = s.pairs[k + 1];
    rz = s.pairs[k + 2];
  } else {
    rx = -pbg_min_image(s.pos[3 * i + 0] - s.pos[3 * j + 0], s.L);
    ry = -pbg_min_image(s.pos[3 * i + 1] - s.pos[3 * j + 1], s.L);
    rz = -pbg_min_image(s.pos[3 * i + 2] - s.pos[3 * j + 2], s.L);
  }
}

// Reconstructs coordinates consistent with packed pair vectors
// (r_0 = 0, r_i = -(r_0 - r_i) from the first column); used only for the
// periodic phases of the reciprocal sum, which ignore lattice shifts.
int launch_positions_from_pairs(const double* pairs, int n, double* pos, cudaStream_t st);

// ---- geometry.cu ---------------------------------------------------------
// Overlap test of one pair with the reference's axis pre-filter
// (bead.c:188-216) and minimum-image distance (bead.c:222-260).
__device__ __forceinline__ bool pair_overlaps(const double* __restrict__ pos,
                                              const double* __restrict__ radii, int i, int j,
                                              double L, double thr) {
  double r[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) r[c] = pos[3 * i + c] - pos[3 * j + c];
  const double rs = radii[i] + radii[j];
  const double rs_pbc = L - rs;
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if (((r[c] > rs) && (r[c] < rs_pbc)) || ((r[c] < -rs) && (r[c] > -rs_pbc))) return false;
  const double x = pbg_min_image(r[0], L), y = pbg_min_image(r[1], L), z = pbg_min_image(r[2], L);
  return sqrt(x * x + y * y + z * z) <= radii[i] + radii[j] + thr;
}

int launch_pointer_matrix(const double* pos, int n, double L, double* rij, cudaStream_t st);
int launch_overlap(const double* pos, const double* radii, int n, double L, double thr,
                   const int* conn, int* flag, cudaStream_t st);

// ---- ewald.cu -------------------------------------------------------------
// Reciprocal-space and real-space tables of one (alpha, m_max, n_max) set.
struct EwaldTables {
  double alpha = 0;
  int m_max = -1, n_max = -1;
  int n_real = 0;      // images with |m|_1 <= m_max (m = 0 included)
  int n_recip = 0;     // half of the n != 0 vectors with |n|_1 <= n_max
  double self_O[6];    // lattice sums of the self block (a-independent part)
  double self_Q[6];
  double* d_real = nullptr;   // n_real x 4 doubles: mx, my, mz, 0
  double* d_recip = nullptr;  // n_recip x 8 doubles: nx, ny, nz, P, R, S, 0, 0
  float* d_recip_f = nullptr; // same, float
};

// Returns the (cached) tables for a parameter set; they live until exit.
int get_ewald_tables(double alpha, int m_max, int n_max, const EwaldTables** out);
// Number of integer points with |x| + |y| + |z| <= m: the real-space images
// of ewald_real = m; (lattice_points_l1(n) - 1) / 2 reciprocal half-vectors
// of ewald_imag = n.
long long lattice_points_l1(int m);
// Host tables of one (alpha, m_max, n_max) set in the layout of EwaldTables
// (real: 4 doubles per image, recip: 8 doubles per half-vector) and the
// a-independent self-block lattice sums.  The one builder behind every
// device copy of the tables.
void build_lattice_tables(double alpha, int m_max, int n_max, std::vector<double>& real,
                          std::vector<double>& recip, double self_O[6], double self_Q[6]);

// Writes scale * M for the free-space (smith == false) or Smith-Ewald RPY
// tensor of positions `pos` into M (row-major, leading dimension ld).
// precision: PBG_PREC_FP64 (double* M) or PBG_PREC_MIXED (float* M).
// `phase` is scratch of phase_scratch_bytes(n, tables) bytes (may be null for
// the free-space tensor).
size_t phase_scratch_bytes(int n, const EwaldTables* t, int precision);
// `pos` feeds the reciprocal phases (for pair-vector input pass the
// reconstructed coordinates of launch_positions_from_pairs).
// M_lower (optional): a second matrix that receives the same values in the
// bead tiles on and below the block diagonal (every element of the lower
// triangle; the rest of it is left as it was).
int launch_rpy_tensor(const PairSource& src, const double* pos, const double* radii, bool smith,
                      const EwaldTables* t, double scale, int precision, void* M, int ld,
                      void* phase, cudaStream_t st, void* M_lower = nullptr);

// ---- lubrication.cu -------------------------------------------------------
int launch_lubrication_add(const PairSource& src, const double* radii, double cutoff,
                           int cichocki, double scale, double* M, int ld, cudaStream_t st);
// Single pair, 18 components (tier-1 JO_2B_R_matrix).
int launch_jo_pair(double ai, double aj, double rx, double ry, double rz, double* out18,
                   cudaStream_t st);

// ---- cholesky.cu ----------------------------------------------------------
// Sets rows/cols n..ld-1 of an ld x ld matrix to the identity.
int launch_pad_identity(void* A, int n, int ld, int precision, cudaStream_t st);
// Workspace: inverted diagonal tiles of the factor followed by the data-flow
// scratch (see cholesky.cu).
size_t cholesky_work_bytes(int ld, int precision);
int launch_cholesky_ws(void* A, int n, int ld, int precision, int* info, void* work, cudaStream_t st);
// cholesky_df.cu
size_t df_work_bytes(int ld);
// X (or null): the same launch also forms the off-diagonal tiles of
// X = inv(L) (ld x ld, lower; launch_trtri_diag copies the diagonal ones from
// invdiag).
int launch_cholesky_df(void* A, int n, int ld, int precision, int* info, void* invdiag, void* work,
                       cudaStream_t st, void* X = nullptr);
size_t spd_inverse_work_bytes(int ld);
int launch_spd_inverse(double* A, int n, int ld, int* info, void* work, cudaStream_t st);

// X's diagonal tiles from invdiag, and out = scale X^T X (optionally with
// every index i -> ld-1-i), on the tensor cores, FP64 or FP32 (cholesky_df.cu).
int launch_trtri_diag(const void* invdiag, void* X, int ld, int precision, cudaStream_t st);
int launch_lauum_tc(const void* X, int ld, double scale, bool reversed, void* out, int precision, cudaStream_t st);
// SPD inverse of the mixed lubricated path (FP32).  The caller puts the
// matrix (order ld, padded) in F; tc_factor_invert factors it in place
// (F = G, lower) and forms X = inv(G); tc_lauum writes scale X^T X on the
// tcgen05 tensor cores (a wait that gives up sets *info = -1);
// tc_reversed_factor writes B = s J X^T J (lower; J reverses all ld indices)
// and the inverted diagonal tiles of that B, for launch_trsv_upper.
struct TcInverseWork {
  float* invdiag;  // nt x 64 x 64
  void* scratch;   // data-flow scratch
  float* X;        // ld x ld
  float* F;        // ld x ld
};
size_t tc_inverse_work_bytes(int ld);
TcInverseWork tc_inverse_work(void* work, int ld);
int tc_factor_invert(int ld, int* info, void* work, cudaStream_t st);
int tc_lauum(const float* X, int ld, float scale, bool reversed, float* out, int* info, cudaStream_t st);
int tc_reversed_factor(const float* X, const float* G, int ld, double s, float* B, float* invdiag,
                       cudaStream_t st);

// Batched factorisation of many independent matrices (one per replica).
struct CholRep {
  void* A;        // ld x ld, padded with the identity beyond n
  void* invdiag;  // nt x 64 x 64: inv(L_kk) tiles
  int* upd;       // nt x nt, zero before the launch
  int* fin;       // nt x nt, zero before the launch
  int* info;      // zero before the launch
  int ld, n, nt, pad;
};
// One replica's task list (task.x = type, replica tag 0) cut into segments
// that a batch interleaves with the other replicas' (see cholesky_df.cu);
// task.x = type | replica << 3 in the merged list.
void cholesky_replica_tasks(int nt, int precision, std::vector<int4>& tasks, std::vector<int>& seg_start);
// Resident CTAs per SM of the batched factorisation kernel, and the SM count.
int cholesky_batch_residency(int precision, int* ctas_per_sm, int* sms);
// ctl: 4 ints (next task, abort, spin failures, error bits), zero before the launch.
// ctas_per_sm: resident CTAs per SM (0 = as many as fit).
int launch_cholesky_batch(int precision, const CholRep* reps, const int4* tasks, int ntasks, int* ctl,
                          int ctas_per_sm, cudaStream_t st);

// Batched RPY / Smith-Ewald tensor build: one argument block per replica and
// a work list of bead tiles (x = replica, y = I, z = J with I >= J).
size_t rpy_batch_arg_bytes();
// Fills the argument block of one replica into `dst` (rpy_batch_arg_bytes() bytes);
// M_lower: the matrix that receives the lower block triangle when a launch asks for it.
void rpy_batch_arg(const double* pos, const double* radii, int n, double L, bool smith, const EwaldTables* t,
                   double scale, void* M, void* M_lower, int ld, void* phase, void* dst);
void rpy_batch_work(int replica, int n, std::vector<int4>& work);
int launch_rpy_batch(int precision, bool smith, const EwaldTables* t, const void* args, const int4* work,
                     int nwork, int n_replicas, bool fill_lower, cudaStream_t st);

}  // namespace pbg
