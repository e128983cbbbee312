// The pbg_system handle (device-resident state of one simulated box).
#pragma once

#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace pbg {
struct ForceField;
}

struct pbg_system {
  pbg_params p{};
  int N = 0, n = 0, ld = 0;  // beads, matrix order 3N, padded order
  bool lub = false, smith = false;
  // Mixed lubricated path (lubrication modes, precision "mixed"): Mff, Rff
  // (and their midpoint copies) are FP32, R stays FP64, D and B are FP32.
  bool mlub = false;
  bool work_holds_R = false;  // inv_work holds G = chol(J R J) and inv(G) of the current R
  void* G = nullptr;          // mlub, midpoint: FP32 G of the step-start R (B = sqrt(kBT) J G^{-T} J)
  bool g_valid = false;       // G belongs to the B in use
  int prec = PBG_PREC_FP64;  // element type of D and B
  size_t es = 8;
  const pbg::EwaldTables* tables = nullptr;

  double* pos = nullptr;       // N x 3
  double* pos_snap = nullptr;  // N x 3, step-start copy (device-resident runs)
  double* radii = nullptr;     // N
  int* conn = nullptr;         // N x N bond matrix or null
  double* force = nullptr;     // ld (3N used)
  bool force_zero = true;        // the external force is known to be zero (pbg_set_force from host or NULL)
  bool b_holds_lower_D = false;  // this step's D build also wrote B's lower triangle (and padding)
  void* D = nullptr;           // ld x ld, prec
  void* B = nullptr;           // ld x ld, prec, lower factor
  void* D0 = nullptr;          // midpoint: step-start D
  double *Mff = nullptr, *Rff = nullptr, *R = nullptr;     // lubrication modes (Mff, Rff FP32 if mlub)
  double *Mff0 = nullptr, *Rff0 = nullptr, *R0 = nullptr;  // midpoint copies
  double *FX = nullptr, *U = nullptr, *BX = nullptr, *ddet = nullptr, *y = nullptr;
  double *rwork = nullptr, *Dy = nullptr, *drift = nullptr, *xi = nullptr;  // ld each
  double *sol = nullptr, *sol0 = nullptr, *res = nullptr, *corr = nullptr;  // ld each: refined solves (mlub)
  void* phase = nullptr;       // Ewald phase tables
  void* chol_work = nullptr;   // inverted diagonal tiles of B
  void* inv_work = nullptr;    // SPD inverse workspace (tensor-core inverse workspace if mlub)
  int* dflags = nullptr;       // [0] overlap, [1] cholesky info, [2] Rff info, [3] D info,
                               // [4] back-substitution wait (-1: gave up)
  int* tflags = nullptr;       // ld / 64 block-row flags of the one-launch back substitution
  bool divergence = false;     // divergence term of the lubricated D (Ermak scheme)
  double* div = nullptr;       // ld: its value this step
  int* hflags = nullptr;       // pinned mirror
  double* hpos = nullptr;      // pinned N x 3 staging for pbg_step_finish

  // Immobile beads (box.py:649-668): overlap partners and force sources only.
  int M = 0;
  double* pos_imm = nullptr;   // M x 3
  double* radii_imm = nullptr; // M
  int* order = nullptr;        // N + M: index in the caller's full bead list
  int* conn_mi = nullptr;      // N x M bond flags, or null
  // Inter-bead forces (interactions.py); null without them.
  pbg::ForceField* ff = nullptr;
  double* ftot = nullptr;      // ld: force of the step (base + interactions)
  double* energy = nullptr;    // interaction energy of the step (device scalar)

  bool have_state = false;
  bool in_step = false;
  double dt = 0;
  int build_Dff = 1, build_Dnf = 1, cholesky = 1;
  int attempts = 0;
  pbg_step_report report{};    // outcome of the last pbg_run
  // Device-side steps of pbg_run (Ermak scheme, noise pool in device memory):
  // one CUDA graph per step -- the step start, a conditional WHILE node over
  // the move attempts, the wrap -- captured once a step repeats with the same
  // flags, dt and force state.
  void* d_run = nullptr;                 // the run's device state (noise cursor, attempts, status)
  void* h_run = nullptr;                 // pinned copy: upload before a step, report after it
  cudaGraphExec_t run_exec = nullptr;
  cudaStream_t cap_stream = nullptr, cap_stream2 = nullptr;
  long long run_key = -1;                // step flags and force state of run_exec
  double run_key_dt = 0;
  int run_key_repeats = 0;
  bool run_refused = false;              // the driver refused the capture: host-driven steps
  long long run_fixed_kernels = 0;       // kernels per replay besides the attempt rounds
  long long run_round_kernels = 0;       // kernels per attempt round
};

namespace pbg {

int create_system(const pbg_params* p, pbg_system** out);
void destroy_system(pbg_system* s);
int system_set_state(pbg_system* s, const double* pos, const double* radii, const int* conn, cudaStream_t st);
int build_nohi(pbg_system* s, cudaStream_t st);
int compute_Dff(pbg_system* s, cudaStream_t st, bool fill_B);
int compute_Dtot(pbg_system* s, cudaStream_t st);
int decompose(pbg_system* s, cudaStream_t st);
int step_begin(pbg_system* s, double dt, int build_Dff, int build_Dnf, int chol, cudaStream_t st);
int set_divergence(pbg_system* s, bool on);
int step_attempt(pbg_system* s, const double* xi, int* accepted, cudaStream_t st);
int step_end(pbg_system* s, cudaStream_t st, double* pos_out = nullptr);
int run(pbg_system* s, long long j0, int n_steps, double dt, int diff_freq, int lub_freq, int chol_freq,
        const double* pool, long long pool_len, cudaStream_t st);
// Drops pbg_run's captured step graph (the system's buffers or interactions changed).
void drop_run_graph(pbg_system* s);
int system_get_matrix(pbg_system* s, int which, double* out, cudaStream_t st);
int system_set_matrix(pbg_system* s, int which, const double* in, cudaStream_t st);
int set_immobile(pbg_system* s, int M, const double* pos, const double* radii, const int* order,
                 const int* conn_mi, cudaStream_t st);
int set_interactions(pbg_system* s, const pbg_interactions* d);
void free_interactions(pbg_system* s);
void free_immobile(pbg_system* s);
// Force of the step into s->ftot and the energy into s->energy (no-op without interactions).
int compute_forces(pbg_system* s, cudaStream_t st);
// Overlap of any mobile bead with any immobile one, OR-ed into *flag.
int overlap_immobile(pbg_system* s, int* flag, cudaStream_t st);
inline const double* step_force(const pbg_system* s) { return s->ff ? s->ftot : s->force; }

}  // namespace pbg
