// Inter-bead forces and immobile beads on sm_100a
// (src/bdsim/pyBrown/interactions.py:57-821, box.py:404-428, 649-668).
//
// The reference evaluates its interactions in Python loops over bead pairs,
// bonds and angles at the step-start positions and sums them into F.  Here:
//   - Lennard-Jones: one warp per mobile bead over every other bead (mobile
//     and immobile), lanes striding the partners, a fixed shuffle tree for the
//     sum (deterministic);
//   - bonds and angles: one thread per term writes its force pieces and
//     energy; one thread per mobile bead then gathers its pieces from a
//     per-bead event list in the reference's loop order;
//   - energy: one block, fixed reduction order.
// Everything is FP64, like the reference.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "system.cuh"

namespace pbg {

struct ForceField {
  int lj = PBG_LJ_NONE;
  double lj_alpha = 0;
  double scale = 1;
  int nb = 0, na = 0;
  double* hc = nullptr;       // N + M hard-core radii
  double* eps = nullptr;      // N + M LJ energies
  int* bonds = nullptr;       // 2 per bond
  double* bond_p = nullptr;   // 2 per bond
  int* angles = nullptr;      // 4 per angle
  double* angle_p = nullptr;  // 2 per angle
  int* bond_off = nullptr;    // N + 1
  int* bond_ev = nullptr;     // (bond << 1) | (minus)
  int* angle_off = nullptr;   // N + 1
  int* angle_ev = nullptr;    // angle * 3 + role
  double* flj = nullptr;      // 3N
  double* elj = nullptr;      // N
  double* bf = nullptr;       // 3 per bond
  double* be = nullptr;       // 1 per bond
  double* af = nullptr;       // 9 per angle
  double* ae = nullptr;       // 1 per angle
};

namespace {

struct Beads {
  const double* pos;      // N x 3 mobile
  const double* pos_imm;  // M x 3 immobile
  int N, M;
  double L;
};

// Minimum-image vector from bead a to bead b as the reference's Python reads
// it: rij[a][b] (bead.c:27-95 computes it for the higher index minus the lower
// one and stores the negation for the transposed entry), rik[a][k]
// (bead.c:99-158, immobile minus mobile) and -rik[b][a].
__device__ __forceinline__ void pointer_ab(const Beads& bs, int a, int b, double p[3]) {
  if (a < bs.N && b < bs.N) {
    const int lo = min(a, b), hi = max(a, b);
    const double s = a < b ? 1.0 : -1.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c] = s * pbg_min_image(bs.pos[3 * hi + c] - bs.pos[3 * lo + c], bs.L);
  } else if (a < bs.N) {
    const double* q = bs.pos_imm + 3 * (b - bs.N);
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c] = pbg_min_image(q[c] - bs.pos[3 * a + c], bs.L);
  } else if (b < bs.N) {
    const double* q = bs.pos_imm + 3 * (a - bs.N);
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c] = -pbg_min_image(q[c] - bs.pos[3 * b + c], bs.L);
  } else {
    p[0] = p[1] = p[2] = 0.0;
  }
}

// LJ force on bead 1 and pair energy (interactions.py:711-821).
__device__ __forceinline__ void lj_pair(int kind, double alpha, double hc1, double hc2, double e1, double e2,
                                        const double p[3], double f[3], double& e) {
  const double sigma = hc1 + hc2;
  const double epsilon = sqrt(e1 * e2);
  const double dist2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  const double dist = sqrt(dist2);
  const double s2 = sigma * sigma / dist2;
  const double s6 = s2 * s2 * s2;
  double coef;
  if (kind == PBG_LJ_6) {
    coef = 6.0 * alpha * epsilon * s6 / dist;
    e = -alpha * epsilon * s6;
  } else if (kind == PBG_LJ_12) {
    const double s12 = s2 * s2 * s2 * s2 * s2 * s2;
    coef = -12.0 * alpha * epsilon * s12 / dist;
    e = alpha * epsilon * s12;
  } else {
    const double s12 = s6 * s6;
    coef = alpha * epsilon / dist * (6 * s6 - 12 * s12);
    e = alpha * epsilon * (s12 - s6);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) f[c] = coef * (p[c] / dist);
}

__global__ void lj_kernel(Beads bs, int kind, double alpha, const double* __restrict__ hc,
                          const double* __restrict__ eps, double* __restrict__ flj, double* __restrict__ elj) {
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (b >= bs.N) return;
  double f[3] = {0.0, 0.0, 0.0}, e = 0.0;
  const int total = bs.N + bs.M;
  for (int j = lane; j < total; j += 32) {
    if (j == b) continue;
    double p[3], g[3], ej;
    pointer_ab(bs, b, j, p);
    lj_pair(kind, alpha, hc[b], hc[j], eps[b], eps[j], p, g, ej);
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c] += g[c];
    // interactions.py:249-289: mobile pairs once (i > j), mobile-immobile pairs once.
    if (j < b || j >= bs.N) e += ej;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c] += __shfl_xor_sync(0xffffffffu, f[c], o);
    e += __shfl_xor_sync(0xffffffffu, e, o);
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) flj[3 * b + c] = f[c];
    elj[b] = e;
  }
}

// Harmonic bond (interactions.py:641-665): f = versor k (d - d_eq) on bead a.
__global__ void bond_kernel(Beads bs, int nb, const int* __restrict__ bonds, const double* __restrict__ prm,
                            double* __restrict__ bf, double* __restrict__ be) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb) return;
  double p[3];
  pointer_ab(bs, bonds[2 * t], bonds[2 * t + 1], p);
  const double deq = prm[2 * t], k = prm[2 * t + 1];
  const double dist = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) bf[3 * t + c] = p[c] / dist * k * (dist - deq);
  be[t] = 0.5 * k * ((dist - deq) * (dist - deq));
}

// Harmonic angle (interactions.py:667-709, angle_pbc bead.py:272-278): the
// angle goes through degrees and back as in the reference.
__global__ void angle_kernel(Beads bs, int na, const int* __restrict__ angles, const double* __restrict__ prm,
                             double* __restrict__ af, double* __restrict__ ae) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na) return;
  const int i = angles[4 * t], j = angles[4 * t + 1], k = angles[4 * t + 2], form = angles[4 * t + 3];
  double p12[3], p23[3];
  if (form == PBG_ANGLE_P12_DIFF) {
    double pik[3], pjk[3];
    pointer_ab(bs, i, k, pik);
    pointer_ab(bs, j, k, pjk);
#pragma unroll
    for (int c = 0; c < 3; ++c) p12[c] = pik[c] - pjk[c];
    pointer_ab(bs, j, k, p23);
  } else {
    pointer_ab(bs, i, j, p12);
    if (form == PBG_ANGLE_P23_DIFF) {
      double pik[3];
      pointer_ab(bs, i, k, pik);
#pragma unroll
      for (int c = 0; c < 3; ++c) p23[c] = pik[c] - p12[c];
    } else {
      pointer_ab(bs, j, k, p23);
    }
  }
  const double d2_12 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
  const double d2_23 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
  const double d12 = sqrt(d2_12), d23 = sqrt(d2_23);
  const double x = -(p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2]) / d12 / d23;
  const double angle = acos(x) * (180.0 / PBG_PI) * (PBG_PI / 180.0);
  const double angle_eq = prm[2 * t] * (PBG_PI / 180.0);
  const double kf = prm[2 * t + 1];
  const double ca = cos(angle);
  const double coef = kf * (angle - angle_eq) / sin(angle);
  double* o = af + 9 * t;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o[c] = coef * ((p23[c] / d23 + ca * p12[c] / d12) / d12);
    o[3 + c] = coef * ((p12[c] - p23[c]) / d12 / d23 - ca * (p12[c] / d2_12 - p23[c] / d2_23));
    o[6 + c] = coef * (-p12[c] / d12 / d23 - ca * p23[c] / d2_23);
  }
  ae[t] = 0.5 * kf * ((angle - angle_eq) * (angle - angle_eq));
}

// F_b = base_b + scale * (LJ_b + bond pieces + angle pieces), the pieces in
// the reference's accumulation order (interactions.py:185-247, 291-414).
__global__ void combine_kernel(int N, double scale, const double* __restrict__ base, int lj,
                               const double* __restrict__ flj, const int* __restrict__ bond_off,
                               const int* __restrict__ bond_ev, const double* __restrict__ bf,
                               const int* __restrict__ angle_off, const int* __restrict__ angle_ev,
                               const double* __restrict__ af, double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= N) return;
  double f[3] = {0.0, 0.0, 0.0};
  if (lj) {
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c] = flj[3 * b + c];
  }
  if (bond_off) {
    for (int q = bond_off[b]; q < bond_off[b + 1]; ++q) {
      const int ev = bond_ev[q];
      const double* g = bf + 3 * (ev >> 1);
      if (ev & 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f[c] -= g[c];
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) f[c] += g[c];
      }
    }
  }
  if (angle_off) {
    for (int q = angle_off[b]; q < angle_off[b + 1]; ++q) {
      const int ev = angle_ev[q];
      const double* g = af + 9 * (ev / 3) + 3 * (ev % 3);
#pragma unroll
      for (int c = 0; c < 3; ++c) f[c] += g[c];
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) out[3 * b + c] = base[3 * b + c] + scale * f[c];
}

// E = sum(LJ) + sum(bonds) + sum(angles) (box.py:404-428 order of the
// interactions), each part reduced in a fixed order by one block.
__global__ void energy_kernel(int N, int lj, const double* __restrict__ elj, int nb, const double* __restrict__ be,
                              int na, const double* __restrict__ ae, double* __restrict__ out) {
  __shared__ double red[256];
  double total = 0.0;
  for (int part = 0; part < 3; ++part) {
    const double* v = part == 0 ? (lj ? elj : nullptr) : part == 1 ? be : ae;
    const int n = part == 0 ? N : part == 1 ? nb : na;
    double s = 0.0;
    if (v)
      for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    total += red[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = total;
}

// Overlap of mobile bead b with immobile bead k (bead.c:169-260): the pair
// vector is the later bead of the full list minus the earlier one.
__global__ void overlap_immobile_kernel(Beads bs, const double* __restrict__ radii,
                                        const double* __restrict__ radii_imm, const int* __restrict__ order,
                                        const int* __restrict__ conn_mi, double thr, int* __restrict__ flag) {
  const long long total = (long long)bs.N * bs.M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / bs.M), k = (int)(t % bs.M);
    if (conn_mi && conn_mi[t]) continue;
    const double* pb = bs.pos + 3 * b;
    const double* pk = bs.pos_imm + 3 * k;
    const bool b_later = order ? order[b] > order[bs.N + k] : false;
    double r[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = b_later ? pb[c] - pk[c] : pk[c] - pb[c];
    const double rs = radii[b] + radii_imm[k];
    const double rs_pbc = bs.L - rs;
    bool far = false;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      far = far || ((r[c] > rs) && (r[c] < rs_pbc)) || ((r[c] < -rs) && (r[c] > -rs_pbc));
    if (far) continue;
    const double x = pbg_min_image(r[0], bs.L), y = pbg_min_image(r[1], bs.L), z = pbg_min_image(r[2], bs.L);
    if (sqrt(x * x + y * y + z * z) <= rs + thr) {
      atomicOr(flag, 1);
      return;
    }
  }
}

template <typename T>
int upload(T** dst, const T* src, size_t count) {
  if (count == 0) {
    *dst = nullptr;
    return PBG_OK;
  }
  if (cudaMalloc((void**)dst, count * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *dst = nullptr;
    pbg_set_error_message("out of device memory for the interactions");
    return PBG_ERR_NOMEM;
  }
  PBG_CUDA_TRY(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyDefault));
  return PBG_OK;
}

template <typename T>
int alloc(T** dst, size_t count) {
  *dst = nullptr;
  if (count == 0) return PBG_OK;
  if (cudaMalloc((void**)dst, count * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *dst = nullptr;
    pbg_set_error_message("out of device memory for the interactions");
    return PBG_ERR_NOMEM;
  }
  return PBG_OK;
}

// Reads n ints / doubles from host or device memory.
template <typename T>
int fetch(std::vector<T>& out, const T* src, size_t n) {
  out.resize(n);
  if (n == 0) return PBG_OK;
  PBG_CUDA_TRY(cudaMemcpy(out.data(), src, n * sizeof(T), cudaMemcpyDefault));
  return PBG_OK;
}

Beads beads_of(const pbg_system* s) { return Beads{s->pos, s->pos_imm, s->N, s->M, s->p.box_length}; }

}  // namespace

void free_interactions(pbg_system* s) {
  ForceField* f = s->ff;
  if (f) {
    void* ptrs[] = {f->hc,      f->eps,      f->bonds,     f->bond_p,   f->angles, f->angle_p, f->bond_off,
                    f->bond_ev, f->angle_off, f->angle_ev, f->flj,      f->elj,    f->bf,      f->be,
                    f->af,      f->ae};
    for (void* p : ptrs)
      if (p) cudaFree(p);
    delete f;
  }
  s->ff = nullptr;
  if (s->ftot) cudaFree(s->ftot);
  if (s->energy) cudaFree(s->energy);
  s->ftot = nullptr;
  s->energy = nullptr;
}

void free_immobile(pbg_system* s) {
  void* ptrs[] = {s->pos_imm, s->radii_imm, s->order, s->conn_mi};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  s->pos_imm = s->radii_imm = nullptr;
  s->order = s->conn_mi = nullptr;
  s->M = 0;
}

int set_immobile(pbg_system* s, int M, const double* pos, const double* radii, const int* order,
                 const int* conn_mi, cudaStream_t st) {
  if (M < 0 || (M > 0 && (!pos || !radii))) return PBG_ERR_ARG;
  if (s->ff) {
    pbg_set_error_message("pbg_set_immobile after pbg_set_interactions: set the immobile beads first");
    return PBG_ERR_STATE;
  }
  PBG_CUDA_TRY(cudaStreamSynchronize(st));
  free_immobile(s);
  if (M == 0) return PBG_OK;
  int rc;
  const size_t N = s->N;
  if ((rc = upload(&s->pos_imm, pos, (size_t)M * 3)) || (rc = upload(&s->radii_imm, radii, (size_t)M)) ||
      (order && (rc = upload(&s->order, order, N + M))) ||
      (conn_mi && (rc = upload(&s->conn_mi, conn_mi, N * M)))) {
    free_immobile(s);
    return rc;
  }
  s->M = M;
  return PBG_OK;
}

int set_interactions(pbg_system* s, const pbg_interactions* d) {
  PBG_CUDA_TRY(cudaDeviceSynchronize());
  free_interactions(s);
  if (!d) return PBG_OK;
  const int N = s->N, M = s->M, total = N + M;
  if ((d->lennard_jones != PBG_LJ_NONE && d->lennard_jones != PBG_LJ_6 && d->lennard_jones != PBG_LJ_12 &&
       d->lennard_jones != PBG_LJ_6_12) ||
      d->n_bonds < 0 || d->n_angles < 0 || (d->n_bonds > 0 && (!d->bonds || !d->bond_params)) ||
      (d->n_angles > 0 && (!d->angles || !d->angle_params)) ||
      (d->lennard_jones != PBG_LJ_NONE && (!d->hard_core_radius || !d->epsilon_lj))) {
    pbg_set_error_message("invalid pbg_interactions");
    return PBG_ERR_ARG;
  }
  std::vector<int> bonds, angles;
  int rc;
  if ((rc = fetch(bonds, d->bonds, (size_t)2 * d->n_bonds)) || (rc = fetch(angles, d->angles, (size_t)4 * d->n_angles)))
    return rc;
  for (int v : bonds)
    if (v < 0 || v >= total) {
      pbg_set_error_message("bond bead index %d out of range", v);
      return PBG_ERR_ARG;
    }
  for (int t = 0; t < d->n_angles; ++t) {
    for (int c = 0; c < 3; ++c)
      if (angles[4 * t + c] < 0 || angles[4 * t + c] >= total) {
        pbg_set_error_message("angle bead index %d out of range", angles[4 * t + c]);
        return PBG_ERR_ARG;
      }
    if (angles[4 * t + 3] < PBG_ANGLE_DIRECT || angles[4 * t + 3] > PBG_ANGLE_P12_DIFF) {
      pbg_set_error_message("invalid angle form %d", angles[4 * t + 3]);
      return PBG_ERR_ARG;
    }
  }
  // Per-mobile-bead event lists in the order the terms are met.
  std::vector<std::vector<int>> bev(N), aev(N);
  for (int t = 0; t < d->n_bonds; ++t) {
    if (bonds[2 * t] < N) bev[bonds[2 * t]].push_back(t << 1);
    if (bonds[2 * t + 1] < N) bev[bonds[2 * t + 1]].push_back((t << 1) | 1);
  }
  for (int t = 0; t < d->n_angles; ++t)
    for (int role = 0; role < 3; ++role)
      if (angles[4 * t + role] < N) aev[angles[4 * t + role]].push_back(t * 3 + role);
  auto flatten = [N](const std::vector<std::vector<int>>& ev, std::vector<int>& off, std::vector<int>& flat) {
    off.assign(N + 1, 0);
    for (int b = 0; b < N; ++b) off[b + 1] = off[b] + (int)ev[b].size();
    flat.clear();
    for (const auto& v : ev) flat.insert(flat.end(), v.begin(), v.end());
  };
  std::vector<int> boff, bflat, aoff, aflat;
  flatten(bev, boff, bflat);
  flatten(aev, aoff, aflat);

  ForceField* f = new ForceField();
  s->ff = f;
  f->lj = d->lennard_jones;
  f->lj_alpha = d->lennard_jones_alpha;
  f->scale = d->unit_scale;
  f->nb = d->n_bonds;
  f->na = d->n_angles;
  bool ok = true;
  auto chk = [&](int r) {
    if (r != PBG_OK) ok = false;
  };
  if (f->lj != PBG_LJ_NONE) {
    chk(upload(&f->hc, d->hard_core_radius, (size_t)total));
    if (ok) chk(upload(&f->eps, d->epsilon_lj, (size_t)total));
    if (ok) chk(alloc(&f->flj, (size_t)3 * N));
    if (ok) chk(alloc(&f->elj, (size_t)N));
  }
  if (ok && f->nb) {
    chk(upload(&f->bonds, bonds.data(), bonds.size()));
    if (ok) chk(upload(&f->bond_p, d->bond_params, (size_t)2 * f->nb));
    if (ok) chk(upload(&f->bond_off, boff.data(), boff.size()));
    if (ok && !bflat.empty()) chk(upload(&f->bond_ev, bflat.data(), bflat.size()));
    if (ok) chk(alloc(&f->bf, (size_t)3 * f->nb));
    if (ok) chk(alloc(&f->be, (size_t)f->nb));
  }
  if (ok && f->na) {
    chk(upload(&f->angles, angles.data(), angles.size()));
    if (ok) chk(upload(&f->angle_p, d->angle_params, (size_t)2 * f->na));
    if (ok) chk(upload(&f->angle_off, aoff.data(), aoff.size()));
    if (ok && !aflat.empty()) chk(upload(&f->angle_ev, aflat.data(), aflat.size()));
    if (ok) chk(alloc(&f->af, (size_t)9 * f->na));
    if (ok) chk(alloc(&f->ae, (size_t)f->na));
  }
  if (ok) chk(alloc(&s->ftot, (size_t)s->ld));
  if (ok) chk(alloc(&s->energy, 1));
  if (ok && cudaMemset(s->ftot, 0, (size_t)s->ld * sizeof(double)) != cudaSuccess) ok = false;
  if (ok && cudaMemset(s->energy, 0, sizeof(double)) != cudaSuccess) ok = false;
  if (!ok) {
    cudaGetLastError();
    free_interactions(s);
    return PBG_ERR_NOMEM;
  }
  return PBG_OK;
}

int compute_forces(pbg_system* s, cudaStream_t st) {
  ForceField* f = s->ff;
  if (!f) return PBG_OK;
  const Beads bs = beads_of(s);
  const int N = s->N;
  if (f->lj != PBG_LJ_NONE) {
    lj_kernel<<<(N * 32 + 255) / 256, 256, 0, st>>>(bs, f->lj, f->lj_alpha, f->hc, f->eps, f->flj, f->elj);
    PBG_CHECK_LAUNCH();
  }
  if (f->nb) {
    bond_kernel<<<(f->nb + 127) / 128, 128, 0, st>>>(bs, f->nb, f->bonds, f->bond_p, f->bf, f->be);
    PBG_CHECK_LAUNCH();
  }
  if (f->na) {
    angle_kernel<<<(f->na + 127) / 128, 128, 0, st>>>(bs, f->na, f->angles, f->angle_p, f->af, f->ae);
    PBG_CHECK_LAUNCH();
  }
  combine_kernel<<<(N + 127) / 128, 128, 0, st>>>(N, f->scale, s->force, f->lj != PBG_LJ_NONE, f->flj,
                                                  f->nb ? f->bond_off : nullptr, f->bond_ev, f->bf,
                                                  f->na ? f->angle_off : nullptr, f->angle_ev, f->af, s->ftot);
  PBG_CHECK_LAUNCH();
  energy_kernel<<<1, 256, 0, st>>>(N, f->lj != PBG_LJ_NONE, f->elj, f->nb, f->be, f->na, f->ae, s->energy);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

int overlap_immobile(pbg_system* s, int* flag, cudaStream_t st) {
  if (s->M == 0) return PBG_OK;
  const long long total = (long long)s->N * s->M;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
  overlap_immobile_kernel<<<blocks, 256, 0, st>>>(beads_of(s), s->radii, s->radii_imm, s->order, s->conn_mi,
                                                  s->p.overlap_treshold, flag);
  PBG_CHECK_LAUNCH();
  return PBG_OK;
}

}  // namespace pbg
