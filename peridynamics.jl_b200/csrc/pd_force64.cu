// pd_force64.cu -- FP64 force-density kernels (the plain FP64 path).
//
// Compiled with -fmad=false: Julia rounds every product and sum separately, and these kernels
// keep the reference's evaluation order, so with one lane per point (G = 1, "exact order")
// the per-point results equal the serial CPU restatement bit for bit:
//   - BB: one bond sweep (failure test, then the bond force) in bond order;
//   - OSB / CMat: phase A per point (failure, damage, weighted volume and dilatation, or the
//     deformation gradient and stress), phase B gathers the force density. The reference
//     scatters b_j -= p V_i while it processes point i; phase B reproduces the order in which
//     those scattered terms reach b_i in the serial loop: first the terms of neighbours j < i
//     (ascending j), then the own bonds of i, then the terms of neighbours j > i.
// With G > 1 lanes per point the same arithmetic is summed in a fixed butterfly order
// (deterministic, not bit-identical to the serial order).
#include "pd_common.cuh"
#include "pd_launch.h"

namespace pd {

__device__ __forceinline__ double4 ld4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
// StaticArrays 3x3 det / inv (column-major), as the CPU restatement
__device__ __forceinline__ double det3(const double* A) {
  double c[3];
  cross3(A + 3, A + 6, c);
  return dot3(A, c);
}
__device__ __forceinline__ void inv3(const double* A, double* R) {
  double x0[3] = {A[0], A[1], A[2]};
  double y0[3], y1[3], y2[3];
  cross3(A + 3, A + 6, y0);
  double d = dot3(x0, y0);
  for (int k = 0; k < 3; k++) { x0[k] = x0[k] / d; y0[k] = y0[k] / d; }
  cross3(A + 6, x0, y1);
  cross3(x0, A + 3, y2);
  for (int c = 0; c < 3; c++) { R[3 * c] = y0[c]; R[1 + 3 * c] = y1[c]; R[2 + 3 * c] = y2[c]; }
}
__device__ __forceinline__ void matmul3(const double* A, const double* B, double* C) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      C[r + 3 * c] = (A[r] * B[3 * c] + A[r + 3] * B[1 + 3 * c]) + A[r + 6] * B[2 + 3 * c];
}
__device__ __forceinline__ void matTmul3(const double* A, const double* B, double* C) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      C[r + 3 * c] = (A[3 * r] * B[3 * c] + A[1 + 3 * r] * B[1 + 3 * c]) + A[2 + 3 * r] * B[2 + 3 * c];
}
__device__ __forceinline__ void matmulT3(const double* A, const double* B, double* C) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      C[r + 3 * c] = (A[r] * B[c] + A[r + 3] * B[c + 3]) + A[r + 6] * B[c + 6];
}
__device__ __forceinline__ void matvec3(const double* A, const double* v, double* w) {
  for (int r = 0; r < 3; r++) w[r] = (A[r] * v[0] + A[r + 3] * v[1]) + A[r + 6] * v[2];
}

// ZEMWan stiffness (zem_stabilization.jl:32-42): C_1[i,j] = sum over k (outer), l (inner) of
// C[i,j,k,l] Kinv[k,l], all 81 products in that order, with C the Hooke tensor that
// get_hooke_matrix builds from the Voigt matrix (constitutive_models.jl:107-133): Voigt index
// of (i,j) in the order (1,1), (2,2), (3,3), (2,3), (1,3), (1,2); a = (1 - nu) lambda / nu on the
// diagonal of the normal block, lambda off it, mu on the diagonal of the shear block.
__device__ __forceinline__ int voigt_of(int i, int j) {
  if (i == j) return i;
  const int m = i + j;
  return m == 3 ? 3 : (m == 2 ? 4 : 5);
}
__device__ __forceinline__ double hooke_of(const DevParam& p, int i, int j, int k, int l) {
  const int I = voigt_of(i, j), J = voigt_of(k, l);
  if (I < 3 && J < 3) return I == J ? p.zwa : p.lambda;
  if (I >= 3 && J >= 3) return I == J ? p.mu : 0.0;
  return 0.0;
}
__device__ void zem_wan64(const DevParam& p, const double* Kinv, double* C1) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) s += hooke_of(p, i, j, k, l) * Kinv[k + 3 * l];
      C1[i + 3 * j] = s;
    }
}

// first_piola_kirchhoff (constitutive_models.jl:35-41, 169-176, 233-244)
__device__ void pk1_64(int cmodel, const DevParam& p, const double* F, double* P) {
  double C[9], S[9];
  if (cmodel == CM_SVK) {
    double E[9];
    matTmul3(F, F, C);
    for (int k = 0; k < 9; k++) E[k] = 0.5 * (C[k] - ((k % 4) == 0 ? 1.0 : 0.0));
    double trE = (E[0] + E[4]) + E[8];
    double a = p.lambda * trE, m2 = 2 * p.mu;
    for (int k = 0; k < 9; k++) S[k] = (k % 4) == 0 ? m2 * E[k] + a : m2 * E[k];
  } else if (cmodel == CM_NEOHOOKE) {
    double J = det3(F), Ci[9];
    matTmul3(F, F, C);
    inv3(C, Ci);
    double lj = p.lambda * log(J);
    for (int k = 0; k < 9; k++) S[k] = p.mu * ((k % 4) == 0 ? -Ci[k] + 1.0 : -Ci[k]) + lj * Ci[k];
  } else {
    double J = det3(F);
    if (J < 2.220446049250313e-16 || isnan(J)) {
      for (int k = 0; k < 9; k++) P[k] = 0.0;
      return;
    }
    double Ci[9];
    matTmul3(F, F, C);
    inv3(C, Ci);
    double trC = (C[0] + C[4]) + C[8];
    double a = 1.0 / 3.0 * trC;
    double jp = pow(J, -2.0 / 3.0);
    double ij = 1.0 / J;
    double vol = p.K / 4 * (J * J - ij * ij);
    for (int k = 0; k < 9; k++)
      S[k] = p.G * ((k % 4) == 0 ? -(a * Ci[k]) + 1.0 : -(a * Ci[k])) * jp + vol * Ci[k];
  }
  matmul3(F, S, P);
}

__device__ __forceinline__ void flag_nan(const DevBody& d, int kstep, double x, double y, double z) {
  if (isnan(x) || isnan(y) || isnan(z)) {
    long long step = d.ctrl->base + kstep;
    if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
    else atomicMin(&d.ctrl->err_step, step);
  }
}

// new bond_active word of a row after the failure tests of its lanes; the warp owns the word
__device__ __forceinline__ void commit_row64(unsigned int* bits, long long word_idx, unsigned old,
                                             bool act, int lane) {
  const unsigned nw = __ballot_sync(0xffffffffu, act);
  if (lane == 0 && nw != old) bits[word_idx] = nw;
}

// -------------------------------------------------------------------------------------------
// BB: bond_based.jl:125-180 (calc_failure! storing the bond length, force_density_point!)
// -------------------------------------------------------------------------------------------
// FAST (mappings other than the serial order): the force uses one division per bond,
// (l - L) / (L l), in place of the reference's (l - L) / L and three divisions by l; the
// forces differ from the serial order by a few units in the last place, as the lane-group sums
// already do. The failure decision keeps the reference's expression.
// ESC: the bond's surface correction factor multiplies its force (bond_based.jl:156, 175)
// rows of neighbour gathers in flight per lane in the FAST loop. Measured on the 500k-point
// bending beam at 4 lanes per point (first two load increments, identical Krylov steps): 2 rows
// (80 registers, three blocks of 256 per SM) block Jacobi 6.59 s / block polynomial 3.00 s; 3 rows
// 7.37 / 3.26 s; 4 rows (116 registers, two blocks per SM) 7.02 / 3.13 s.
#ifndef PD_BB64_ROWS
#define PD_BB64_ROWS 2
#endif
template <int G, bool MULTI, bool FAST, bool ESC>
__global__ void __launch_bounds__(256, FAST && PD_BB64_ROWS <= 2 ? 3 : 2) k_bb64(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double bx = 0.0, by = 0.0, bz = 0.0;
    int na = 0;
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    if (FAST) {
      // PD_BB64_ROWS rows per iteration: as many independent neighbour gathers in flight per
      // lane; the bonds are still added row by row
      constexpr int RU = PD_BB64_ROWS;
      const int self = valid ? (int)i : 0;
      for (int r = 0; r < rows; r += RU) {
        const long long wi = (sbase >> 5) + r;
        unsigned w[RU];
        int j[RU];
        double Lsv[RU];
        bool hv[RU], act[RU];
        double4 xv[RU];
#pragma unroll
        for (int u = 0; u < RU; u++) {
          const bool in = r + u < rows;
          w[u] = in ? d.bits[wi + u] : 0u;
          hv[u] = in && (r + u) * G + gl < cnt;
          const long long b = sbase + (long long)(r + u) * 32 + lane;
          j[u] = hv[u] ? __ldg(d.nbr + b) : self;
          Lsv[u] = hv[u] ? __ldg(d.len64 + b) : 1.0;
        }
#pragma unroll
        for (int u = 0; u < RU; u++) xv[u] = ld4(d.cur + j[u]);
#pragma unroll
        for (int u = 0; u < RU; u++) {
          act[u] = false;
          if (!hv[u]) continue;
          const double4 xj = xv[u];
          const double Ls = Lsv[u];
          const double L = fabs(Ls);
          const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
          const double l = sqrt((dx * dx + dy * dy) + dz * dz);
          // the failure test keeps the reference's eps = (l - L) / L (bonds that may fail only)
          const bool brk = Ls > 0 && (l - L) / L > P.epsc;
          act[u] = ((w[u] >> lane) & 1u) && !brk;
          const double q = (l - L) / (L * l);  // eps / l
          const double bcb =
              MULTI ? 0.5 * (P.bc + d.params[d.meta[j[u]] & META_PID_MASK].bc) : P.bc;
          const double bet = ESC ? __ldg(d.sc64 + sbase + (long long)(r + u) * 32 + lane) : 1.0;
          const double sc = act[u] ? bet * bcb * q * xj.w : 0.0;
          bx += sc * dx;
          by += sc * dy;
          bz += sc * dz;
        }
#pragma unroll
        for (int u = 0; u < RU; u++) {
          na += act[u];
          if (r + u < rows) commit_row64(d.bits, wi + u, w[u], act[u], lane);
        }
      }
    } else
    for (int r = 0; r < rows; r++) {
      const long long wi = (sbase >> 5) + r;
      const unsigned word = d.bits[wi];
      const int k = r * G + gl;
      bool act = false;
      if (k < cnt) {
        const long long b = sbase + (long long)r * 32 + lane;
        const int j = __ldg(d.nbr + b);
        const double Ls = __ldg(d.len64 + b);
        const double L = fabs(Ls);
        const double4 xj = ld4(d.cur + j);
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        {
          const double eps = (l - L) / L;
          act = ((word >> lane) & 1u) && !(eps > P.epsc && Ls > 0);
          const double om = act ? (ESC ? __ldg(d.sc64 + b) : 1.0) : 0.0;
          double sc;
          if (MULTI) {
            const double bcj = d.params[d.meta[j] & META_PID_MASK].bc;
            sc = om * (P.bc + bcj) / 2 * eps * xj.w;
          } else {
            sc = om * P.bc * eps * xj.w;
          }
          bx += sc * dx / l;
          by += sc * dy / l;
          bz += sc * dz / l;
        }
      }
      na += act;
      commit_row64(d.bits, wi, word, act, lane);
    }
    if (G > 1) {
      bx = group_sum<G>(bx); by = group_sum<G>(by); bz = group_sum<G>(bz); na = group_sum<G>(na);
    }
    if (valid && gl == 0) {
      d.b64[3 * i] = bx; d.b64[3 * i + 1] = by; d.b64[3 * i + 2] = bz;
      d.n_active[i] = na;
      flag_nan(d, kstep, bx, by, bz);
    }
  }
}

// -------------------------------------------------------------------------------------------
// OSB phase A: calc_failure! (ordinary_state_based.jl:107-126), calc_damage!,
// calc_weighted_volume (:176-189), calc_dilatation (:191-204), c1, c2 (:135-136)
// -------------------------------------------------------------------------------------------
// ESC: the bond factor beta in the weighted volume and the dilatation (:182, :198)
template <int G, bool EXACT, bool ESC>
__global__ void PD_LB64 k_osb_a64(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double wvol = 0.0, sdil = 0.0;
    int na = 0;
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const double4 Xi = valid ? ld4(d.X0 + i) : make_double4(0, 0, 0, 0);
    for (int r = 0; r < rows; r++) {
      const long long wi = (sbase >> 5) + r;
      const unsigned word = d.bits[wi];
      const int k = r * G + gl;
      bool act = false;
      if (k < cnt) {
        const long long b = sbase + (long long)r * 32 + lane;
        const int j = __ldg(d.nbr + b);
        const double Ls = __ldg(d.len64 + b);
        const double L = fabs(Ls);
        const double4 xj = ld4(d.cur + j), Xj = ld4(d.X0 + j);
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        const double eps = (l - L) / L;
        act = ((word >> lane) & 1u) && !(eps > P.epsc && Ls > 0);
        const double DX = Xj.x - Xi.x, DY = Xj.y - Xi.y, DZ = Xj.z - Xi.z;
        const double om = act ? omega_of(d.kernel, P.delta, L) : 0.0;
        const double bet = ESC ? __ldg(d.sc64 + b) : 1.0;
        wvol += om * bet * ((DX * DX + DY * DY) + DZ * DZ) * xj.w;
        if (!EXACT) sdil += om * bet * L * (l - L) * xj.w;
      }
      na += act;
      commit_row64(d.bits, wi, word, act, lane);
    }
    if (G > 1) {
      wvol = group_sum<G>(wvol); sdil = group_sum<G>(sdil); na = group_sum<G>(na);
    }
    double dil = 0.0;
    if (EXACT) {
      // second sweep of the reference with c1 = 3 / wvol inside every term; the bits were
      // written above by lane 0 of the warp, so the decision is recomputed from the same eps
      __syncwarp();
      const double c1d = 3.0 / wvol;
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        if (k >= cnt || wvol == 0.0) continue;
        const long long b = sbase + (long long)r * 32 + lane;
        const int j = __ldg(d.nbr + b);
        const double Ls = __ldg(d.len64 + b);
        const double L = fabs(Ls);
        const double4 xj = ld4(d.cur + j);
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        const double eps = (l - L) / L;
        const bool act = bond_bit_live(d.bits, b) && !(eps > P.epsc && Ls > 0);
        const double om = act ? omega_of(d.kernel, P.delta, L) : 0.0;
        dil += om * (ESC ? __ldg(d.sc64 + b) : 1.0) * c1d * L * (l - L) * xj.w;
      }
    } else if (wvol != 0.0) {
      dil = 3.0 / wvol * sdil;
    }
    if (valid && gl == 0) {
      double c1 = 0.0, c2 = 0.0;
      if (wvol != 0.0) {
        c1 = 15.0 * P.G / wvol;
        c2 = dil * (3.0 * P.K / wvol - c1 / 3.0);
      }
      d.coef64[i] = make_double4(c1, c2, wvol, dil);
      d.n_active[i] = na;
    }
  }
}

// p = omega beta (c2 L + c1 (l - L)) / l (ordinary_state_based.jl:144), coefficients of the
// bond owner o with the partner q (ParameterHandler form :165-166 when MULTI)
template <bool MULTI>
__device__ __forceinline__ double osb_s64(const double4& co, const DevParam& Po, const DevParam& Pq,
                                          double om, double bet, double L, double l) {
  double c1, c2;
  if (MULTI) {
    c1 = 15.0 * (Po.G + Pq.G) / (2 * co.z);
    c2 = co.w * (3.0 * (Po.K + Pq.K) / (2 * co.z) - c1 / 3.0);
  } else {
    c1 = co.x;
    c2 = co.y;
  }
  return om * bet * (c2 * L + c1 * (l - L)) / l;
}

// -------------------------------------------------------------------------------------------
// OSB phase B: force_density_point! (ordinary_state_based.jl:128-174) in gather form
// -------------------------------------------------------------------------------------------
// ESC: beta of the bond, which is also the factor of its reverse bond (equal by construction)
template <int G, bool EXACT, bool MULTI, bool ESC>
__global__ void PD_LB64 k_osb_b64(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double bx = 0.0, by = 0.0, bz = 0.0;
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const double4 ci = valid ? d.coef64[i] : make_double4(0, 0, 0, 0);
    const bool own = ci.z != 0.0;
    // own term of the bond in slot b
    auto own_term = [&](long long b) {
      const int j = __ldg(d.nbr + b);
      const double L = fabs(__ldg(d.len64 + b));
      const double4 xj = ld4(d.cur + j);
      const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
      const double l = sqrt((dx * dx + dy * dy) + dz * dz);
      const bool act = bond_bit(d.bits, b);
      const double om = act ? omega_of(d.kernel, Pi.delta, L) : 0.0;
      const DevParam& Pj = MULTI ? d.params[d.meta[j] & META_PID_MASK] : Pi;
      const double sc = osb_s64<MULTI>(ci, Pi, Pj, om, ESC ? __ldg(d.sc64 + b) : 1.0, L, l);
      bx += sc * dx * xj.w;
      by += sc * dy * xj.w;
      bz += sc * dz * xj.w;
    };
    // term that j's loop scatters into b_i through its bond j -> i
    auto nbr_term = [&](long long b) {
      const int j = __ldg(d.nbr + b);
      const double4 cj = d.coef64[j];
      if (cj.z == 0.0) return;  // j returned early (iszero(wvol))
      const double L = fabs(__ldg(d.len64 + b));
      const double4 xj = ld4(d.cur + j);
      const double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      const double l = sqrt((dx * dx + dy * dy) + dz * dz);
      const bool act = d.sym ? bond_bit(d.bits, b) : bond_bit(d.bits, rev_slot(d, b, j));
      const DevParam& Pj = d.params[d.meta[j] & META_PID_MASK];
      const double om = act ? omega_of(d.kernel, Pj.delta, L) : 0.0;
      const double sc = osb_s64<MULTI>(cj, Pj, Pi, om, ESC ? __ldg(d.sc64 + b) : 1.0, L, l);
      bx += -(sc * dx) * xj.w;
      by += -(sc * dy) * xj.w;
      bz += -(sc * dz) * xj.w;
    };
    if (EXACT) {
      // the serial scatter order: neighbours j < i, own bonds, neighbours j > i
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        const long long b = sbase + (long long)r * 32 + lane;
        if (k < cnt && __ldg(d.nbr + b) < i) nbr_term(b);
      }
      if (own)
        for (int r = 0; r < rows; r++) {
          const int k = r * G + gl;
          if (k < cnt) own_term(sbase + (long long)r * 32 + lane);
        }
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        const long long b = sbase + (long long)r * 32 + lane;
        if (k < cnt && __ldg(d.nbr + b) > i) nbr_term(b);
      }
    } else {
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        if (k >= cnt) continue;
        const long long b = sbase + (long long)r * 32 + lane;
        if (own) own_term(b);
        nbr_term(b);
      }
    }
    if (G > 1) { bx = group_sum<G>(bx); by = group_sum<G>(by); bz = group_sum<G>(bz); }
    if (valid && gl == 0) {
      d.b64[3 * i] = bx; d.b64[3 * i + 1] = by; d.b64[3 * i + 2] = bz;
      flag_nan(d, kstep, bx, by, bz);
    }
  }
}

// -------------------------------------------------------------------------------------------
// OSB phases for the mappings other than the serial order: two rows per iteration (two
// neighbour gathers in flight per lane), the weighted volume from the stored bond length
// (L^2 for |X_j - X_i|^2, equal to a few units in the last place), and in phase B the point's
// own term and its neighbour's term of a bond summed before one division by l. The failure
// test keeps the reference's eps = (l - L) / L. Results differ from the serial order by a few
// units in the last place, as the lane-group sums already do.
// -------------------------------------------------------------------------------------------
template <int G, bool ESC>
__global__ void __launch_bounds__(256, 3) k_osb_a64f(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double wvol = 0.0, sdil = 0.0;
    int na = 0;
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const int self = valid ? (int)i : 0;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const long long wi = (sbase >> 5) + r;
      const unsigned w0 = d.bits[wi], w1 = two ? d.bits[wi + 1] : 0u;
      const int k0 = r * G + gl, k1 = k0 + G;
      const bool h0 = k0 < cnt, h1 = two && k1 < cnt;
      const long long b0 = sbase + (long long)r * 32 + lane, b1 = b0 + 32;
      const int j0 = h0 ? __ldg(d.nbr + b0) : self, j1 = h1 ? __ldg(d.nbr + b1) : self;
      const double Ls0 = h0 ? __ldg(d.len64 + b0) : 1.0, Ls1 = h1 ? __ldg(d.len64 + b1) : 1.0;
      const double4 x0 = ld4(d.cur + j0), x1 = ld4(d.cur + j1);
      bool act0 = false, act1 = false;
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (!(u ? h1 : h0)) continue;
        const double4 xj = u ? x1 : x0;
        const double Ls = u ? Ls1 : Ls0;
        const double L = fabs(Ls);
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        const double eps = (l - L) / L;
        const bool act = (((u ? w1 : w0) >> lane) & 1u) && !(eps > P.epsc && Ls > 0);
        if (act) {
          const double bet = ESC ? __ldg(d.sc64 + (u ? b1 : b0)) : 1.0;
          const double t = omega_of(d.kernel, P.delta, L) * bet * xj.w;
          wvol += t * (L * L);
          sdil += t * L * (l - L);
        }
        if (u) act1 = act; else act0 = act;
      }
      na += act0 + act1;
      commit_row64(d.bits, wi, w0, act0, lane);
      if (two) commit_row64(d.bits, wi + 1, w1, act1, lane);
    }
    if (G > 1) {
      wvol = group_sum<G>(wvol); sdil = group_sum<G>(sdil); na = group_sum<G>(na);
    }
    if (valid && gl == 0) {
      double c1 = 0.0, c2 = 0.0, dil = 0.0;
      if (wvol != 0.0) {
        dil = 3.0 / wvol * sdil;
        c1 = 15.0 * P.G / wvol;
        c2 = dil * (3.0 * P.K / wvol - c1 / 3.0);
      }
      d.coef64[i] = make_double4(c1, c2, wvol, dil);
      d.n_active[i] = na;
    }
  }
}

// omega beta (c2 L + c1 (l - L)) of a bond owner o with partner q: osb_s64 before its division
template <bool MULTI>
__device__ __forceinline__ double osb_num64(const double4& co, const DevParam& Po, const DevParam& Pq,
                                            double om, double bet, double L, double l) {
  double c1, c2;
  if (MULTI) {
    c1 = 15.0 * (Po.G + Pq.G) / (2 * co.z);
    c2 = co.w * (3.0 * (Po.K + Pq.K) / (2 * co.z) - c1 / 3.0);
  } else {
    c1 = co.x;
    c2 = co.y;
  }
  return om * bet * (c2 * L + c1 * (l - L));
}

template <int G, bool MULTI, bool ESC>
__global__ void __launch_bounds__(256, 2) k_osb_b64f(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double bx = 0.0, by = 0.0, bz = 0.0;
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const double4 ci = valid ? d.coef64[i] : make_double4(0, 0, 0, 0);
    const bool own = ci.z != 0.0;
    const int self = valid ? (int)i : 0;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const long long wi = (sbase >> 5) + r;
      const unsigned w0 = __ldg(d.bits + wi), w1 = two ? __ldg(d.bits + wi + 1) : 0u;
      const int k0 = r * G + gl, k1 = k0 + G;
      const bool h0 = k0 < cnt, h1 = two && k1 < cnt;
      const long long b0 = sbase + (long long)r * 32 + lane, b1 = b0 + 32;
      const int j0 = h0 ? __ldg(d.nbr + b0) : self, j1 = h1 ? __ldg(d.nbr + b1) : self;
      const double Ls0 = h0 ? __ldg(d.len64 + b0) : 1.0, Ls1 = h1 ? __ldg(d.len64 + b1) : 1.0;
      const double4 x0 = ld4(d.cur + j0), x1 = ld4(d.cur + j1);
      const double4 c0 = d.coef64[j0], c1 = d.coef64[j1];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (!(u ? h1 : h0)) continue;
        const double4 xj = u ? x1 : x0;
        const double4 cj = u ? c1 : c0;
        const int j = u ? j1 : j0;
        const long long b = u ? b1 : b0;
        const double L = fabs(u ? Ls1 : Ls0);
        const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        const bool ai = ((u ? w1 : w0) >> lane) & 1u;
        const bool aj = d.sym ? ai : bond_bit(d.bits, rev_slot(d, b, j));
        const DevParam& Pj = d.params[d.meta[j] & META_PID_MASK];
        const double bet = ESC ? __ldg(d.sc64 + b) : 1.0;
        double num = 0.0;
        if (own && ai) num += osb_num64<MULTI>(ci, Pi, Pj, omega_of(d.kernel, Pi.delta, L), bet, L, l);
        // j returned early for a zero weighted volume (iszero(wvol))
        if (cj.z != 0.0 && aj)
          num += osb_num64<MULTI>(cj, Pj, Pi, omega_of(d.kernel, Pj.delta, L), bet, L, l);
        const double sc = num / l * xj.w;
        bx += sc * dx;
        by += sc * dy;
        bz += sc * dz;
      }
    }
    if (G > 1) { bx = group_sum<G>(bx); by = group_sum<G>(by); bz = group_sum<G>(bz); }
    if (valid && gl == 0) {
      d.b64[3 * i] = bx; d.b64[3 * i + 1] = by; d.b64[3 * i + 2] = bz;
      flag_nan(d, kstep, bx, by, bz);
    }
  }
}

// -------------------------------------------------------------------------------------------
// CMat phase A: calc_failure! (bond_system.jl:309-327), calc_damage!,
// calc_deformation_gradient! (correspondence.jl:193-214), too_much_damage! (:288-298),
// calc_first_piola_kirchhoff! (:216-224)
// -------------------------------------------------------------------------------------------
template <int G>
__global__ void PD_LB64 k_c_a64(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double K[9], Ft[9];
    for (int q = 0; q < 9; q++) { K[q] = 0.0; Ft[q] = 0.0; }
    int na = 0;
    const unsigned meta = valid ? d.meta[i] : 0u;
    const DevParam& P = d.params[meta & META_PID_MASK];
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const double4 Xi = valid ? ld4(d.X0 + i) : make_double4(0, 0, 0, 0);
    for (int r = 0; r < rows; r++) {
      const long long wi = (sbase >> 5) + r;
      const unsigned word = d.bits[wi];
      const int k = r * G + gl;
      bool act = false;
      if (k < cnt) {
        const long long b = sbase + (long long)r * 32 + lane;
        const int j = __ldg(d.nbr + b);
        const double Ls = __ldg(d.len64 + b);
        const double L = fabs(Ls);
        const double4 xj = ld4(d.cur + j), Xj = ld4(d.X0 + j);
        const double dx[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
        const double l = sqrt(dot3(dx, dx));
        const double eps = (l - L) / L;
        act = ((word >> lane) & 1u) && !(eps > P.epsc && Ls > 0);
        const double DX[3] = {Xj.x - Xi.x, Xj.y - Xi.y, Xj.z - Xi.z};
        const double om = act ? omega_of(d.kernel, P.delta, L) : 0.0;
        const double temp = om * xj.w;
        for (int c = 0; c < 3; c++)
          for (int q = 0; q < 3; q++) {
            K[q + 3 * c] = K[q + 3 * c] + temp * (DX[q] * DX[c]);
            Ft[q + 3 * c] = Ft[q + 3 * c] + temp * (dx[q] * DX[c]);
          }
      }
      na += act;
      commit_row64(d.bits, wi, word, act, lane);
    }
    if (G > 1) {
      for (int q = 0; q < 9; q++) { K[q] = group_sum<G>(K[q]); Ft[q] = group_sum<G>(Ft[q]); }
      na = group_sum<G>(na);
    }
    bool killed = false;
    if (valid && gl == 0) {
      const double damage = 1.0 - (double)na / (double)cnt;
      double Kinv[9], F[9];
      inv3(K, Kinv);
      matmul3(Ft, Kinv, F);
      bool hasnan = false;
      for (int q = 0; q < 9; q++) { d.F64[9 * i + q] = F[q]; hasnan |= isnan(F[q]); }
      // a halo row sees only part of its bonds: its owner decides (the kill arrives with the
      // halo exchange of the phase-A state)
      killed = (meta & META_KILLED) || (!(meta & META_HALO) && (damage > d.maxdmg || hasnan));
      if (killed) {
        if (!(meta & META_KILLED)) d.meta[i] = meta | META_KILLED;
        na = 0;
      } else {
        double Pm[9], PKinv[9];
        pk1_64(d.cmodel, P, F, Pm);
        matmul3(Pm, Kinv, PKinv);
        for (int q = 0; q < 9; q++) d.PK64[9 * i + q] = PKinv[q];
        if (d.zem == ZEM_WAN) {
          double C1[9];
          zem_wan64(P, Kinv, C1);
          for (int q = 0; q < 9; q++) d.C164[9 * i + q] = C1[q];
        }
      }
      d.n_active[i] = na;
    }
    if (!d.sym) {
      // directed bond states: a killed point loses all its bonds (correspondence.jl:293)
      if (G > 1) killed = group_bcast<G>(killed);
      const unsigned kill_mask = __ballot_sync(0xffffffffu, valid && killed);
      if (kill_mask && lane == 0)
        for (int r = 0; r < rows; r++) d.bits[(sbase >> 5) + r] &= ~kill_mask;
    }
  }
}

// -------------------------------------------------------------------------------------------
// CMat phase B: c_force_density! (correspondence.jl:226-279) in gather form; the stabilisation
// term is (w beta) z for ZEMSilling (C1 null) and (w C_1) z for ZEMWan
// -------------------------------------------------------------------------------------------
__device__ __forceinline__ void c_bond_t64(const double* F, const double* PK, const double* C1,
                                           double beta, double om, const double* DX,
                                           const double* dx, double* t) {
  double FD[3], z[3], W[9], WD[3], tz[3];
  matvec3(F, DX, FD);
  for (int q = 0; q < 3; q++) z[q] = dx[q] - FD[q];
  if (C1) {
    double W1[9];
    for (int q = 0; q < 9; q++) W1[q] = om * C1[q];
    matvec3(W1, z, tz);
  } else {
    const double ob = om * beta;
    for (int q = 0; q < 3; q++) tz[q] = ob * z[q];
  }
  for (int q = 0; q < 9; q++) W[q] = om * PK[q];
  matvec3(W, DX, WD);
  for (int q = 0; q < 3; q++) t[q] = WD[q] + tz[q];
}

template <int G, bool EXACT>
__global__ void PD_LB64 k_c_b64(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    double bx = 0.0, by = 0.0, bz = 0.0;
    const double4 xi = valid ? ld4(d.cur + i) : make_double4(0, 0, 0, 0);
    const double4 Xi = valid ? ld4(d.X0 + i) : make_double4(0, 0, 0, 0);
    const unsigned mi = valid ? d.meta[i] : META_KILLED;
    const DevParam& Pi = d.params[mi & META_PID_MASK];
    const bool own = !(mi & META_KILLED);
    const bool wan = d.zem == ZEM_WAN;
    double Fi[9], PKi[9], Ci[9];
    for (int q = 0; q < 9; q++) {
      Fi[q] = own ? d.F64[9 * i + q] : 0.0;
      PKi[q] = own ? d.PK64[9 * i + q] : 0.0;
      Ci[q] = own && wan ? d.C164[9 * i + q] : 0.0;
    }
    auto own_term = [&](long long b) {
      const int j = __ldg(d.nbr + b);
      const double L = fabs(__ldg(d.len64 + b));
      const double4 xj = ld4(d.cur + j), Xj = ld4(d.X0 + j);
      const double DX[3] = {Xj.x - Xi.x, Xj.y - Xi.y, Xj.z - Xi.z};
      const double dx[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
      const bool act = bond_bit(d.bits, b);
      const double om = act ? omega_of(d.kernel, Pi.delta, L) : 0.0;
      double t[3];
      c_bond_t64(Fi, PKi, wan ? Ci : nullptr, Pi.beta, om, DX, dx, t);
      bx += t[0] * xj.w; by += t[1] * xj.w; bz += t[2] * xj.w;
    };
    auto nbr_term = [&](long long b) {
      const int j = __ldg(d.nbr + b);
      const unsigned mj = d.meta[j];
      if (mj & META_KILLED) return;  // j returned early after too_much_damage!
      const double L = fabs(__ldg(d.len64 + b));
      const bool act = d.sym ? bond_bit(d.bits, b) : bond_bit(d.bits, rev_slot(d, b, j));
      const DevParam& Pj = d.params[mj & META_PID_MASK];
      const double4 xj = ld4(d.cur + j), Xj = ld4(d.X0 + j);
      const double DX[3] = {Xi.x - Xj.x, Xi.y - Xj.y, Xi.z - Xj.z};
      const double dx[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
      const double om = act ? omega_of(d.kernel, Pj.delta, L) : 0.0;
      double Fj[9], PKj[9], Cj[9], t[3];
      for (int q = 0; q < 9; q++) { Fj[q] = d.F64[9 * (long long)j + q]; PKj[q] = d.PK64[9 * (long long)j + q]; }
      if (wan)
        for (int q = 0; q < 9; q++) Cj[q] = d.C164[9 * (long long)j + q];
      c_bond_t64(Fj, PKj, wan ? Cj : nullptr, Pj.beta, om, DX, dx, t);
      bx += -t[0] * xj.w; by += -t[1] * xj.w; bz += -t[2] * xj.w;
    };
    if (EXACT) {
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        const long long b = sbase + (long long)r * 32 + lane;
        if (k < cnt && __ldg(d.nbr + b) < i) nbr_term(b);
      }
      if (own)
        for (int r = 0; r < rows; r++) {
          const int k = r * G + gl;
          if (k < cnt) own_term(sbase + (long long)r * 32 + lane);
        }
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        const long long b = sbase + (long long)r * 32 + lane;
        if (k < cnt && __ldg(d.nbr + b) > i) nbr_term(b);
      }
    } else {
      for (int r = 0; r < rows; r++) {
        const int k = r * G + gl;
        if (k >= cnt) continue;
        const long long b = sbase + (long long)r * 32 + lane;
        if (own) own_term(b);
        nbr_term(b);
      }
    }
    if (G > 1) { bx = group_sum<G>(bx); by = group_sum<G>(by); bz = group_sum<G>(bz); }
    if (valid && gl == 0) {
      d.b64[3 * i] = bx; d.b64[3 * i + 1] = by; d.b64[3 * i + 2] = bz;
      flag_nan(d, kstep, bx, by, bz);
    }
  }
}

// cauchy_stress (stress.jl:112-116) of the stored F, for the export of the CMat stress field
__global__ void k_cauchy64(DevBody d, const double* F, int from_h32, double* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam P = d.params[d.meta[i] & META_PID_MASK];
  double Fm[9], Pm[9], Ps[9], S[9];
  for (int k = 0; k < 9; k++)
    Fm[k] = from_h32 ? (double)d.H32[9 * i + k] + ((k % 4) == 0 ? 1.0 : 0.0) : F[9 * i + k];
  pk1_64(d.cmodel, P, Fm, Pm);
  const double J = det3(Fm), iJ = 1 / J;
  for (int k = 0; k < 9; k++) Ps[k] = iJ * Pm[k];
  matmulT3(Ps, Fm, S);
  const bool killed = d.meta[i] & META_KILLED;
  for (int k = 0; k < 9; k++) out[9 * i + k] = killed ? 0.0 : S[k];
}

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------
#define PD_DISPATCH_G(G, CALL)                  \
  switch (G) {                                  \
    case 1: { constexpr int GG = 1; CALL; } break;  \
    case 2: { constexpr int GG = 2; CALL; } break;  \
    case 4: { constexpr int GG = 4; CALL; } break;  \
    case 8: { constexpr int GG = 8; CALL; } break;  \
    case 16: { constexpr int GG = 16; CALL; } break; \
    default: { constexpr int GG = 32; CALL; } break; \
  }

static int grid_for(long long nslices, int block) {
  long long warps = nslices;
  long long blocks = (warps + block / 32 - 1) / (block / 32);
  if (blocks < 1) blocks = 1;
  if (PD_GRID_BLOCKS_PER_SM > 0 && blocks > 148LL * PD_GRID_BLOCKS_PER_SM)
    blocks = 148LL * PD_GRID_BLOCKS_PER_SM;
  return (int)blocks;
}

template <bool ESC>
static void launch_bb64(const DevBody& d, const LaunchCfg& c, int G, int grid, int kstep, cudaStream_t s) {
  if (c.exact) {
    if (d.multi) k_bb64<1, true, false, ESC><<<grid, c.block, 0, s>>>(d, kstep);
    else k_bb64<1, false, false, ESC><<<grid, c.block, 0, s>>>(d, kstep);
  } else if (d.multi) {
    PD_DISPATCH_G(G, (k_bb64<GG, true, true, ESC><<<grid, c.block, 0, s>>>(d, kstep)));
  } else {
    PD_DISPATCH_G(G, (k_bb64<GG, false, true, ESC><<<grid, c.block, 0, s>>>(d, kstep)));
  }
}

template <bool ESC>
static int launch_osb64(const DevBody& d, const LaunchCfg& c, int G, int grid, int kstep, bool A,
                        bool B, cudaStream_t s) {
  int launches = 0;
  if (A) {
    if (c.exact) k_osb_a64<1, true, ESC><<<grid, c.block, 0, s>>>(d, kstep);
    else { PD_DISPATCH_G(G, (k_osb_a64f<GG, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
    launches++;
  }
  if (B) {
    if (c.exact) {
      if (d.multi) k_osb_b64<1, true, true, ESC><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_b64<1, true, false, ESC><<<grid, c.block, 0, s>>>(d, kstep);
    } else if (d.multi) {
      PD_DISPATCH_G(G, (k_osb_b64f<GG, true, ESC><<<grid, c.block, 0, s>>>(d, kstep)));
    } else {
      PD_DISPATCH_G(G, (k_osb_b64f<GG, false, ESC><<<grid, c.block, 0, s>>>(d, kstep)));
    }
    launches++;
  }
  return launches;
}

int launch_force64(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s) {
  const int G = d.lg;
  const int grid = grid_for(d.nslices, c.block);
  const bool A = phase != 2, B = phase != 1;
  int launches = 0;
  if (d.material == MAT_BB) {
    if (!A) return 0;
    if (d.sc64) launch_bb64<true>(d, c, G, grid, kstep, s);
    else launch_bb64<false>(d, c, G, grid, kstep, s);
    return 1;
  }
  if (d.material == MAT_OSB) {
    if (d.sc64) return launch_osb64<true>(d, c, G, grid, kstep, A, B, s);
    return launch_osb64<false>(d, c, G, grid, kstep, A, B, s);
  }
  if (A) {
    PD_DISPATCH_G(G, (k_c_a64<GG><<<grid, c.block, 0, s>>>(d, kstep)));
    launches++;
  }
  if (B) {
    if (c.exact) k_c_b64<1, true><<<grid, c.block, 0, s>>>(d, kstep);
    else { PD_DISPATCH_G(G, (k_c_b64<GG, false><<<grid, c.block, 0, s>>>(d, kstep))); }
    launches++;
  }
  return launches;
}

void launch_cauchy64(const DevBody& d, const double* F, int from_h32, double* out, cudaStream_t s) {
  int grid = (int)((d.n + 255) / 256);
  if (grid < 1) grid = 1;
  k_cauchy64<<<grid, 256, 0, s>>>(d, F, from_h32, out);
}

}  // namespace pd
