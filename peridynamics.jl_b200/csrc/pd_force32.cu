// pd_force32.cu -- FP32-compensated force-density kernels (the fast path).
//
// Per bond, in FP32:
//   du  = (float)(u_j - u_i)           difference of the FP64 displacements, then rounded
//   eta = xi + du                       deformed bond vector from the stored FP32 offset xi
//   l   = |eta|
//   e   = l - L = (2 xi.du + du.du) / (l + L)   (no cancellation at stretches ~1e-4)
// Per-point sums use Kahan-compensated FP32 accumulation and a fixed-order compensated
// reduction over the G lanes of a point, so results are deterministic.
//
// The state-based materials run in gather form (phase A per point, phase B per point reading
// the phase-A state of the neighbours) instead of the reference's scatter b_j -= p V_i.
// With symmetric bond lists and symmetric bond states one bit per bond serves both
// directions; otherwise the reverse-bond index gives the state of bond j -> i.
//
// Correspondence in FP32 uses the displacement gradient H = F - I (so that F - I does not
// cancel) and a horizon-scaled shape tensor K' = K / delta^5 (the unscaled det K underflows
// FP32 for millimetre lattices). The stress formulas are the reference's, rewritten in
// terms of E = (H + H^T + H^T H) / 2 without cancelling subtractions.
#include "pd_common.cuh"
#include "pd_launch.h"
#include "pd_pack.cuh"

namespace pd {

__device__ __forceinline__ double4 ld4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

struct BondF {
  float gx, gy, gz, L, rL;
  float dux, duy, duz;
  float ex, ey, ez, l, rl, e, eps;
  bool fp;
};

// One bond in FP32: the cancellation-free extension e = l - L, the stretch, and the inverse
// lengths (reciprocal and reciprocal square root; the FP32 path is not bit-matched).
__device__ __forceinline__ void bond32(const float4 g, const float4& hi, const float4& lo,
                                       const float4& hj, const float4& lj, BondF& B) {
  B.gx = g.x; B.gy = g.y; B.gz = g.z;
  B.L = fabsf(g.w);
  B.rL = __fdividef(1.f, B.L);
  B.fp = g.w > 0.f;
  B.dux = (hj.x - hi.x) + (lj.x - lo.x);
  B.duy = (hj.y - hi.y) + (lj.y - lo.y);
  B.duz = (hj.z - hi.z) + (lj.z - lo.z);
  B.ex = g.x + B.dux; B.ey = g.y + B.duy; B.ez = g.z + B.duz;
  const float l2 = B.ex * B.ex + B.ey * B.ey + B.ez * B.ez;
  B.rl = rsqrtf(l2);
  B.l = l2 * B.rl;
  const float xd = g.x * B.dux + g.y * B.duy + g.z * B.duz;
  const float dd = B.dux * B.dux + B.duy * B.duy + B.duz * B.duz;
  B.e = __fdividef(2.f * xd + dd, B.l + B.L);
  B.eps = B.e * B.rL;
}

// influence function with the reciprocal length at hand
__device__ __forceinline__ float omega_r(int kernel, float delta, float L, float rL) {
  if (kernel == KER_LINEAR) return delta * rL;
  return omega_of_f(kernel, delta, L);
}

// LIN: the reference's default linear kernel delta / L chosen at compile time. The phase-A
// kernels instantiate it: without the general form's code per bond, OSB phase A took 3 % and
// CMat phase A 5.6 % less time on the 1M-point blocks (the same values bit for bit). Phase B
// keeps the general form, which measured faster there.
template <bool LIN>
__device__ __forceinline__ float omega_t(int kernel, float delta, float L, float rL) {
  if constexpr (LIN) return delta * rL;
  else return omega_r(kernel, delta, L, rL);
}

__device__ __forceinline__ void flag_nan32(const DevBody& d, int kstep, float x, float y, float z) {
  if (isnan(x) || isnan(y) || isnan(z)) {
    long long step = d.ctrl->base + kstep;
    if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
    else atomicMin(&d.ctrl->err_step, step);
  }
}

// failure test of CriticalStretch (bond_system.jl:309-327): eps > eps_c with permission
__device__ __forceinline__ bool fails32(const BondF& B, float epsc) {
  return B.eps > epsc && B.fp;
}

// new bond_active word of a row after the failure tests of its lanes; the warp owns the word
__device__ __forceinline__ void commit_row(unsigned int* bits, long long word_idx, unsigned old,
                                           bool act, int lane) {
  const unsigned nw = __ballot_sync(0xffffffffu, act);
  if (lane == 0 && nw != old) bits[word_idx] = nw;
}

// -------------------------------------------------------------------------------------------
// BB (bond_based.jl:125-180): one sweep, failure then the pairwise force
// -------------------------------------------------------------------------------------------
// ESC: the bond's surface correction factor multiplies its force (bond_based.jl:156, 175)
template <int G, bool MULTI, bool ESC>
__global__ void PD_LB k_bb32(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum bx, by, bz;
    int na = 0;
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float epsc = P.epscf, bci = P.bcf;
    for (int r = 0; r < rows; r++) {
      const long long wi = (sbase >> 5) + r;
      const unsigned word = d.bits[wi];
      const int k = r * G + gl;
      bool act = false;
      if (k < cnt) {
        const long long b = sbase + (long long)r * 32 + lane;
        const int j = __ldg(d.nbr + b);
        const float4 g = __ldg(d.geo + b);
        const float bet = ESC ? __ldg(d.sc32 + b) : 1.f;  // loaded with the bond record
        const float4 hj = __ldg(d.uhi + j), lj = __ldg(d.ulo + j);
        BondF B;
        bond32(g, hi, lo, hj, lj, B);
        act = ((word >> lane) & 1u) && !fails32(B, epsc);
        if (act) {
          float bc = bci;
          if (MULTI) bc = 0.5f * (bci + d.params[d.meta[j] & META_PID_MASK].bcf);
          float sc = bc * B.eps * hj.w * B.rl;
          if (ESC) sc *= bet;
          bx.add(sc * B.ex); by.add(sc * B.ey); bz.add(sc * B.ez);
        }
      }
      na += act;
      commit_row(d.bits, wi, word, act, lane);
    }
    if (G > 1) { group_reduce<G>(bx); group_reduce<G>(by); group_reduce<G>(bz); na = group_sum<G>(na); }
    if (valid && gl == 0) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      d.n_active[i] = na;
      flag_nan32(d, kstep, x, y, z);
    }
  }
}

// Two-row BB (pipe 4): the bond records and neighbour gathers of rows r and r + 1 are issued
// before either row is processed (two dependent gathers in flight per lane, as the OSB
// two-row kernels); each lane adds its bonds in row order, so the sums equal k_bb32's.
// Measured on the 1M-point BB block: 0.581 ms per step at 4 resident blocks (64 registers),
// 0.602 ms at 3, 0.725 ms at 5.
#ifndef PD_MINB_UBB
#define PD_MINB_UBB 4
#endif
template <int G, bool MULTI, bool ESC>
__global__ void __launch_bounds__(256, PD_MINB_UBB) k_bb32u(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum bx, by, bz;
    int na = 0;
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float epsc = P.epscf, bci = P.bcf;
    const int self = valid ? (int)i : 0;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const long long wi = (sbase >> 5) + r;
      const unsigned w0 = d.bits[wi], w1 = two ? d.bits[wi + 1] : 0u;
      const int k0 = r * G + gl;
      const bool h0 = k0 < cnt, h1 = two && k0 + G < cnt;
      const long long b0 = sbase + (long long)r * 32 + lane;
      int j0 = self, j1 = self;
      float4 g0 = make_float4(0.f, 0.f, 0.f, 1.f), g1 = g0;
      float s0 = 1.f, s1 = 1.f;
      if (h0) { j0 = __ldg(d.nbr + b0); g0 = __ldg(d.geo + b0); if (ESC) s0 = __ldg(d.sc32 + b0); }
      if (h1) { j1 = __ldg(d.nbr + b0 + 32); g1 = __ldg(d.geo + b0 + 32); if (ESC) s1 = __ldg(d.sc32 + b0 + 32); }
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      bool act0 = false, act1 = false;
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (!(u ? h1 : h0)) continue;
        const float4 hj = u ? hj1 : hj0;
        BondF B;
        bond32(u ? g1 : g0, hi, lo, hj, u ? lj1 : lj0, B);
        const bool act = (((u ? w1 : w0) >> lane) & 1u) && !fails32(B, epsc);
        if (act) {
          float bc = bci;
          if (MULTI) bc = 0.5f * (bci + d.params[d.meta[u ? j1 : j0] & META_PID_MASK].bcf);
          float sc = bc * B.eps * hj.w * B.rl;
          if (ESC) sc *= u ? s1 : s0;
          bx.add(sc * B.ex); by.add(sc * B.ey); bz.add(sc * B.ez);
        }
        if (u) act1 = act; else act0 = act;
      }
      na += act0 + act1;
      commit_row(d.bits, wi, w0, act0, lane);
      if (two) commit_row(d.bits, wi + 1, w1, act1, lane);
    }
    if (G > 1) { group_reduce<G>(bx); group_reduce<G>(by); group_reduce<G>(bz); na = group_sum<G>(na); }
    if (valid && gl == 0) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      d.n_active[i] = na;
      flag_nan32(d, kstep, x, y, z);
    }
  }
}

// -------------------------------------------------------------------------------------------
// OSB phase A (ordinary_state_based.jl:107-126, 176-204): failure, weighted volume m,
// dilatation theta, and c1 = 15 G / m, c2 = theta (3 K / m - c1 / 3) (:135-136)
// -------------------------------------------------------------------------------------------
// ESC: the bond factor beta in the weighted volume and the dilatation (:182, :198).
// FULLM: the weighted volume m depends on the reference bonds and their states only; it is
// summed over the active bonds when FULLM (the first evaluation, or after bond states changed
// outside the kernels), otherwise the stored m of the point loses the terms of the bonds that
// break in this evaluation.
template <int G, bool ESC, bool FULLM>
__global__ void PD_LB_A k_osb_a32(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum m, th;
    float dm = 0.f;
    int na = 0;
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float epsc = P.epscf, delta = P.deltaf;
    const long long b0 = sbase + lane;
    int jn = 0;
    float4 gn = make_float4(0.f, 0.f, 0.f, 0.f);
    float sn = 1.f;
    if (rows > 0 && gl < cnt) {
      jn = __ldg(d.nbr + b0); gn = __ldg(d.geo + b0);
      if (ESC) sn = __ldg(d.sc32 + b0);
    }
    for (int r = 0; r < rows; r++) {
      const long long wi = (sbase >> 5) + r;
      const unsigned word = d.bits[wi];
      const int k = r * G + gl;
      const int j = jn;
      const float4 g = gn;
      const float bet = sn;
      if (r + 1 < rows && k + G < cnt) {
        const long long b1 = b0 + (long long)(r + 1) * 32;
        jn = __ldg(d.nbr + b1);
        gn = __ldg(d.geo + b1);
        if (ESC) sn = __ldg(d.sc32 + b1);
      }
      bool act = false;
      if (k < cnt) {
        const float4 hj = __ldg(d.uhi + j), lj = __ldg(d.ulo + j);
        BondF B;
        bond32(g, hi, lo, hj, lj, B);
        act = ((word >> lane) & 1u) && !fails32(B, epsc);
        if (act) {
          float om = omega_r(d.kernel, delta, B.L, B.rL) * hj.w;
          if (ESC) om *= bet;
          if (FULLM) m.add(om * (B.gx * B.gx + B.gy * B.gy + B.gz * B.gz));
          th.add(om * B.L * B.e);
        } else if (!FULLM && ((word >> lane) & 1u)) {  // breaks now: leaves the stored m
          float om = omega_r(d.kernel, delta, B.L, B.rL) * hj.w;
          if (ESC) om *= bet;
          dm += om * (B.gx * B.gx + B.gy * B.gy + B.gz * B.gz);
        }
      }
      na += act;
      commit_row(d.bits, wi, word, act, lane);
    }
    if (G > 1) {
      if (FULLM) group_reduce<G>(m); else dm = group_sum<G>(dm);
      group_reduce<G>(th); na = group_sum<G>(na);
    }
    if (valid && gl == 0) {
      const float wv = FULLM ? m.value() : (dm != 0.f ? d.cm32[i].x - dm : d.cm32[i].x);
      float c1 = 0.f, c2 = 0.f, dil = 0.f;
      if (wv != 0.f) {
        dil = 3.f / wv * th.value();
        c1 = 15.f * P.Gf / wv;
        c2 = dil * (3.f * P.Kf / wv - c1 / 3.f);
      }
      d.cc32[i] = make_float2(c1, c2);
      d.cm32[i] = make_float2(wv, dil);
      d.n_active[i] = na;
    }
  }
}

// s = omega (c2 L + c1 e) of the bond owner o with partner q; with ParameterHandler
// semantics (ordinary_state_based.jl:165-166) c1, c2 come from (wvol, dil) and both moduli
template <bool MULTI>
__device__ __forceinline__ float osb_s32(const float2& c, const float2& m, const DevParam& Po,
                                         const DevParam& Pq, float om, float L, float e) {
  float c1 = c.x, c2 = c.y;
  if (MULTI) {
    if (m.x == 0.f) return 0.f;
    c1 = 15.f * (Po.Gf + Pq.Gf) / (2.f * m.x);
    c2 = m.y * (3.f * (Po.Kf + Pq.Kf) / (2.f * m.x) - c1 / 3.f);
  }
  return om * (c2 * L + c1 * e);
}

// -------------------------------------------------------------------------------------------
// OSB phase B (ordinary_state_based.jl:128-174): b_i = sum_j (s_ij + s_ji) V_j eta / l
// -------------------------------------------------------------------------------------------
// ESC: beta of the bond, which is also the factor of its reverse bond (equal by construction)
template <int G, bool MULTI, bool ESC>
__global__ void PD_LB k_osb_b32(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum bx, by, bz;
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float2 ci = valid ? d.cc32[i] : make_float2(0.f, 0.f);
    const float2 mi = (MULTI && valid) ? d.cm32[i] : make_float2(0.f, 0.f);
    // the bond stream of row r + 1 is loaded while row r is processed
    const unsigned* wrow = d.bits + (sbase >> 5);
    const long long b0 = sbase + lane;
    int jn = 0;
    float4 gn = make_float4(0.f, 0.f, 0.f, 0.f);
    float sn = 1.f;
    unsigned wn = 0;
    if (rows > 0) {
      wn = __ldg(wrow);
      if (gl < cnt) {
        jn = __ldg(d.nbr + b0); gn = __ldg(d.geo + b0);
        if (ESC) sn = __ldg(d.sc32 + b0);
      }
    }
    for (int r = 0; r < rows; r++) {
      const int j = jn;
      const float4 g = gn;
      const float bet = sn;
      const unsigned word = wn;
      const int k = r * G + gl;
      if (r + 1 < rows) {
        wn = __ldg(wrow + r + 1);
        if (k + G < cnt) {
          const long long b1 = b0 + (long long)(r + 1) * 32;
          jn = __ldg(d.nbr + b1);
          gn = __ldg(d.geo + b1);
          if (ESC) sn = __ldg(d.sc32 + b1);
        }
      }
      if (k >= cnt) continue;
      const long long b = b0 + (long long)r * 32;
      const bool ai = (word >> lane) & 1u;
      const bool aj = d.sym ? ai : bond_bit(d.bits, rev_slot(d, b, j));
      if (!(ai || aj)) continue;
      const float4 hj = __ldg(d.uhi + j), lj = __ldg(d.ulo + j);
      const float2 cj = __ldg(d.cc32 + j);
      const float2 mj = MULTI ? __ldg(d.cm32 + j) : make_float2(0.f, 0.f);
      BondF B;
      bond32(g, hi, lo, hj, lj, B);
      const DevParam* Pj = &Pi;
      if (MULTI) Pj = &d.params[d.meta[j] & META_PID_MASK];
      const float oi = ai ? omega_r(d.kernel, Pi.deltaf, B.L, B.rL) : 0.f;
      const float oj = aj ? omega_r(d.kernel, Pj->deltaf, B.L, B.rL) : 0.f;
      const float si = osb_s32<MULTI>(ci, mi, Pi, *Pj, oi, B.L, B.e);
      const float sj = osb_s32<MULTI>(cj, mj, *Pj, Pi, oj, B.L, B.e);
      float f = (si + sj) * hj.w * B.rl;
      if (ESC) f *= bet;
      bx.add(f * B.ex); by.add(f * B.ey); bz.add(f * B.ez);
    }
    if (G > 1) { group_reduce<G>(bx); group_reduce<G>(by); group_reduce<G>(bz); }
    if (valid && gl == 0) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      flag_nan32(d, kstep, x, y, z);
    }
  }
}

// -------------------------------------------------------------------------------------------
// Two-row variants of the OSB kernels (pipe 4): the neighbour indices of rows r and r + 1
// are loaded together and all their gathers issued before either row is processed, so two
// dependent gathers are in flight per lane. Each lane still adds its bonds in row order:
// the results equal the one-row kernels' bit for bit. Measured on the 8M-point block (one
// lane per point): 10.8 -> 9.4 ms per step with both kernels held to 4 blocks per SM (60 and
// 63 registers, no spills); three or four rows per iteration, or register arrays in place
// of the named pairs, were slower.
// -------------------------------------------------------------------------------------------
#ifndef PD_MINB_UA
#define PD_MINB_UA 4
#endif
#ifndef PD_MINB_UB
#define PD_MINB_UB 4
#endif
template <int G, bool ESC, bool FULLM, bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_UA) k_osb_a32u(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum m, th;
    float dm = 0.f;
    int na = 0;
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float epsc = P.epscf, delta = P.deltaf;
    const int self = valid ? (int)i : 0;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const long long wi = (sbase >> 5) + r;
      const unsigned w0 = d.bits[wi], w1 = two ? d.bits[wi + 1] : 0u;
      const int k0 = r * G + gl;
      const bool h0 = k0 < cnt, h1 = two && k0 + G < cnt;
      const long long b0 = sbase + (long long)r * 32 + lane;
      int j0 = self, j1 = self;
      float4 g0 = make_float4(0.f, 0.f, 0.f, 1.f), g1 = g0;
      float s0 = 1.f, s1 = 1.f;
      if (h0) { j0 = __ldg(d.nbr + b0); g0 = __ldg(d.geo + b0); if (ESC) s0 = __ldg(d.sc32 + b0); }
      if (h1) { j1 = __ldg(d.nbr + b0 + 32); g1 = __ldg(d.geo + b0 + 32); if (ESC) s1 = __ldg(d.sc32 + b0 + 32); }
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      bool act0 = false, act1 = false;
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (!(u ? h1 : h0)) continue;
        const float4 hj = u ? hj1 : hj0;
        BondF B;
        bond32(u ? g1 : g0, hi, lo, hj, u ? lj1 : lj0, B);
        const bool act = (((u ? w1 : w0) >> lane) & 1u) && !fails32(B, epsc);
        if (act) {
          float om = omega_t<LIN>(d.kernel, delta, B.L, B.rL) * hj.w;
          if (ESC) om *= u ? s1 : s0;
          if (FULLM) m.add(om * (B.gx * B.gx + B.gy * B.gy + B.gz * B.gz));
          th.add(om * B.L * B.e);
        } else if (!FULLM && (((u ? w1 : w0) >> lane) & 1u)) {  // breaks now (see k_osb_a32)
          float om = omega_t<LIN>(d.kernel, delta, B.L, B.rL) * hj.w;
          if (ESC) om *= u ? s1 : s0;
          dm += om * (B.gx * B.gx + B.gy * B.gy + B.gz * B.gz);
        }
        if (u) act1 = act; else act0 = act;
      }
      na += act0 + act1;
      commit_row(d.bits, wi, w0, act0, lane);
      if (two) commit_row(d.bits, wi + 1, w1, act1, lane);
    }
    if (G > 1) {
      if (FULLM) group_reduce<G>(m); else dm = group_sum<G>(dm);
      group_reduce<G>(th); na = group_sum<G>(na);
    }
    if (valid && gl == 0) {
      const float wv = FULLM ? m.value() : (dm != 0.f ? d.cm32[i].x - dm : d.cm32[i].x);
      float c1 = 0.f, c2 = 0.f, dil = 0.f;
      if (wv != 0.f) {
        dil = 3.f / wv * th.value();
        c1 = 15.f * P.Gf / wv;
        c2 = dil * (3.f * P.Kf / wv - c1 / 3.f);
      }
      d.cc32[i] = make_float2(c1, c2);
      d.cm32[i] = make_float2(wv, dil);
      d.n_active[i] = na;
    }
  }
}

template <int G, bool MULTI, bool ESC>
__global__ void __launch_bounds__(256, PD_MINB_UB) k_osb_b32u(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum bx, by, bz;
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float2 ci = valid ? d.cc32[i] : make_float2(0.f, 0.f);
    const float2 mi = (MULTI && valid) ? d.cm32[i] : make_float2(0.f, 0.f);
    const unsigned* wrow = d.bits + (sbase >> 5);
    const int self = valid ? (int)i : 0;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const unsigned w0 = __ldg(wrow + r), w1 = two ? __ldg(wrow + r + 1) : 0u;
      const int k0 = r * G + gl;
      const long long b0 = sbase + (long long)r * 32 + lane;
      bool h0 = k0 < cnt, h1 = two && k0 + G < cnt;
      int j0 = self, j1 = self;
      float4 g0 = make_float4(0.f, 0.f, 0.f, 1.f), g1 = g0;
      float s0 = 1.f, s1 = 1.f;
      if (h0) { j0 = __ldg(d.nbr + b0); g0 = __ldg(d.geo + b0); if (ESC) s0 = __ldg(d.sc32 + b0); }
      if (h1) { j1 = __ldg(d.nbr + b0 + 32); g1 = __ldg(d.geo + b0 + 32); if (ESC) s1 = __ldg(d.sc32 + b0 + 32); }
      const bool ai0 = (w0 >> lane) & 1u, ai1 = (w1 >> lane) & 1u;
      const bool aj0 = h0 && (d.sym ? ai0 : bond_bit(d.bits, rev_slot(d, b0, j0)));
      const bool aj1 = h1 && (d.sym ? ai1 : bond_bit(d.bits, rev_slot(d, b0 + 32, j1)));
      h0 = h0 && (ai0 || aj0);
      h1 = h1 && (ai1 || aj1);
      if (!h0) j0 = self;
      if (!h1) j1 = self;
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      const float2 cj0 = __ldg(d.cc32 + j0), cj1 = __ldg(d.cc32 + j1);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (!(u ? h1 : h0)) continue;
        const int j = u ? j1 : j0;
        const float4 hj = u ? hj1 : hj0;
        const float2 cj = u ? cj1 : cj0;
        const float2 mj = MULTI ? __ldg(d.cm32 + j) : make_float2(0.f, 0.f);
        BondF B;
        bond32(u ? g1 : g0, hi, lo, hj, u ? lj1 : lj0, B);
        const DevParam* Pj = &Pi;
        if (MULTI) Pj = &d.params[d.meta[j] & META_PID_MASK];
        const bool ai = u ? ai1 : ai0, aj = u ? aj1 : aj0;
        const float oi = ai ? omega_r(d.kernel, Pi.deltaf, B.L, B.rL) : 0.f;
        const float oj = aj ? omega_r(d.kernel, Pj->deltaf, B.L, B.rL) : 0.f;
        const float si = osb_s32<MULTI>(ci, mi, Pi, *Pj, oi, B.L, B.e);
        const float sj = osb_s32<MULTI>(cj, mj, *Pj, Pi, oj, B.L, B.e);
        float f = (si + sj) * hj.w * B.rl;
        if (ESC) f *= u ? s1 : s0;
        bx.add(f * B.ex); by.add(f * B.ey); bz.add(f * B.ez);
      }
    }
    if (G > 1) { group_reduce<G>(bx); group_reduce<G>(by); group_reduce<G>(bz); }
    if (valid && gl == 0) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      flag_nan32(d, kstep, x, y, z);
    }
  }
}

// ------------------------------------------------------------------------------------------
// FP32 3x3 helpers (column-major) for the correspondence material
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void fcross(const float* a, const float* b, float* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ void finv3(const float* A, float* R) {
  float x0[3] = {A[0], A[1], A[2]}, y0[3], y1[3], y2[3];
  fcross(A + 3, A + 6, y0);
  const float d = x0[0] * y0[0] + x0[1] * y0[1] + x0[2] * y0[2];
  for (int k = 0; k < 3; k++) { x0[k] /= d; y0[k] /= d; }
  fcross(A + 6, x0, y1);
  fcross(x0, A + 3, y2);
  for (int c = 0; c < 3; c++) { R[3 * c] = y0[c]; R[1 + 3 * c] = y1[c]; R[2 + 3 * c] = y2[c]; }
}
__device__ __forceinline__ void fmatmul(const float* A, const float* B, float* C) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      C[r + 3 * c] = A[r] * B[3 * c] + A[r + 3] * B[1 + 3 * c] + A[r + 6] * B[2 + 3 * c];
}

// P(F = I + H) of the reference's models, written without the cancelling F^T F - I
__device__ void pk1_32(int cmodel, const DevParam& p, const float* H, float* P) {
  float E[9], S[9], HS[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      const float hth = H[3 * r] * H[3 * c] + H[1 + 3 * r] * H[1 + 3 * c] + H[2 + 3 * r] * H[2 + 3 * c];
      E[r + 3 * c] = 0.5f * (H[r + 3 * c] + H[c + 3 * r] + hth);
    }
  const float trE = E[0] + E[4] + E[8];
  if (cmodel == CM_SVK) {
    // S = lambda tr(E) I + 2 mu E
    for (int k = 0; k < 9; k++) S[k] = 2.f * p.muf * E[k] + ((k % 4) == 0 ? p.lambdaf * trE : 0.f);
  } else {
    // J - 1 = tr H + (principal 2x2 minors of H) + det H
    const float m2 = (H[0] * H[4] - H[3] * H[1]) + (H[0] * H[8] - H[6] * H[2]) + (H[4] * H[8] - H[7] * H[5]);
    float dH;
    {
      float c[3];
      fcross(H + 3, H + 6, c);
      dH = H[0] * c[0] + H[1] * c[1] + H[2] * c[2];
    }
    const float jm1 = (H[0] + H[4] + H[8]) + m2 + dH;
    const float J = 1.f + jm1;
    float C[9], Ci[9], T[9];
    for (int k = 0; k < 9; k++) C[k] = 2.f * E[k] + ((k % 4) == 0 ? 1.f : 0.f);
    finv3(C, Ci);
    if (cmodel == CM_NEOHOOKE) {
      // S = mu (I - C^-1) + lambda ln J C^-1 = C^-1 (2 mu E + lambda ln J I)
      const float lj = p.lambdaf * log1pf(jm1);
      for (int k = 0; k < 9; k++) T[k] = 2.f * p.muf * E[k] + ((k % 4) == 0 ? lj : 0.f);
    } else {
      // NeoHookePenalty: S = C^-1 (2 G J^(-2/3) dev E + K/4 (J^2 - J^-2) I), P = 0 if J < eps
      if (!(J >= 2.220446049250313e-16f)) {
        for (int k = 0; k < 9; k++) P[k] = 0.f;
        return;
      }
      const float jp = expf(-2.f / 3.f * log1pf(jm1));
      const float iJ = 1.f / J;
      const float vol = 0.25f * p.Kf * (jm1 * (J + 1.f) * iJ) * (J + iJ);
      for (int k = 0; k < 9; k++)
        T[k] = 2.f * p.Gf * jp * (E[k] - ((k % 4) == 0 ? trE / 3.f : 0.f)) + ((k % 4) == 0 ? vol : 0.f);
    }
    fmatmul(Ci, T, S);
  }
  // P = F S = S + H S
  fmatmul(H, S, HS);
  for (int k = 0; k < 9; k++) P[k] = S[k] + HS[k];
}

// -------------------------------------------------------------------------------------------
// CMat phase A (correspondence.jl:193-224, 288-298; bond_system.jl:309-327)
// -------------------------------------------------------------------------------------------
// The phase-B state of a live point, from the scaled inverse shape tensor Kinv (the true
// K^-1 = Kinv / delta^5), P K^-1 (scaled the same way) and H = F - I. The bond term
// w (P K^-1 xi + S (dx - F xi)) is w (A xi + S du) with A = P K^-1 - S H, where S is the
// stabilising stiffness: ZEMSilling beta I (c_force_density!, correspondence.jl:226-251; beta
// in cst32), ZEMWan C : K^-1 (correspondence.jl:253-285, zem_stabilization.jl:32-42; the six
// entries of the symmetric S in zw32, from the nonzero entries of the Hooke tensor: a = (1 - nu)
// lambda / nu and lambda in the normal block, mu (both index orders) in the shear block).
__device__ __forceinline__ void c_state_store32(const DevBody& d, const DevParam& P, long long i,
                                                const float* PK, const float* Kinv, const float* H,
                                                float id5) {
  float A[9];
  float4* cs = d.cst32 + 3 * i;
  if (d.zem == ZEM_WAN) {
    const float a = P.zwaf, l = P.lambdaf, m = P.muf;
    const float S0 = (a * Kinv[0] + l * Kinv[4] + l * Kinv[8]) * id5;
    const float S1 = (l * Kinv[0] + a * Kinv[4] + l * Kinv[8]) * id5;
    const float S2 = (l * Kinv[0] + l * Kinv[4] + a * Kinv[8]) * id5;
    const float S01 = m * (Kinv[3] + Kinv[1]) * id5;
    const float S02 = m * (Kinv[6] + Kinv[2]) * id5;
    const float S12 = m * (Kinv[7] + Kinv[5]) * id5;
    const float Sm[9] = {S0, S01, S02, S01, S1, S12, S02, S12, S2};
    float SH[9];
    fmatmul(Sm, H, SH);
#pragma unroll
    for (int q = 0; q < 9; q++) A[q] = PK[q] * id5 - SH[q];
    d.zw32[2 * i] = make_float4(S0, S1, S2, S01);
    d.zw32[2 * i + 1] = make_float4(S02, S12, 0.f, 0.f);
  } else {
#pragma unroll
    for (int q = 0; q < 9; q++) A[q] = PK[q] * id5 - P.betaf * H[q];
  }
  cs[0] = make_float4(A[0], A[1], A[2], A[3]);
  cs[1] = make_float4(A[4], A[5], A[6], A[7]);
  cs[2] = make_float4(A[8], d.zem == ZEM_WAN ? 0.f : P.betaf, 0.f, 0.f);
}

// a killed point's phase-B state: no term of its own, none for its neighbours
__device__ __forceinline__ void c_state_clear32(const DevBody& d, long long i) {
  float4* cs = d.cst32 + 3 * i;
  cs[0] = make_float4(0.f, 0.f, 0.f, 0.f);
  cs[1] = make_float4(0.f, 0.f, 0.f, 0.f);
  cs[2] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (d.zem == ZEM_WAN) {
    d.zw32[2 * i] = make_float4(0.f, 0.f, 0.f, 0.f);
    d.zw32[2 * i + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// the correspondence phase A keeps 15 compensated 3x3 sums per point: it gets its own
// occupancy bound (PD_MINB_CA resident blocks per SM). Measured on the 1M-point CMat block:
// 1.50 / 1.44 / 1.49 ms at 2 / 3 / 4 blocks (109 / 80 / 64 registers).
#ifndef PD_MINB_CA
#define PD_MINB_CA 3
#endif
// The shape tensor K depends on the reference bonds and their states only. FULLK sums it over
// the active bonds (the first evaluation, or after bond states changed outside the kernels);
// otherwise the stored K of the point loses the terms of the bonds that break in this
// evaluation, and only the nine sums of the deformation gradient run over all bonds.
// the variant that updates the stored shape tensors keeps 9 compensated sums and the next row's
// bond record in flight. Measured on the 1M-point CMat block: phase A 0.97 ms at 3 resident
// blocks (80 registers), 1.01 ms at 4 (64, with spills); without the row prefetch 1.09 ms at 4
// and 1.22 ms at 3; the full-sum variant took 1.43 ms every step.
#ifndef PD_MINB_CAI
#define PD_MINB_CAI 3
#endif
template <int G, bool FULLK, bool LIN>
__global__ void __launch_bounds__(256, FULLK ? PD_MINB_CA : PD_MINB_CAI) k_c_a32(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum K[FULLK ? 6 : 1], Hs[9];
    float dK[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int na = 0;
    const unsigned meta = valid ? d.meta[i] : 0u;
    const DevParam& P = d.params[meta & META_PID_MASK];
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float epsc = P.epscf, id = P.inv_delta, vs = P.vscale;
    // the bond record of row r + 1 is loaded while row r is processed
    const long long b0 = sbase + lane;
    int jn = 0;
    float4 gn = make_float4(0.f, 0.f, 0.f, 0.f);
    if (rows > 0 && gl < cnt) { jn = __ldg(d.nbr + b0); gn = __ldg(d.geo + b0); }
    for (int r = 0; r < rows; r++) {
      const long long wi = (sbase >> 5) + r;
      const unsigned word = d.bits[wi];
      const int k = r * G + gl;
      const int j = jn;
      const float4 g = gn;
      if (r + 1 < rows && k + G < cnt) {
        const long long b1 = b0 + (long long)(r + 1) * 32;
        jn = __ldg(d.nbr + b1);
        gn = __ldg(d.geo + b1);
      }
      bool act = false;
      if (k < cnt) {
        const float4 hj = __ldg(d.uhi + j), lj = __ldg(d.ulo + j);
        BondF B;
        bond32(g, hi, lo, hj, lj, B);
        act = ((word >> lane) & 1u) && !fails32(B, epsc);
        if (act) {
          const float t = omega_t<LIN>(d.kernel, P.deltaf, B.L, B.rL) * hj.w * vs;
          const float X[3] = {B.gx * id, B.gy * id, B.gz * id};
          const float U[3] = {B.dux * id, B.duy * id, B.duz * id};
          if constexpr (FULLK) {
            K[0].add(t * X[0] * X[0]); K[1].add(t * X[1] * X[1]); K[2].add(t * X[2] * X[2]);
            K[3].add(t * X[0] * X[1]); K[4].add(t * X[0] * X[2]); K[5].add(t * X[1] * X[2]);
          }
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int q = 0; q < 3; q++) Hs[q + 3 * c].add(t * U[q] * X[c]);
        } else if (!FULLK && ((word >> lane) & 1u)) {
          // the bond breaks now: its term leaves the stored shape tensor
          const float t = omega_t<LIN>(d.kernel, P.deltaf, B.L, B.rL) * hj.w * vs;
          const float X[3] = {B.gx * id, B.gy * id, B.gz * id};
          dK[0] += t * X[0] * X[0]; dK[1] += t * X[1] * X[1]; dK[2] += t * X[2] * X[2];
          dK[3] += t * X[0] * X[1]; dK[4] += t * X[0] * X[2]; dK[5] += t * X[1] * X[2];
        }
      }
      na += act;
      commit_row(d.bits, wi, word, act, lane);
    }
    if (G > 1) {
      if constexpr (FULLK) {
#pragma unroll
        for (int q = 0; q < 6; q++) group_reduce<G>(K[q]);
      } else {
#pragma unroll
        for (int q = 0; q < 6; q++) dK[q] = group_sum<G>(dK[q]);
      }
#pragma unroll
      for (int q = 0; q < 9; q++) group_reduce<G>(Hs[q]);
      na = group_sum<G>(na);
    }
    bool killed = false;
    if (valid && gl == 0) {
      float k6[6];
      float2* ks = reinterpret_cast<float2*>(d.K32 + 6 * i);
      if constexpr (FULLK) {
#pragma unroll
        for (int q = 0; q < 6; q++) k6[q] = K[q].value();
        ks[0] = make_float2(k6[0], k6[1]); ks[1] = make_float2(k6[2], k6[3]); ks[2] = make_float2(k6[4], k6[5]);
      } else {
        const float2 a0 = ks[0], a1 = ks[1], a2 = ks[2];
        k6[0] = a0.x; k6[1] = a0.y; k6[2] = a1.x; k6[3] = a1.y; k6[4] = a2.x; k6[5] = a2.y;
        if (dK[0] != 0.f || dK[1] != 0.f || dK[2] != 0.f) {  // a bond broke
#pragma unroll
          for (int q = 0; q < 6; q++) k6[q] -= dK[q];
          ks[0] = make_float2(k6[0], k6[1]); ks[1] = make_float2(k6[2], k6[3]); ks[2] = make_float2(k6[4], k6[5]);
        }
      }
      const float Km[9] = {k6[0], k6[3], k6[4],
                           k6[3], k6[1], k6[5],
                           k6[4], k6[5], k6[2]};
      float Kinv[9], Hm[9], H[9];
      finv3(Km, Kinv);
      for (int q = 0; q < 9; q++) Hm[q] = Hs[q].value();
      fmatmul(Hm, Kinv, H);
      bool hasnan = false;
      for (int q = 0; q < 9; q++) { d.H32[9 * i + q] = H[q]; hasnan |= isnan(H[q]); }
      const double damage = 1.0 - (double)na / (double)cnt;
      // a halo row sees only part of its bonds: its owner decides (the kill arrives with the
      // halo exchange of the phase-A state)
      killed = (meta & META_KILLED) || (!(meta & META_HALO) && (damage > d.maxdmg || hasnan));
      if (killed) {
        if (!(meta & META_KILLED)) d.meta[i] = meta | META_KILLED;
        na = 0;
        c_state_clear32(d, i);
      } else {
        float Pm[9], PK[9];
        pk1_32(d.cmodel, P, H, Pm);
        fmatmul(Pm, Kinv, PK);
        c_state_store32(d, P, i, PK, Kinv, H, id * id * id * id * id);
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
// CMat phase B (correspondence.jl:226-279): with A = P K^-1 - S H (c_state_store32),
//   t_ij = w (A_i xi + S_i du), and j's term -t_ji = w (A_j xi + S_j du);
// S = beta I (ZEMSilling) or the symmetric C : K^-1 of the point (ZEMWan, template flag WAN)
// -------------------------------------------------------------------------------------------
// row q of S du for the symmetric S = {S00, S11, S22, S01, S02, S12}
__device__ __forceinline__ float sym_row(const float* S, int q, const float* du) {
  if (q == 0) return S[0] * du[0] + S[3] * du[1] + S[4] * du[2];
  if (q == 1) return S[3] * du[0] + S[1] * du[1] + S[5] * du[2];
  return S[4] * du[0] + S[5] * du[1] + S[2] * du[2];
}

// phase B with the next row's bond record in flight holds 80 registers at 3 resident blocks.
// Measured on the 1M-point CMat block: 0.95 ms at 3 blocks; 1.21 ms at 4 (64 registers, 120 B
// of spills); 1.12 ms for the kernel without the prefetch at 4.
#ifndef PD_MINB_CB
#define PD_MINB_CB 3
#endif
// SYM: symmetric bond states (one bit serves both directions), dispatched from d.sym; the
// variant without the reverse-bond lookup code took 1.1 % less time on the 1M-point block
template <int G, bool SYM, bool WAN>
__global__ void __launch_bounds__(256, PD_MINB_CB) k_c_b32(DevBody d, int kstep) {
  if (d.ctrl->err) return;
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    KSum bx, by, bz;
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    float Ai[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, bi = 0.f;
    if (valid) {
      const float4 a0 = d.cst32[3 * i], a1 = d.cst32[3 * i + 1], a2 = d.cst32[3 * i + 2];
      Ai[0] = a0.x; Ai[1] = a0.y; Ai[2] = a0.z; Ai[3] = a0.w;
      Ai[4] = a1.x; Ai[5] = a1.y; Ai[6] = a1.z; Ai[7] = a1.w; Ai[8] = a2.x;
      bi = a2.y;
    }
    float Wi[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if constexpr (WAN) {
      if (valid) {
        const float4 w0 = d.zw32[2 * i], w1 = d.zw32[2 * i + 1];
        Wi[0] = w0.x; Wi[1] = w0.y; Wi[2] = w0.z; Wi[3] = w0.w; Wi[4] = w1.x; Wi[5] = w1.y;
      }
    }
    // the bond record of row r + 1 is loaded while row r is processed (as k_osb_b32)
    const unsigned* wrow = d.bits + (sbase >> 5);
    const long long b0 = sbase + lane;
    int jn = 0;
    float4 gn = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned wn = 0;
    if (rows > 0) {
      wn = __ldg(wrow);
      if (gl < cnt) { jn = __ldg(d.nbr + b0); gn = __ldg(d.geo + b0); }
    }
    for (int r = 0; r < rows; r++) {
      const unsigned word = wn;
      const int j = jn;
      const float4 g = gn;
      const int k = r * G + gl;
      if (r + 1 < rows) {
        wn = __ldg(wrow + r + 1);
        if (k + G < cnt) {
          const long long b1 = b0 + (long long)(r + 1) * 32;
          jn = __ldg(d.nbr + b1);
          gn = __ldg(d.geo + b1);
        }
      }
      if (k >= cnt) continue;
      const long long b = b0 + (long long)r * 32;
      const bool ai = (word >> lane) & 1u;
      const bool aj = (SYM || d.sym) ? ai : bond_bit(d.bits, rev_slot(d, b, j));
      if (!(ai || aj)) continue;
      const float4 hj = __ldg(d.uhi + j), lj = __ldg(d.ulo + j);
      const float4 c0 = __ldg(d.cst32 + 3 * (long long)j), c1 = __ldg(d.cst32 + 3 * (long long)j + 1),
                   c2 = __ldg(d.cst32 + 3 * (long long)j + 2);
      const float L = fabsf(g.w);
      const float du[3] = {(hj.x - hi.x) + (lj.x - lo.x), (hj.y - hi.y) + (lj.y - lo.y),
                           (hj.z - hi.z) + (lj.z - lo.z)};
      const float oi = ai ? omega_of_f(d.kernel, Pi.deltaf, L) : 0.f;
      float oj = 0.f;
      if (aj) {
        float dj = Pi.deltaf;
        if (d.multi) dj = d.params[d.meta[j] & META_PID_MASK].deltaf;
        oj = omega_of_f(d.kernel, dj, L);
      }
      const float Aj[9] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x};
      const float bj = c2.y;
      const float V = hj.w;
      float Wj[6];
      if constexpr (WAN) {
        const float4 w0 = __ldg(d.zw32 + 2 * (long long)j), w1 = __ldg(d.zw32 + 2 * (long long)j + 1);
        Wj[0] = w0.x; Wj[1] = w0.y; Wj[2] = w0.z; Wj[3] = w0.w; Wj[4] = w1.x; Wj[5] = w1.y;
      }
      float t[3];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float si = WAN ? sym_row(Wi, q, du) : bi * du[q];
        const float sj = WAN ? sym_row(Wj, q, du) : bj * du[q];
        const float ti = Ai[q] * g.x + Ai[q + 3] * g.y + Ai[q + 6] * g.z + si;
        const float tj = Aj[q] * g.x + Aj[q + 3] * g.y + Aj[q + 6] * g.z + sj;
        t[q] = (oi * ti + oj * tj) * V;
      }
      bx.add(t[0]); by.add(t[1]); bz.add(t[2]);
    }
    if (G > 1) { group_reduce<G>(bx); group_reduce<G>(by); group_reduce<G>(bz); }
    if (valid && gl == 0) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      flag_nan32(d, kstep, x, y, z);
    }
  }
}

// -------------------------------------------------------------------------------------------
// CMat phases with packed pairs and the next row pair's bond stream in flight (bond-stream
// variant 5; one lane per point, one parameter set; phase B for symmetric bond states). The
// per-bond sums are those of k_c_a32 / k_c_b32: the x and y rows of every 3x3 sum are one
// packed pair, z is scalar (the shape-tensor and force sums compensated, the
// displacement-gradient sums of phase A plain); bond states select the contributions (inactive bonds
// and padding slots gather their own point and add zero). The per-point epilogue of phase A is
// k_c_a32's. Phase B: with one influence value for both directions, t_ij + the term of j is
// w V_j ((A_i + A_j) xi + (beta_i + beta_j) du).
// -------------------------------------------------------------------------------------------
// occupancy bound of both packed correspondence phases: 3 resident blocks of 256 threads (80
// registers, with 48-100 bytes of spills). Measured on the 1M-point CMat block: step 1.445 ms
// at 3 blocks against 1.686 ms at 2 (110 registers, no spills) and 1.865 ms for the one-row
// kernels.
#ifndef PD_MINB_CQA
#define PD_MINB_CQA 3
#endif
#ifndef PD_MINB_CQB
#define PD_MINB_CQB 3
#endif

struct BondC {
  float2 dxy;   // displacement difference, x and y
  float dz;
  float L, rL, eps;
};

__device__ __forceinline__ void bond_c(const float4& g, const float4& hj, const float4& lj,
                                       const float2 nhi, const float nhz, const float2 nlo,
                                       const float nlz, BondC& B) {
  using namespace pack;
  B.dxy = add2(add2(xy(hj), nhi), add2(xy(lj), nlo));
  B.dz = (hj.z + nhz) + (lj.z + nlz);
  const float2 exy = add2(xy(g), B.dxy);
  const float ez = g.z + B.dz;
  const float2 e2 = mul2(exy, exy);
  const float l2 = fmaf(ez, ez, e2.x + e2.y);
  const float l = l2 * rsqrtf(l2);
  const float2 gd = mul2(xy(g), B.dxy);
  const float xd = fmaf(g.z, B.dz, gd.x + gd.y);
  const float2 d2 = mul2(B.dxy, B.dxy);
  const float dd = fmaf(B.dz, B.dz, d2.x + d2.y);
  B.L = fabsf(g.w);
  B.rL = __fdividef(1.f, B.L);
  B.eps = __fdividef(fmaf(2.f, xd, dd), l + B.L) * B.rL;
}

template <bool FULLK, bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_CQA) k_c_a32q(DevBody d, int kstep) {
  using namespace pack;
  if (d.ctrl->err) return;
  const int lane = threadIdx.x & 31;
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long s = warp0; s < d.nslices; s += nwarps) {
    const long long i = s * 32 + lane;
    const bool valid = i < d.n;
    const int self = valid ? (int)i : 0;
    const long long sbase = d.soff[s];
    const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
    const int cnt = valid ? (int)(d.off[i + 1] - d.off[i]) : 0;
    const unsigned meta = valid ? d.meta[i] : 0u;
    const DevParam& P = d.params[meta & META_PID_MASK];
    const float4 hi = d.uhi[self], lo = d.ulo[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const float epsc = P.epscf, id = P.inv_delta, vs = P.vscale;
    const float2 id2 = make_float2(id, id);
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    unsigned* pw = d.bits + (sbase >> 5);
    KSum2 K01, K23, K45;        // FULLK: (xx, yy), (zz, xy), (xz, yz)
    // rows x, y of column c of the displacement-gradient sum, and row z: plain FP32 sums (with
    // compensated sums phase A took 0.648 against 0.594 ms on the 1M-point CMat block, and the
    // FP32 displacement after 250 steps was within 1.33e-7 of FP64 against 1.37e-7 here, RMS
    // 7.85e-8 both: the error of the form comes from elsewhere)
    float2 Hxy[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    float Hz[3] = {0.f, 0.f, 0.f};
    float dK[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int na = 0;
    int nj0 = self, nj1 = self;
    float4 ng0 = make_float4(0.f, 0.f, 0.f, 1.f), ng1 = ng0;
    unsigned nw0 = 0u, nw1 = 0u;
    auto load_pair = [&](int r) {
      const bool two = r + 1 < rows;
      nw0 = pw[r];
      nw1 = two ? pw[r + 1] : 0u;
      nj0 = ld_stream(pn + 32 * r);
      ng0 = ld_stream(pg + 32 * r);
      if (two) { nj1 = ld_stream(pn + 32 * r + 32); ng1 = ld_stream(pg + 32 * r + 32); }
      else { nj1 = self; ng1 = make_float4(0.f, 0.f, 0.f, 1.f); }
    };
    if (rows > 0) load_pair(0);
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const unsigned w0 = nw0, w1 = nw1;
      const bool a0 = (w0 >> lane) & 1u, a1 = (w1 >> lane) & 1u;
      const int j0 = a0 ? nj0 : self, j1 = a1 ? nj1 : self;
      const float4 g0 = ng0, g1 = ng1;
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      if (r + 2 < rows) load_pair(r + 2);
      bool act0, act1;
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& g = u ? g1 : g0;
        const float4& hj = u ? hj1 : hj0;
        const bool a = u ? a1 : a0;
        BondC B;
        bond_c(g, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const bool act = a && !(B.eps > epsc && g.w > 0.f);
        const float om = omega_t<LIN>(d.kernel, P.deltaf, B.L, B.rL) * hj.w * vs;
        const float t = act ? om : 0.f;
        const float2 X = mul2(xy(g), id2);
        const float Xz = g.z * id;
        const float2 tU = mul2(make_float2(t, t), mul2(B.dxy, id2));
        const float tUz = t * (B.dz * id);
        Hxy[0] = add2(Hxy[0], mul2(tU, make_float2(X.x, X.x))); Hz[0] += tUz * X.x;
        Hxy[1] = add2(Hxy[1], mul2(tU, make_float2(X.y, X.y))); Hz[1] += tUz * X.y;
        Hxy[2] = add2(Hxy[2], mul2(tU, make_float2(Xz, Xz)));   Hz[2] += tUz * Xz;
        if constexpr (FULLK) {
          const float2 tX = mul2(make_float2(t, t), X);
          const float tXz = t * Xz;
          K01.add(mul2(tX, X));
          K23.add(make_float2(tXz * Xz, tX.x * X.y));
          K45.add(mul2(tX, make_float2(Xz, Xz)));
        } else if (a && !act) {
          // the bond breaks now: its term leaves the stored shape tensor
          dK[0] += om * X.x * X.x; dK[1] += om * X.y * X.y; dK[2] += om * Xz * Xz;
          dK[3] += om * X.x * X.y; dK[4] += om * X.x * Xz; dK[5] += om * X.y * Xz;
        }
        if (u) act1 = act; else act0 = act;
      }
      na += (int)act0 + (int)act1;
      const unsigned c0 = __ballot_sync(0xffffffffu, act0);
      const unsigned c1 = __ballot_sync(0xffffffffu, act1);
      if (lane == 0) {
        if (c0 != w0) pw[r] = c0;
        if (two && c1 != w1) pw[r + 1] = c1;
      }
    }
    bool killed = false;
    if (valid) {
      float k6[6];
      float2* ks = reinterpret_cast<float2*>(d.K32 + 6 * i);
      if constexpr (FULLK) {
        const float2 v01 = K01.value(), v23 = K23.value(), v45 = K45.value();
        k6[0] = v01.x; k6[1] = v01.y; k6[2] = v23.x; k6[3] = v23.y; k6[4] = v45.x; k6[5] = v45.y;
        ks[0] = make_float2(k6[0], k6[1]); ks[1] = make_float2(k6[2], k6[3]); ks[2] = make_float2(k6[4], k6[5]);
      } else {
        const float2 b0 = ks[0], b1 = ks[1], b2 = ks[2];
        k6[0] = b0.x; k6[1] = b0.y; k6[2] = b1.x; k6[3] = b1.y; k6[4] = b2.x; k6[5] = b2.y;
        if (dK[0] != 0.f || dK[1] != 0.f || dK[2] != 0.f) {  // a bond broke
#pragma unroll
          for (int q = 0; q < 6; q++) k6[q] -= dK[q];
          ks[0] = make_float2(k6[0], k6[1]); ks[1] = make_float2(k6[2], k6[3]); ks[2] = make_float2(k6[4], k6[5]);
        }
      }
      const float Km[9] = {k6[0], k6[3], k6[4],
                           k6[3], k6[1], k6[5],
                           k6[4], k6[5], k6[2]};
      float Kinv[9], Hm[9], H[9];
      finv3(Km, Kinv);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        Hm[3 * c] = Hxy[c].x; Hm[3 * c + 1] = Hxy[c].y; Hm[3 * c + 2] = Hz[c];
      }
      fmatmul(Hm, Kinv, H);
      bool hasnan = false;
      for (int q = 0; q < 9; q++) { d.H32[9 * i + q] = H[q]; hasnan |= isnan(H[q]); }
      const double damage = 1.0 - (double)na / (double)cnt;
      killed = (meta & META_KILLED) || (!(meta & META_HALO) && (damage > d.maxdmg || hasnan));
      if (killed) {
        if (!(meta & META_KILLED)) d.meta[i] = meta | META_KILLED;
        na = 0;
        c_state_clear32(d, i);
      } else {
        float Pm[9], PK[9];
        pk1_32(d.cmodel, P, H, Pm);
        fmatmul(Pm, Kinv, PK);
        c_state_store32(d, P, i, PK, Kinv, H, id * id * id * id * id);
      }
      d.n_active[i] = na;
    }
    if (!d.sym) {
      // directed bond states: a killed point loses all its bonds (correspondence.jl:293)
      const unsigned kill_mask = __ballot_sync(0xffffffffu, valid && killed);
      if (kill_mask && lane == 0)
        for (int r = 0; r < rows; r++) d.bits[(sbase >> 5) + r] &= ~kill_mask;
    }
  }
}

template <bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_CQB) k_c_b32q(DevBody d, int kstep) {
  using namespace pack;
  if (d.ctrl->err) return;
  const int lane = threadIdx.x & 31;
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long s = warp0; s < d.nslices; s += nwarps) {
    const long long i = s * 32 + lane;
    const bool valid = i < d.n;
    const int self = valid ? (int)i : 0;
    const long long sbase = d.soff[s];
    const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
    const DevParam& P = d.params[d.meta[self] & META_PID_MASK];
    const float delta = P.deltaf;
    const float4 hi = d.uhi[self], lo = d.ulo[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const float4 ci0 = d.cst32[3 * (long long)self], ci1 = d.cst32[3 * (long long)self + 1],
                 ci2 = d.cst32[3 * (long long)self + 2];
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    const unsigned* pw = d.bits + (sbase >> 5);
    KSum2 bxy;
    KSum1 bz;
    int nj0 = self, nj1 = self;
    float4 ng0 = make_float4(0.f, 0.f, 0.f, 1.f), ng1 = ng0;
    unsigned nw0 = 0u, nw1 = 0u;
    auto load_pair = [&](int r) {
      const bool two = r + 1 < rows;
      nw0 = ld_stream(pw + r);
      nw1 = two ? ld_stream(pw + r + 1) : 0u;
      nj0 = ld_stream(pn + 32 * r);
      ng0 = ld_stream(pg + 32 * r);
      if (two) { nj1 = ld_stream(pn + 32 * r + 32); ng1 = ld_stream(pg + 32 * r + 32); }
      else { nj1 = self; ng1 = make_float4(0.f, 0.f, 0.f, 1.f); }
    };
    if (rows > 0) load_pair(0);
    for (int r = 0; r < rows; r += 2) {
      const bool a0 = (nw0 >> lane) & 1u, a1 = (nw1 >> lane) & 1u;
      const int j0 = a0 ? nj0 : self, j1 = a1 ? nj1 : self;
      const float4 g0 = ng0, g1 = ng1;
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      const float4* cj0 = d.cst32 + 3 * (long long)j0;
      const float4* cj1 = d.cst32 + 3 * (long long)j1;
      const float4 c00 = __ldg(cj0), c01 = __ldg(cj0 + 1), c02 = __ldg(cj0 + 2);
      const float4 c10 = __ldg(cj1), c11 = __ldg(cj1 + 1), c12 = __ldg(cj1 + 2);
      if (r + 2 < rows) load_pair(r + 2);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& g = u ? g1 : g0;
        const float4& hj = u ? hj1 : hj0;
        const float4& lj = u ? lj1 : lj0;
        const float4& c0 = u ? c10 : c00;
        const float4& c1 = u ? c11 : c01;
        const float4& c2 = u ? c12 : c02;
        const float2 dxy = add2(add2(xy(hj), nhi), add2(xy(lj), nlo));
        const float dz = (hj.z + nhz) + (lj.z + nlz);
        // S = A_i + A_j (column-major: columns (S0 S1 S2), (S3 S4 S5), (S6 S7 S8)); beta_i + beta_j
        const float2 S01 = add2(make_float2(ci0.x, ci0.y), make_float2(c0.x, c0.y));
        const float2 S23 = add2(make_float2(ci0.z, ci0.w), make_float2(c0.z, c0.w));
        const float2 S45 = add2(make_float2(ci1.x, ci1.y), make_float2(c1.x, c1.y));
        const float2 S67 = add2(make_float2(ci1.z, ci1.w), make_float2(c1.z, c1.w));
        const float2 S8b = add2(make_float2(ci2.x, ci2.y), make_float2(c2.x, c2.y));
        // rows x, y: S01 xi_x + (S3, S4) xi_y + S67 xi_z + beta du
        const float2 S34 = make_float2(S23.y, S45.x);
        float2 txy = mul2(make_float2(S8b.y, S8b.y), dxy);
        txy = add2(txy, mul2(S01, make_float2(g.x, g.x)));
        txy = add2(txy, mul2(S34, make_float2(g.y, g.y)));
        txy = add2(txy, mul2(S67, make_float2(g.z, g.z)));
        const float tz = fmaf(S23.x, g.x, fmaf(S45.y, g.y, fmaf(S8b.x, g.z, S8b.y * dz)));
        const float L = fabsf(g.w);
        float f = omega_of_f(LIN ? KER_LINEAR : d.kernel, delta, L) * hj.w;
        f = (u ? a1 : a0) ? f : 0.f;
        bxy.add(mul2(make_float2(f, f), txy));
        bz.add(f * tz);
      }
    }
    if (valid) {
      const float2 v = bxy.value();
      const float z = bz.value();
      d.b32[3 * i] = v.x;
      d.b32[3 * i + 1] = v.y;
      d.b32[3 * i + 2] = z;
      flag_nan32(d, kstep, v.x, v.y, z);
    }
  }
}

// the packed correspondence kernels: one lane per point, one parameter set; phase B also needs
// symmetric bond states and ZEMSilling. With ZEMWan the packed phase B (both points' stiffness
// gathered with the next row pair in flight) spilled and took 1.37 ms on the 1M-point block
// against 1.12 ms for k_c_b32, so ZEMWan's phase B is the one-row kernel.
static bool cq_supported(const DevBody& d, int phase) {
  if (d.material != MAT_CMAT || d.lg != 1 || d.multi) return false;
  if (phase == 2 && (!d.sym || d.zem == ZEM_WAN)) return false;
  return true;
}

bool packed_supported(const DevBody& d, int phase) { return pk_supported(d, phase) || cq_supported(d, phase); }

// ------------------------------------------------------------------------------------------
#define PD_DISPATCH_G(G, CALL)                          \
  switch (G) {                                          \
    case 1: { constexpr int GG = 1; CALL; } break;      \
    case 2: { constexpr int GG = 2; CALL; } break;      \
    case 4: { constexpr int GG = 4; CALL; } break;      \
    case 8: { constexpr int GG = 8; CALL; } break;      \
    case 16: { constexpr int GG = 16; CALL; } break;    \
    default: { constexpr int GG = 32; CALL; } break;    \
  }

static int grid_for32(long long nslices, int block) {
  long long warps = nslices;
  long long blocks = (warps + block / 32 - 1) / (block / 32);
  if (blocks < 1) blocks = 1;
  if (PD_GRID_BLOCKS_PER_SM > 0 && blocks > 148LL * PD_GRID_BLOCKS_PER_SM)
    blocks = 148LL * PD_GRID_BLOCKS_PER_SM;
  return (int)blocks;
}

// BB: the two-row kernel for pipe 4, else the one-row kernel
template <bool ESC>
static void launch_bb32(const DevBody& d, const LaunchCfg& c, int G, int grid, int kstep, cudaStream_t s) {
  if (c.pipe == 4) {
    if (d.multi) { PD_DISPATCH_G(G, (k_bb32u<GG, true, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
    else { PD_DISPATCH_G(G, (k_bb32u<GG, false, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
  } else if (d.multi) {
    PD_DISPATCH_G(G, (k_bb32<GG, true, ESC><<<grid, c.block, 0, s>>>(d, kstep)));
  } else {
    PD_DISPATCH_G(G, (k_bb32<GG, false, ESC><<<grid, c.block, 0, s>>>(d, kstep)));
  }
}

// OSB: the two-row kernels for pipe 4, else the one-row kernels (also for pipes 1-3 when the
// surface correction is on: the TMA-staged stream carries no bond factors)
template <bool ESC>
static int launch_osb32(const DevBody& d, const LaunchCfg& c, int G, int grid, int kstep, bool A,
                        bool B, cudaStream_t s) {
  int launches = 0;
  if (c.pipe == 4) {
    if (A) {
      if (d.kernel == KER_LINEAR) {
        if (c.fullk) { PD_DISPATCH_G(G, (k_osb_a32u<GG, ESC, true, true><<<grid, c.block, 0, s>>>(d, kstep))); }
        else { PD_DISPATCH_G(G, (k_osb_a32u<GG, ESC, false, true><<<grid, c.block, 0, s>>>(d, kstep))); }
      } else if (c.fullk) {
        PD_DISPATCH_G(G, (k_osb_a32u<GG, ESC, true, false><<<grid, c.block, 0, s>>>(d, kstep)));
      } else {
        PD_DISPATCH_G(G, (k_osb_a32u<GG, ESC, false, false><<<grid, c.block, 0, s>>>(d, kstep)));
      }
      launches++;
    }
    if (B) {
      if (d.multi) { PD_DISPATCH_G(G, (k_osb_b32u<GG, true, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
      else { PD_DISPATCH_G(G, (k_osb_b32u<GG, false, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
      launches++;
    }
    return launches;
  }
  if (A) {
    if (c.fullk) { PD_DISPATCH_G(G, (k_osb_a32<GG, ESC, true><<<grid, c.block, 0, s>>>(d, kstep))); }
    else { PD_DISPATCH_G(G, (k_osb_a32<GG, ESC, false><<<grid, c.block, 0, s>>>(d, kstep))); }
    launches++;
  }
  if (B) {
    if (d.multi) { PD_DISPATCH_G(G, (k_osb_b32<GG, true, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
    else { PD_DISPATCH_G(G, (k_osb_b32<GG, false, ESC><<<grid, c.block, 0, s>>>(d, kstep))); }
    launches++;
  }
  return launches;
}

int launch_force32(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s) {
  const int G = d.lg;
  const int grid = grid_for32(d.nslices, c.block);
  const bool A = phase != 2, B = phase != 1;
  int launches = 0;
  if (d.material == MAT_BB) {
    if (!A) return 0;
    if (c.pipe == 5 && pk_supported(d, 1)) return launch_force32_pk(d, c, kstep, 1, s);
    LaunchCfg c4 = c;
    if (c.pipe == 5) c4.pipe = 4;   // the two-row kernel where the packed one does not apply
    if (d.sc32) launch_bb32<true>(d, c4, G, grid, kstep, s);
    else launch_bb32<false>(d, c4, G, grid, kstep, s);
    return 1;
  }
  if (d.material == MAT_OSB) {
    if (c.pipe == 5) {
      // the packed kernels where they apply, the two-row kernels for the other phase
      LaunchCfg c4 = c;
      c4.pipe = 4;
      const bool pa = A && pk_supported(d, 1), pb = B && pk_supported(d, 2);
      if (A) launches += pa ? launch_force32_pk(d, c, kstep, 1, s)
                            : (d.sc32 ? launch_osb32<true>(d, c4, G, grid, kstep, true, false, s)
                                      : launch_osb32<false>(d, c4, G, grid, kstep, true, false, s));
      if (B) launches += pb ? launch_force32_pk(d, c, kstep, 2, s)
                            : (d.sc32 ? launch_osb32<true>(d, c4, G, grid, kstep, false, true, s)
                                      : launch_osb32<false>(d, c4, G, grid, kstep, false, true, s));
      return launches;
    }
    if (d.sc32) return launch_osb32<true>(d, c, G, grid, kstep, A, B, s);
    return launch_osb32<false>(d, c, G, grid, kstep, A, B, s);
  }
  const bool lin = d.kernel == KER_LINEAR;
  if (A && c.pipe == 5 && cq_supported(d, 1)) {
    if (c.fullk) {
      if (lin) k_c_a32q<true, true><<<grid, c.block, 0, s>>>(d, kstep);
      else k_c_a32q<true, false><<<grid, c.block, 0, s>>>(d, kstep);
    } else {
      if (lin) k_c_a32q<false, true><<<grid, c.block, 0, s>>>(d, kstep);
      else k_c_a32q<false, false><<<grid, c.block, 0, s>>>(d, kstep);
    }
    launches++;
  } else if (A) {
    if (d.kernel == KER_LINEAR) {
      if (c.fullk) { PD_DISPATCH_G(G, (k_c_a32<GG, true, true><<<grid, c.block, 0, s>>>(d, kstep))); }
      else { PD_DISPATCH_G(G, (k_c_a32<GG, false, true><<<grid, c.block, 0, s>>>(d, kstep))); }
    } else if (c.fullk) {
      PD_DISPATCH_G(G, (k_c_a32<GG, true, false><<<grid, c.block, 0, s>>>(d, kstep)));
    } else {
      PD_DISPATCH_G(G, (k_c_a32<GG, false, false><<<grid, c.block, 0, s>>>(d, kstep)));
    }
    launches++;
  }
  const bool wan = d.zem == ZEM_WAN;
  if (B && c.pipe == 5 && cq_supported(d, 2)) {
    if (lin) k_c_b32q<true><<<grid, c.block, 0, s>>>(d, kstep);
    else k_c_b32q<false><<<grid, c.block, 0, s>>>(d, kstep);
    launches++;
  } else if (B) {
    if (wan) {
      if (d.sym) { PD_DISPATCH_G(G, (k_c_b32<GG, true, true><<<grid, c.block, 0, s>>>(d, kstep))); }
      else { PD_DISPATCH_G(G, (k_c_b32<GG, false, true><<<grid, c.block, 0, s>>>(d, kstep))); }
    } else if (d.sym) {
      PD_DISPATCH_G(G, (k_c_b32<GG, true, false><<<grid, c.block, 0, s>>>(d, kstep)));
    } else {
      PD_DISPATCH_G(G, (k_c_b32<GG, false, false><<<grid, c.block, 0, s>>>(d, kstep)));
    }
    launches++;
  }
  return launches;
}

}  // namespace pd
