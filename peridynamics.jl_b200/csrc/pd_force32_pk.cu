// pd_force32_pk.cu -- FP32-compensated OSB force kernels written for instruction count
// (bond-stream variant 5: one lane per point, the sliced layout of G = 1).
//
// The OSB phases of the two-row kernels (pd_force32.cu) issue about 93 (phase A) and 116
// (phase B) warp instructions per bond row, and run at 61 % / 71 % issue utilisation and
// 0.74 / 0.70 of the measured HBM copy rate on the 1M-point block: they are limited by
// instruction issue as much as by DRAM. These kernels compute the same quantities with fewer
// instructions:
//   - the x and y components of every per-bond 3-vector (displacement difference, deformed
//     bond vector, the force and its compensated sum) are one packed pair (f32x2: one
//     instruction for both components), z is scalar;
//   - bond states select the contribution instead of branching around it: inactive bonds and
//     padding slots gather their own point (always in bounds) and add zero;
//   - the bond stream is addressed from the slice base with 32-bit row offsets;
//   - phase B is written for symmetric bond states with one parameter set, where the two
//     directions of a bond share its influence value: s_ij + s_ji = w ((c2_i + c2_j) L +
//     (c1_i + c1_j) e), one packed add for both coefficient sums.
// The arithmetic is the FP32 form of pd_force32.cu (deformed bond vector from the stored
// reference offset, cancellation-free extension, Kahan sums); roundings differ from the
// two-row kernels only in the order of a few operations.
#include "pd_common.cuh"
#include "pd_launch.h"

namespace pd {

namespace {

// packed FP32 pairs (sm_100 f32x2): flush-to-zero as the rest of the FP32 force path
__device__ __forceinline__ unsigned long long pk(float2 v) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}

// Kahan sum of pairs with the negated compensation n = -c: y = x + n, t = s + y,
// n = (s - t) + y, s = t (the value is s + n)
struct KSum2 {
  float2 s, n;
  __device__ __forceinline__ KSum2() : s(make_float2(0.f, 0.f)), n(make_float2(0.f, 0.f)) {}
  __device__ __forceinline__ void add(float2 x) {
    const float2 y = add2(x, n);
    const float2 t = add2(s, y);
    n = add2(sub2(s, t), y);
    s = t;
  }
  __device__ __forceinline__ float2 value() const { return add2(s, n); }
};

struct KSum1 {
  float s, n;
  __device__ __forceinline__ KSum1() : s(0.f), n(0.f) {}
  __device__ __forceinline__ void add(float x) {
    const float y = x + n;
    const float t = s + y;
    n = (s - t) + y;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s + n; }
};

__device__ __forceinline__ float2 xy(const float4& v) { return make_float2(v.x, v.y); }

// the bond in FP32 (as bond32 of pd_force32.cu): du = (h_j - h_i) + (l_j - l_i),
// eta = xi + du, l = |eta|, e = l - L = (2 xi.du + du.du) / (l + L)
struct BondP {
  float2 exy;     // deformed bond vector, x and y
  float ez;
  float rl, L, rL, e;
};

__device__ __forceinline__ void bond_pk(const float4& g, const float4& hj, const float4& lj,
                                        const float2 nhi, const float nhz, const float2 nlo,
                                        const float nlz, BondP& B) {
  const float2 dxy = add2(add2(xy(hj), nhi), add2(xy(lj), nlo));
  const float dz = (hj.z + nhz) + (lj.z + nlz);
  B.exy = add2(xy(g), dxy);
  B.ez = g.z + dz;
  const float2 e2 = mul2(B.exy, B.exy);
  const float l2 = fmaf(B.ez, B.ez, e2.x + e2.y);
  B.rl = rsqrtf(l2);
  const float l = l2 * B.rl;
  const float2 gd = mul2(xy(g), dxy);
  const float xd = fmaf(g.z, dz, gd.x + gd.y);
  const float2 d2 = mul2(dxy, dxy);
  const float dd = fmaf(dz, dz, d2.x + d2.y);
  B.L = fabsf(g.w);
  B.rL = __fdividef(1.f, B.L);
  B.e = __fdividef(fmaf(2.f, xd, dd), l + B.L);
}

template <bool LIN>
__device__ __forceinline__ float omega_pk(int kernel, float delta, float L, float rL) {
  if constexpr (LIN) return delta * rL;
  else return kernel == KER_LINEAR ? delta * rL : omega_of_f(kernel, delta, L);
}

}  // namespace

#ifndef PD_MINB_PA
#define PD_MINB_PA 4
#endif
#ifndef PD_MINB_PB
#define PD_MINB_PB 4
#endif

// -------------------------------------------------------------------------------------------
// OSB phase A (ordinary_state_based.jl:107-126, 176-204): failure, weighted volume, dilatation,
// c1 = 15 G / m, c2 = theta (3 K / m - c1 / 3) (:135-136). FULLM: the weighted volume summed
// over the active bonds, else the stored one minus the terms of the bonds breaking now (as
// k_osb_a32 of pd_force32.cu).
// -------------------------------------------------------------------------------------------
template <bool FULLM, bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_PA) k_osb_a32p(DevBody d, int kstep) {
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
    const float epsc = P.epscf, delta = P.deltaf;
    const float4 hi = d.uhi[self], lo = d.ulo[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    unsigned* pw = d.bits + (sbase >> 5);
    KSum2 mt;       // FULLM: (m, theta)
    KSum1 th;       // !FULLM: theta
    float dm = 0.f;
    int na = 0;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;   // uniform over the warp
      const unsigned w0 = pw[r], w1 = two ? pw[r + 1] : 0u;
      const bool a0 = (w0 >> lane) & 1u, a1 = (w1 >> lane) & 1u;
      int j0 = __ldg(pn + 32 * r), j1 = self;
      const float4 g0 = __ldg(pg + 32 * r);
      float4 g1 = make_float4(0.f, 0.f, 0.f, 1.f);
      if (two) { j1 = __ldg(pn + 32 * r + 32); g1 = __ldg(pg + 32 * r + 32); }
      j0 = a0 ? j0 : self;
      j1 = a1 ? j1 : self;
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      bool act0, act1;
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& g = u ? g1 : g0;
        const float4& hj = u ? hj1 : hj0;
        const bool a = u ? a1 : a0;
        BondP B;
        bond_pk(g, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const float eps = B.e * B.rL;
        const bool act = a && !(eps > epsc && g.w > 0.f);
        const float om = omega_pk<LIN>(d.kernel, delta, B.L, B.rL) * hj.w;
        const float th_b = act ? om * B.L * B.e : 0.f;
        if (FULLM) {
          const float2 g2 = mul2(xy(g), xy(g));
          const float xi2 = fmaf(g.z, g.z, g2.x + g2.y);
          mt.add(make_float2(act ? om * xi2 : 0.f, th_b));
        } else {
          th.add(th_b);
          if (a && !act) {   // breaks now: its term leaves the stored weighted volume
            const float2 g2 = mul2(xy(g), xy(g));
            dm += om * fmaf(g.z, g.z, g2.x + g2.y);
          }
        }
        if (u) act1 = act; else act0 = act;
      }
      na += (int)act0 + (int)act1;
      const unsigned nw0 = __ballot_sync(0xffffffffu, act0);
      const unsigned nw1 = __ballot_sync(0xffffffffu, act1);
      if (lane == 0) {
        if (nw0 != w0) pw[r] = nw0;
        if (two && nw1 != w1) pw[r + 1] = nw1;
      }
    }
    if (valid) {
      float wv, tv;
      if (FULLM) {
        const float2 v = mt.value();
        wv = v.x;
        tv = v.y;
      } else {
        const float m0 = d.cm32[i].x;
        wv = dm != 0.f ? m0 - dm : m0;
        tv = th.value();
      }
      float c1 = 0.f, c2 = 0.f, dil = 0.f;
      if (wv != 0.f) {
        dil = 3.f / wv * tv;
        c1 = 15.f * P.Gf / wv;
        c2 = dil * (3.f * P.Kf / wv - c1 / 3.f);
      }
      d.cc32[i] = make_float2(c1, c2);
      d.cm32[i] = make_float2(wv, dil);
      d.n_active[i] = na;
    }
  }
}

// -------------------------------------------------------------------------------------------
// OSB phase B (ordinary_state_based.jl:128-149) for symmetric bond states and one parameter
// set: b_i = sum_j w ((c2_i + c2_j) L + (c1_i + c1_j) e) V_j eta / l over the active bonds.
// -------------------------------------------------------------------------------------------
template <bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_PB) k_osb_b32p(DevBody d, int kstep) {
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
    const float2 ci = d.cc32[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    const unsigned* pw = d.bits + (sbase >> 5);
    KSum2 bxy;
    KSum1 bz;
    for (int r = 0; r < rows; r += 2) {
      const bool two = r + 1 < rows;
      const unsigned w0 = __ldg(pw + r), w1 = two ? __ldg(pw + r + 1) : 0u;
      const bool a0 = (w0 >> lane) & 1u, a1 = (w1 >> lane) & 1u;
      int j0 = __ldg(pn + 32 * r), j1 = self;
      const float4 g0 = __ldg(pg + 32 * r);
      float4 g1 = make_float4(0.f, 0.f, 0.f, 1.f);
      if (two) { j1 = __ldg(pn + 32 * r + 32); g1 = __ldg(pg + 32 * r + 32); }
      j0 = a0 ? j0 : self;
      j1 = a1 ? j1 : self;
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      const float2 cj0 = __ldg(d.cc32 + j0), cj1 = __ldg(d.cc32 + j1);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& hj = u ? hj1 : hj0;
        BondP B;
        bond_pk(u ? g1 : g0, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const float2 cs = add2(ci, u ? cj1 : cj0);          // (c1_i + c1_j, c2_i + c2_j)
        const float om = omega_pk<LIN>(d.kernel, delta, B.L, B.rL);
        float f = om * fmaf(cs.y, B.L, cs.x * B.e) * hj.w * B.rl;
        f = (u ? a1 : a0) ? f : 0.f;
        bxy.add(mul2(make_float2(f, f), B.exy));
        bz.add(f * B.ez);
      }
    }
    if (valid) {
      const float2 v = bxy.value();
      const float z = bz.value();
      d.b32[3 * i] = v.x;
      d.b32[3 * i + 1] = v.y;
      d.b32[3 * i + 2] = z;
      if (isnan(v.x) || isnan(v.y) || isnan(z)) {
        const long long step = d.ctrl->base + kstep;
        if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
        else atomicMin(&d.ctrl->err_step, step);
      }
    }
  }
}

// Phase B with the bond stream of the next row pair loaded while the current pair is
// gathered and computed (one pair of rows ahead): the DRAM latency of the stream overlaps the
// gathers and arithmetic of the pair before it. MB resident blocks per SM.
template <bool LIN, int MB>
__global__ void __launch_bounds__(256, MB) k_osb_b32q(DevBody d, int kstep) {
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
    const float2 ci = d.cc32[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    const unsigned* pw = d.bits + (sbase >> 5);
    KSum2 bxy;
    KSum1 bz;
    // stream records of the pair (r, r + 1): neighbour (self when inactive), geometry, state
    int nj0 = self, nj1 = self;
    float4 ng0 = make_float4(0.f, 0.f, 0.f, 1.f), ng1 = ng0;
    unsigned nw0 = 0u, nw1 = 0u;
    auto load_pair = [&](int r) {
      const bool two = r + 1 < rows;
      nw0 = __ldg(pw + r);
      nw1 = two ? __ldg(pw + r + 1) : 0u;
      nj0 = __ldg(pn + 32 * r);
      ng0 = __ldg(pg + 32 * r);
      if (two) { nj1 = __ldg(pn + 32 * r + 32); ng1 = __ldg(pg + 32 * r + 32); }
      else { nj1 = self; ng1 = make_float4(0.f, 0.f, 0.f, 1.f); }
    };
    if (rows > 0) load_pair(0);
    for (int r = 0; r < rows; r += 2) {
      const bool a0 = (nw0 >> lane) & 1u, a1 = (nw1 >> lane) & 1u;
      const int j0 = a0 ? nj0 : self, j1 = a1 ? nj1 : self;
      const float4 g0 = ng0, g1 = ng1;
      // gathers of this pair, then the stream of the next pair, then the arithmetic
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      const float2 cj0 = __ldg(d.cc32 + j0), cj1 = __ldg(d.cc32 + j1);
      if (r + 2 < rows) load_pair(r + 2);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& hj = u ? hj1 : hj0;
        BondP B;
        bond_pk(u ? g1 : g0, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const float2 cs = add2(ci, u ? cj1 : cj0);
        const float om = omega_pk<LIN>(d.kernel, delta, B.L, B.rL);
        float f = om * fmaf(cs.y, B.L, cs.x * B.e) * hj.w * B.rl;
        f = (u ? a1 : a0) ? f : 0.f;
        bxy.add(mul2(make_float2(f, f), B.exy));
        bz.add(f * B.ez);
      }
    }
    if (valid) {
      const float2 v = bxy.value();
      const float z = bz.value();
      d.b32[3 * i] = v.x;
      d.b32[3 * i + 1] = v.y;
      d.b32[3 * i + 2] = z;
      if (isnan(v.x) || isnan(v.y) || isnan(z)) {
        const long long step = d.ctrl->base + kstep;
        if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
        else atomicMin(&d.ctrl->err_step, step);
      }
    }
  }
}

// Phase A with the next row pair's stream loaded one pair ahead (as k_osb_b32q).
template <bool FULLM, bool LIN, int MB>
__global__ void __launch_bounds__(256, MB) k_osb_a32q(DevBody d, int kstep) {
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
    const float epsc = P.epscf, delta = P.deltaf;
    const float4 hi = d.uhi[self], lo = d.ulo[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    unsigned* pw = d.bits + (sbase >> 5);
    KSum2 mt;
    KSum1 th;
    float dm = 0.f;
    int na = 0;
    int nj0 = self, nj1 = self;
    float4 ng0 = make_float4(0.f, 0.f, 0.f, 1.f), ng1 = ng0;
    unsigned nw0 = 0u, nw1 = 0u;
    // the state words are plain loads: this warp owns them and rewrites them below
    auto load_pair = [&](int r) {
      const bool two = r + 1 < rows;
      nw0 = pw[r];
      nw1 = two ? pw[r + 1] : 0u;
      nj0 = __ldg(pn + 32 * r);
      ng0 = __ldg(pg + 32 * r);
      if (two) { nj1 = __ldg(pn + 32 * r + 32); ng1 = __ldg(pg + 32 * r + 32); }
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
        BondP B;
        bond_pk(g, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const float eps = B.e * B.rL;
        const bool act = a && !(eps > epsc && g.w > 0.f);
        const float om = omega_pk<LIN>(d.kernel, delta, B.L, B.rL) * hj.w;
        const float th_b = act ? om * B.L * B.e : 0.f;
        if (FULLM) {
          const float2 g2 = mul2(xy(g), xy(g));
          const float xi2 = fmaf(g.z, g.z, g2.x + g2.y);
          mt.add(make_float2(act ? om * xi2 : 0.f, th_b));
        } else {
          th.add(th_b);
          if (a && !act) {
            const float2 g2 = mul2(xy(g), xy(g));
            dm += om * fmaf(g.z, g.z, g2.x + g2.y);
          }
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
    if (valid) {
      float wv, tv;
      if (FULLM) {
        const float2 v = mt.value();
        wv = v.x;
        tv = v.y;
      } else {
        const float m0 = d.cm32[i].x;
        wv = dm != 0.f ? m0 - dm : m0;
        tv = th.value();
      }
      float c1 = 0.f, c2 = 0.f, dil = 0.f;
      if (wv != 0.f) {
        dil = 3.f / wv * tv;
        c1 = 15.f * P.Gf / wv;
        c2 = dil * (3.f * P.Kf / wv - c1 / 3.f);
      }
      d.cc32[i] = make_float2(c1, c2);
      d.cm32[i] = make_float2(wv, dil);
      d.n_active[i] = na;
    }
  }
}

// -------------------------------------------------------------------------------------------
// Bond stream staged STAGES row pairs ahead through shared memory (cp.async): every lane copies
// its own slots (neighbour index and geometry of rows r and r + 1) into a per-warp ring, lanes 0
// and 1 the two state words; the bytes in flight cost no registers. The gathers and arithmetic
// are those of k_osb_b32p / k_osb_a32p.
// -------------------------------------------------------------------------------------------
template <int STAGES>
struct StreamRing {
  float4 g[STAGES][2][32];
  int j[STAGES][2][32];
  unsigned w[STAGES][2];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// copies of the row pair (r, r + 1) into stage st (rows past the slice copy nothing)
template <int STAGES>
__device__ __forceinline__ void stage_pair(StreamRing<STAGES>& R, int st, int r, int rows,
                                           const int* pn, const float4* pg, const unsigned* pw,
                                           int lane) {
  if (r < rows) {
    cp_async16(&R.g[st][0][lane], pg + 32 * r);
    cp_async4(&R.j[st][0][lane], pn + 32 * r);
    if (lane == 0) cp_async4(&R.w[st][0], pw + r);
  }
  if (r + 1 < rows) {
    cp_async16(&R.g[st][1][lane], pg + 32 * r + 32);
    cp_async4(&R.j[st][1][lane], pn + 32 * r + 32);
    if (lane == 1) cp_async4(&R.w[st][1], pw + r + 1);
  }
  cp_commit();
}

template <bool LIN, int STAGES>
__global__ void __launch_bounds__(256, 4) k_osb_b32c(DevBody d, int kstep) {
  __shared__ StreamRing<STAGES> ring[8];
  if (d.ctrl->err) return;
  const int lane = threadIdx.x & 31;
  StreamRing<STAGES>& R = ring[threadIdx.x >> 5];
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long s = warp0; s < d.nslices; s += nwarps) {
    const long long i = s * 32 + lane;
    const bool valid = i < d.n;
    const int self = valid ? (int)i : 0;
    const long long sbase = d.soff[s];
    const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    const unsigned* pw = d.bits + (sbase >> 5);
    __syncwarp();   // the ring's previous slice is consumed by every lane
#pragma unroll
    for (int q = 0; q < STAGES - 1; q++) stage_pair(R, q, 2 * q, rows, pn, pg, pw, lane);
    const DevParam& P = d.params[d.meta[self] & META_PID_MASK];
    const float delta = P.deltaf;
    const float4 hi = d.uhi[self], lo = d.ulo[self];
    const float2 ci = d.cc32[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    KSum2 bxy;
    KSum1 bz;
    for (int r = 0, q = 0; r < rows; r += 2, q++) {
      // the pair STAGES - 1 ahead goes into the stage this pair's predecessor freed
      __syncwarp();
      stage_pair(R, (q + STAGES - 1) % STAGES, r + 2 * (STAGES - 1), rows, pn, pg, pw, lane);
      cp_wait<STAGES - 1>();
      __syncwarp();   // the state words copied by lanes 0 and 1
      const int st = q % STAGES;
      const bool two = r + 1 < rows;
      const unsigned w0 = R.w[st][0], w1 = two ? R.w[st][1] : 0u;
      const bool a0 = (w0 >> lane) & 1u, a1 = (w1 >> lane) & 1u;
      const int j0 = a0 ? R.j[st][0][lane] : self;
      const int j1 = a1 ? R.j[st][1][lane] : self;
      const float4 g0 = R.g[st][0][lane];
      const float4 g1 = two ? R.g[st][1][lane] : make_float4(0.f, 0.f, 0.f, 1.f);
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      const float2 cj0 = __ldg(d.cc32 + j0), cj1 = __ldg(d.cc32 + j1);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& hj = u ? hj1 : hj0;
        BondP B;
        bond_pk(u ? g1 : g0, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const float2 cs = add2(ci, u ? cj1 : cj0);
        const float om = omega_pk<LIN>(d.kernel, delta, B.L, B.rL);
        float f = om * fmaf(cs.y, B.L, cs.x * B.e) * hj.w * B.rl;
        f = (u ? a1 : a0) ? f : 0.f;
        bxy.add(mul2(make_float2(f, f), B.exy));
        bz.add(f * B.ez);
      }
    }
    cp_wait<0>();
    if (valid) {
      const float2 v = bxy.value();
      const float z = bz.value();
      d.b32[3 * i] = v.x;
      d.b32[3 * i + 1] = v.y;
      d.b32[3 * i + 2] = z;
      if (isnan(v.x) || isnan(v.y) || isnan(z)) {
        const long long step = d.ctrl->base + kstep;
        if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
        else atomicMin(&d.ctrl->err_step, step);
      }
    }
  }
}

// the packed kernels serve one lane per point, OSB without surface correction and with one
// parameter set; phase B also needs symmetric bond states
bool pk_supported(const DevBody& d, int phase) {
  if (d.material != MAT_OSB || d.lg != 1 || d.sc32 != nullptr || d.multi) return false;
  if (phase == 2 && !d.sym) return false;
  return true;
}

static int grid_pk(long long nslices, int block) {
  long long blocks = (nslices + block / 32 - 1) / (block / 32);
  if (blocks < 1) blocks = 1;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  return (int)blocks;
}

template <int MBA, int MBB>
static int launch_q(const DevBody& d, const LaunchCfg& c, int grid, int kstep, int phase, cudaStream_t s) {
  const bool lin = d.kernel == KER_LINEAR;
  int launches = 0;
  if (phase != 2) {
    if (c.fullk) {
      if (lin) k_osb_a32q<true, true, MBA><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_a32q<true, false, MBA><<<grid, c.block, 0, s>>>(d, kstep);
    } else {
      if (lin) k_osb_a32q<false, true, MBA><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_a32q<false, false, MBA><<<grid, c.block, 0, s>>>(d, kstep);
    }
    launches++;
  }
  if (phase != 1) {
    if (lin) k_osb_b32q<true, MBB><<<grid, c.block, 0, s>>>(d, kstep);
    else k_osb_b32q<false, MBB><<<grid, c.block, 0, s>>>(d, kstep);
    launches++;
  }
  return launches;
}

int launch_force32_pk(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s) {
  const int grid = grid_pk(d.nslices, c.block);
  if (c.pipe == 6) return launch_q<4, 3>(d, c, grid, kstep, phase, s);
  if (c.pipe == 7) return launch_q<3, 2>(d, c, grid, kstep, phase, s);
  if (c.pipe == 8) return launch_q<4, 4>(d, c, grid, kstep, phase, s);
  if (c.pipe == 9) {
    int launches = phase != 2 ? launch_q<4, 3>(d, c, grid, kstep, 1, s) : 0;
    if (phase != 1) {
      if (d.kernel == KER_LINEAR) k_osb_b32c<true, 4><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_b32c<false, 4><<<grid, c.block, 0, s>>>(d, kstep);
      launches++;
    }
    return launches;
  }
  const bool lin = d.kernel == KER_LINEAR;
  int launches = 0;
  if (phase != 2) {
    if (c.fullk) {
      if (lin) k_osb_a32p<true, true><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_a32p<true, false><<<grid, c.block, 0, s>>>(d, kstep);
    } else {
      if (lin) k_osb_a32p<false, true><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_a32p<false, false><<<grid, c.block, 0, s>>>(d, kstep);
    }
    launches++;
  }
  if (phase != 1) {
    if (lin) k_osb_b32p<true><<<grid, c.block, 0, s>>>(d, kstep);
    else k_osb_b32p<false><<<grid, c.block, 0, s>>>(d, kstep);
    launches++;
  }
  return launches;
}

}  // namespace pd
