// pd_force32_pk.cu -- FP32-compensated OSB force kernels with fewer instructions per bond and
// the bond stream of the next row pair in flight (bond-stream variant 5: one lane per point,
// the sliced layout of G = 1).
//
// The two-row kernels (pd_force32.cu) issue about 93 (phase A) and 116 (phase B) warp
// instructions per bond row. These compute the same quantities with 75 / 68:
//   - the x and y components of every per-bond 3-vector (displacement difference, deformed
//     bond vector, the force and its compensated sum) are one packed pair (f32x2: one
//     instruction for both components), z is scalar;
//   - bond states select the contribution instead of branching around it: inactive bonds and
//     padding slots gather their own point (always in bounds) and add zero;
//   - the bond stream is addressed from the slice base with 32-bit row offsets;
//   - phase B is written for symmetric bond states with one parameter set, where the two
//     directions of a bond share its influence value: s_ij + s_ji = w ((c2_i + c2_j) L +
//     (c1_i + c1_j) e), one packed add for both coefficient sums.
// With fewer instructions alone the kernels ran slower (issue utilisation fell from 71 % to
// 40 %, long-scoreboard stalls per issue rose from 4.7 to 14.7 on the 1M-point block): the
// phases are bound by the latency of the bond stream and the neighbour gathers that depend on
// it, not by issue. The freed registers therefore hold the next row pair's stream records,
// loaded after the current pair's gathers and before its arithmetic, so the DRAM latency of
// the stream overlaps the gathers and arithmetic of the pair before it. The stream loads are
// streaming (evict-first) loads, so that the bond records, read once, leave L2 to the
// neighbours' point records.
// The arithmetic is the FP32 form of pd_force32.cu (deformed bond vector from the stored
// reference offset, cancellation-free extension, Kahan sums); roundings differ from the
// two-row kernels only in the order of a few operations.
#include "pd_common.cuh"
#include "pd_launch.h"
#include "pd_pack.cuh"

namespace pd {

namespace {

using namespace pack;

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

// occupancy bounds: phase A at 4 resident blocks of 256 threads (59 registers), phase B at 3
// (72 registers; at 4 it spills). Measured on the 8M-point OSB block, blocks of 128:
// 4.24 / 4.47 ms against 4.40 / 4.70 ms for the two-row kernels; phase B at 4 blocks (with
// spills) 4.78 ms, at 2 blocks 6.18 ms.
#ifndef PD_MINB_QA
#define PD_MINB_QA 4
#endif
#ifndef PD_MINB_QB
#define PD_MINB_QB 3
#endif

// Phase B with the bond stream of the next row pair loaded while the current pair is
// gathered and computed (one pair of rows ahead): the DRAM latency of the stream overlaps the
// gathers and arithmetic of the pair before it. MB resident blocks per SM.
template <bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_QB) k_osb_b32q(DevBody d, int kstep) {
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
      // gathers of this pair, then the stream of the next pair, then the arithmetic
      const float4 hj0 = __ldg(d.uhi + j0), lj0 = __ldg(d.ulo + j0);
      const float4 hj1 = __ldg(d.uhi + j1), lj1 = __ldg(d.ulo + j1);
      const float2 cj0 = __ldg(d.cc32 + j0), cj1 = __ldg(d.cc32 + j1);
      if (r + 2 < rows) load_pair(r + 2);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4& g = u ? g1 : g0;
        const float4& hj = u ? hj1 : hj0;
        BondP B;
        bond_pk(g, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
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
template <bool FULLM, bool LIN>
__global__ void __launch_bounds__(256, PD_MINB_QA) k_osb_a32q(DevBody d, int kstep) {
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

// BB (calc_failure! and force_density_point!, bond_based.jl:125-161) in one sweep with packed
// pairs and the next row pair's stream in flight, as the OSB phases above: f = bc eps V_j eta / l
// for the bonds that stay active, the failure test on eps = e / L.
#ifndef PD_MINB_QBB
#define PD_MINB_QBB 4
#endif
__global__ void __launch_bounds__(256, PD_MINB_QBB) k_bb32q(DevBody d, int kstep) {
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
    const float epsc = P.epscf, bc = P.bcf;
    const float4 hi = d.uhi[self], lo = d.ulo[self];
    const float2 nhi = make_float2(-hi.x, -hi.y), nlo = make_float2(-lo.x, -lo.y);
    const float nhz = -hi.z, nlz = -lo.z;
    const int* pn = d.nbr + sbase + lane;
    const float4* pg = d.geo + sbase + lane;
    unsigned* pw = d.bits + (sbase >> 5);
    KSum2 bxy;
    KSum1 bz;
    int na = 0;
    int nj0 = self, nj1 = self;
    float4 ng0 = make_float4(0.f, 0.f, 0.f, 1.f), ng1 = ng0;
    unsigned nw0 = 0u, nw1 = 0u;
    // the state words are plain loads: this warp owns them and rewrites them below
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
        BondP B;
        bond_pk(g, hj, u ? lj1 : lj0, nhi, nhz, nlo, nlz, B);
        const float eps = B.e * B.rL;
        const bool act = a && !(eps > epsc && g.w > 0.f);
        const float sc = act ? bc * eps * hj.w * B.rl : 0.f;
        bxy.add(mul2(make_float2(sc, sc), B.exy));
        bz.add(sc * B.ez);
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
      const float2 v = bxy.value();
      const float z = bz.value();
      d.b32[3 * i] = v.x;
      d.b32[3 * i + 1] = v.y;
      d.b32[3 * i + 2] = z;
      d.n_active[i] = na;
      if (isnan(v.x) || isnan(v.y) || isnan(z)) {
        const long long step = d.ctrl->base + kstep;
        if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
        else atomicMin(&d.ctrl->err_step, step);
      }
    }
  }
}

// the packed kernels serve one lane per point, BB and OSB without surface correction and with
// one parameter set; OSB's phase B also needs symmetric bond states
bool pk_supported(const DevBody& d, int phase) {
  if (d.material == MAT_CMAT || d.lg != 1 || d.sc32 != nullptr || d.multi) return false;
  if (d.material == MAT_BB) return phase == 1;
  if (phase == 2 && !d.sym) return false;
  return true;
}

static int grid_pk(long long nslices, int block) {
  long long blocks = (nslices + block / 32 - 1) / (block / 32);
  if (blocks < 1) blocks = 1;
  if (PD_GRID_BLOCKS_PER_SM > 0 && blocks > 148LL * PD_GRID_BLOCKS_PER_SM)
    blocks = 148LL * PD_GRID_BLOCKS_PER_SM;
  return (int)blocks;
}

int launch_force32_pk(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s) {
  const int grid = grid_pk(d.nslices, c.block);
  const bool lin = d.kernel == KER_LINEAR;
  int launches = 0;
  if (d.material == MAT_BB) {
    if (phase == 2) return 0;
    k_bb32q<<<grid, c.block, 0, s>>>(d, kstep);
    return 1;
  }
  if (phase != 2) {
    if (c.fullk) {
      if (lin) k_osb_a32q<true, true><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_a32q<true, false><<<grid, c.block, 0, s>>>(d, kstep);
    } else {
      if (lin) k_osb_a32q<false, true><<<grid, c.block, 0, s>>>(d, kstep);
      else k_osb_a32q<false, false><<<grid, c.block, 0, s>>>(d, kstep);
    }
    launches++;
  }
  if (phase != 1) {
    if (lin) k_osb_b32q<true><<<grid, c.block, 0, s>>>(d, kstep);
    else k_osb_b32q<false><<<grid, c.block, 0, s>>>(d, kstep);
    launches++;
  }
  return launches;
}

}  // namespace pd
