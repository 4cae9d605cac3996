// pd_force32_tma.cu -- FP32-compensated force kernels with the bond stream staged in shared
// memory by TMA bulk copies (the fast path on sm_100a).
//
// Each warp owns a ring of NS stages in shared memory; a stage holds CR rows of the sliced
// bond layout (32 neighbour indices and 32 float4 bond vectors per row). Lane 0 issues one
// cp.async.bulk per array and chunk (no multicast; the source is this GPU's memory) and
// arms the stage's mbarrier with the expected byte count; the warp consumes chunk t while
// the copies of chunks t+1 .. t+NS-1 are in flight, so no HBM latency sits on the per-row
// dependency chain. The neighbour gathers (displacement, phase-A state) of row r+1 are
// issued before row r is computed. Waits are bounded: on a timeout the kernel records
// error 3 in the control block, drains its own copies (bounded again) and returns.
//
// Arithmetic per bond and per point is the one of pd_force32.cu.
#include "pd_common.cuh"
#include "pd_launch.h"

// resident blocks of 128 threads per SM the register allocation must allow
#ifndef PD_TMA_MINB
#define PD_TMA_MINB 6
#endif

namespace pd {

namespace tma {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_bar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void bar_arrive_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool bar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false after `limit` polls
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity, unsigned limit) {
  for (unsigned it = 0; it < limit; it++)
    if (bar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

constexpr unsigned WAIT_LIMIT = 1u << 24;

}  // namespace tma

__device__ __forceinline__ double4 ld4t(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

struct BondT {
  float L, rL, dux, duy, duz, ex, ey, ez, rl, e, eps;
  bool fp;
};

__device__ __forceinline__ void bond_t(const float4 g, const float4& hi, const float4& lo, const float4& hj,
                                       const float4& lj, BondT& B) {
  B.L = fabsf(g.w);
  B.rL = __fdividef(1.f, B.L);
  B.fp = g.w > 0.f;
  B.dux = (hj.x - hi.x) + (lj.x - lo.x);
  B.duy = (hj.y - hi.y) + (lj.y - lo.y);
  B.duz = (hj.z - hi.z) + (lj.z - lo.z);
  B.ex = g.x + B.dux; B.ey = g.y + B.duy; B.ez = g.z + B.duz;
  const float l2 = B.ex * B.ex + B.ey * B.ey + B.ez * B.ez;
  B.rl = rsqrtf(l2);
  const float l = l2 * B.rl;
  const float xd = g.x * B.dux + g.y * B.duy + g.z * B.duz;
  const float dd = B.dux * B.dux + B.duy * B.duy + B.duz * B.duz;
  B.e = __fdividef(2.f * xd + dd, l + B.L);
  B.eps = B.e * B.rL;
}

__device__ __forceinline__ float omega_t(int kernel, float delta, float L, float rL) {
  if (kernel == KER_LINEAR) return delta * rL;
  return omega_of_f(kernel, delta, L);
}

__device__ __forceinline__ void flag_nan_t(const DevBody& d, int kstep, float x, float y, float z) {
  if (isnan(x) || isnan(y) || isnan(z)) {
    long long step = d.ctrl->base + kstep;
    if (atomicExch(&d.ctrl->err, 1) == 0) d.ctrl->err_step = step;
    else atomicMin(&d.ctrl->err_step, step);
  }
}

__device__ __forceinline__ void flag_timeout(const DevBody& d) { atomicExch(&d.ctrl->err, 3); }

// Per-warp chunk stream over the warp's slices s = warp0, warp0 + nwarps, ...: chunk c of
// slice s covers rows [c CR, min((c+1) CR, rows(s))). A slice without rows still yields one
// empty chunk so that its points are finalised.
template <int CR, int NS>
struct Stream {
  float4* geo;                 // [NS][CR][32]
  int* nbr;                    // [NS][CR][32]
  unsigned long long* bar;     // [NS]
  long long ps;                // producer slice
  int pc, prow;                // producer chunk, rows of the producer slice
  long long pbase;

  // per-warp region, a multiple of 128 bytes so that every warp's copies land 16-byte aligned
  static constexpr unsigned BYTES = ((NS * CR * 32 * (16 + 4) + NS * 8) + 127) / 128 * 128;

  __device__ __forceinline__ void setup(unsigned char* base) {
    geo = reinterpret_cast<float4*>(base);
    nbr = reinterpret_cast<int*>(base + NS * CR * 32 * 16);
    bar = reinterpret_cast<unsigned long long*>(base + NS * CR * 32 * 20);
  }

  __device__ __forceinline__ void producer_begin(const DevBody& d, long long s0) {
    ps = s0;
    pc = 0;
    if (ps < d.nslices) {
      pbase = d.soff[ps];
      prow = (int)((d.soff[ps + 1] - pbase) >> 5);
    }
  }

  // lane 0: issue the next chunk into stage `st`; returns false when the stream is done
  __device__ __forceinline__ bool issue(const DevBody& d, long long nwarps, int st) {
    if (ps >= d.nslices) return false;
    const int r0 = pc * CR;
    const int nr = min(CR, prow - r0);
    if (nr > 0) {
      const long long slot = pbase + (long long)r0 * 32;
      tma::bar_arrive_tx(&bar[st], (unsigned)nr * 32u * 20u);
      tma::bulk_g2s(geo + st * CR * 32, d.geo + slot, (unsigned)nr * 512u, &bar[st]);
      tma::bulk_g2s(nbr + st * CR * 32, d.nbr + slot, (unsigned)nr * 128u, &bar[st]);
    } else {
      tma::bar_arrive(&bar[st]);
    }
    pc++;
    if (pc * CR >= prow) {  // next slice
      ps += nwarps;
      pc = 0;
      if (ps < d.nslices) {
        pbase = d.soff[ps];
        prow = (int)((d.soff[ps + 1] - pbase) >> 5);
      }
    }
    return true;
  }
};

#define PD_TMA_PROLOGUE(CR, NS)                                                               \
  extern __shared__ __align__(16) unsigned char pd_smem[];                                    \
  using S = Stream<CR, NS>;                                                                   \
  S st;                                                                                       \
  const int lane = threadIdx.x & 31;                                                          \
  st.setup(pd_smem + (threadIdx.x >> 5) * S::BYTES);                                          \
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;            \
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;                          \
  if (d.ctrl->err) return;                                                                    \
  if (lane == 0) {                                                                            \
    for (int q = 0; q < NS; q++) tma::bar_init(&st.bar[q], 1);                                \
    tma::fence_bar_init();                                                                    \
  }                                                                                           \
  __syncwarp();                                                                               \
  st.producer_begin(d, warp0);                                                                \
  int issued = 0;                                                                             \
  if (lane == 0)                                                                              \
    for (int q = 0; q < NS - 1; q++)                                                          \
      if (st.issue(d, nwarps, q)) issued++;                                                   \
  issued = __shfl_sync(0xffffffffu, issued, 0);                                               \
  long long t = 0; /* consumer chunk counter */                                               \
  bool timed_out = false;

// waits for chunk t (all lanes), after lane 0 refilled the stage freed by chunk t-1
#define PD_TMA_NEXT(CR, NS)                                                                   \
  __syncwarp();                                                                               \
  if (lane == 0) {                                                                            \
    if (st.issue(d, nwarps, (int)((t + NS - 1) % NS))) issued++;                              \
  }                                                                                           \
  issued = __shfl_sync(0xffffffffu, issued, 0);                                               \
  const int stg = (int)(t % NS);                                                              \
  if (!tma::bar_wait(&st.bar[stg], (unsigned)((t / NS) & 1), tma::WAIT_LIMIT)) {              \
    timed_out = true;                                                                         \
  }                                                                                           \
  timed_out = __any_sync(0xffffffffu, timed_out);

// drain: every issued chunk has been waited for, except after a timeout
#define PD_TMA_EPILOGUE(NS)                                                                   \
  if (timed_out) {                                                                            \
    if (lane == 0) flag_timeout(d);                                                           \
    for (long long q = t; q < issued; q++)                                                    \
      tma::bar_wait(&st.bar[q % NS], (unsigned)((q / NS) & 1), tma::WAIT_LIMIT);              \
  }

// -------------------------------------------------------------------------------------------
// OSB phase A (ordinary_state_based.jl:107-126, 176-204), G = 1
// -------------------------------------------------------------------------------------------
template <int CR, int NS>
__global__ void __launch_bounds__(128, PD_TMA_MINB) k_osb_a32t(DevBody d, int kstep) {
  PD_TMA_PROLOGUE(CR, NS)
  for (long long s = warp0; s < d.nslices && !timed_out; s += nwarps) {
    const long long i = s * 32 + lane;
    const bool valid = i < d.n;
    const long long sbase = d.soff[s];
    const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
    const int cnt = valid ? (int)(d.off[i + 1] - d.off[i]) : 0;
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float epsc = P.epscf, delta = P.deltaf;
    KSum m, th;
    int na = 0;
    const int nchunks = rows > 0 ? (rows + CR - 1) / CR : 1;
    for (int c = 0; c < nchunks; c++, t++) {
      PD_TMA_NEXT(CR, NS)
      if (timed_out) break;
      const int nr = min(CR, rows - c * CR);
      const float4* gs = st.geo + stg * CR * 32;
      const int* ns_ = st.nbr + stg * CR * 32;
      float4 hn = make_float4(0.f, 0.f, 0.f, 0.f), ln = hn;
      if (nr > 0 && c * CR < cnt) { const int j0 = ns_[lane]; hn = __ldg(d.uhi + j0); ln = __ldg(d.ulo + j0); }
      for (int q = 0; q < nr; q++) {
        const int r = c * CR + q;
        const long long wi = (sbase >> 5) + r;
        const unsigned word = d.bits[wi];
        const float4 hj = hn, lj = ln;
        if (q + 1 < nr && r + 1 < cnt) {
          const int j1 = ns_[(q + 1) * 32 + lane];
          hn = __ldg(d.uhi + j1);
          ln = __ldg(d.ulo + j1);
        }
        bool act = false;
        if (r < cnt) {
          const float4 g = gs[q * 32 + lane];
          BondT B;
          bond_t(g, hi, lo, hj, lj, B);
          act = ((word >> lane) & 1u) && !(B.eps > epsc && B.fp);
          if (act) {
            const float om = omega_t(d.kernel, delta, B.L, B.rL) * hj.w;
            m.add(om * (g.x * g.x + g.y * g.y + g.z * g.z));
            th.add(om * B.L * B.e);
          }
        }
        na += act;
        const unsigned nw = __ballot_sync(0xffffffffu, act);
        if (lane == 0 && nw != word) d.bits[wi] = nw;
      }
    }
    if (timed_out) break;
    if (valid) {
      const float wv = m.value();
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
  PD_TMA_EPILOGUE(NS)
}

// -------------------------------------------------------------------------------------------
// OSB phase B (ordinary_state_based.jl:128-174): b_i = sum_j (s_ij + s_ji) V_j eta / l, G = 1
// -------------------------------------------------------------------------------------------
template <int CR, int NS, bool MULTI>
__global__ void __launch_bounds__(128, PD_TMA_MINB) k_osb_b32t(DevBody d, int kstep) {
  PD_TMA_PROLOGUE(CR, NS)
  for (long long s = warp0; s < d.nslices && !timed_out; s += nwarps) {
    const long long i = s * 32 + lane;
    const bool valid = i < d.n;
    const long long sbase = d.soff[s];
    const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
    const int cnt = valid ? (int)(d.off[i + 1] - d.off[i]) : 0;
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float2 ci = valid ? d.cc32[i] : make_float2(0.f, 0.f);
    const float2 mi = (MULTI && valid) ? d.cm32[i] : make_float2(0.f, 0.f);
    KSum bx, by, bz;
    const int nchunks = rows > 0 ? (rows + CR - 1) / CR : 1;
    for (int c = 0; c < nchunks; c++, t++) {
      PD_TMA_NEXT(CR, NS)
      if (timed_out) break;
      const int nr = min(CR, rows - c * CR);
      const float4* gs = st.geo + stg * CR * 32;
      const int* ns_ = st.nbr + stg * CR * 32;
      float4 hn = make_float4(0.f, 0.f, 0.f, 0.f), ln = hn;
      float2 cn = make_float2(0.f, 0.f), mn = cn;
      if (nr > 0 && c * CR < cnt) {
        const int j0 = ns_[lane];
        hn = __ldg(d.uhi + j0);
        ln = __ldg(d.ulo + j0);
        cn = __ldg(d.cc32 + j0);
        if (MULTI) mn = __ldg(d.cm32 + j0);
      }
      for (int q = 0; q < nr; q++) {
        const int r = c * CR + q;
        const unsigned word = __ldg(d.bits + (sbase >> 5) + r);
        const float4 hj = hn, lj = ln;
        const float2 cj = cn, mj = mn;
        const int j = ns_[q * 32 + lane];
        if (q + 1 < nr && r + 1 < cnt) {
          const int j1 = ns_[(q + 1) * 32 + lane];
          hn = __ldg(d.uhi + j1);
          ln = __ldg(d.ulo + j1);
          cn = __ldg(d.cc32 + j1);
          if (MULTI) mn = __ldg(d.cm32 + j1);
        }
        if (r >= cnt) continue;
        const bool ai = (word >> lane) & 1u;
        const bool aj = d.sym ? ai : bond_bit(d.bits, rev_slot(d, sbase + (long long)r * 32 + lane, j));
        if (!(ai || aj)) continue;
        const float4 g = gs[q * 32 + lane];
        BondT B;
        bond_t(g, hi, lo, hj, lj, B);
        const DevParam* Pj = &Pi;
        if (MULTI) Pj = &d.params[d.meta[j] & META_PID_MASK];
        const float oi = ai ? omega_t(d.kernel, Pi.deltaf, B.L, B.rL) : 0.f;
        const float oj = aj ? omega_t(d.kernel, Pj->deltaf, B.L, B.rL) : 0.f;
        float c1i = ci.x, c2i = ci.y, c1j = cj.x, c2j = cj.y;
        if (MULTI) {
          c1i = mi.x == 0.f ? 0.f : 15.f * (Pi.Gf + Pj->Gf) / (2.f * mi.x);
          c2i = mi.x == 0.f ? 0.f : mi.y * (3.f * (Pi.Kf + Pj->Kf) / (2.f * mi.x) - c1i / 3.f);
          c1j = mj.x == 0.f ? 0.f : 15.f * (Pj->Gf + Pi.Gf) / (2.f * mj.x);
          c2j = mj.x == 0.f ? 0.f : mj.y * (3.f * (Pj->Kf + Pi.Kf) / (2.f * mj.x) - c1j / 3.f);
        }
        const float si = oi * (c2i * B.L + c1i * B.e);
        const float sj = oj * (c2j * B.L + c1j * B.e);
        const float f = (si + sj) * hj.w * B.rl;
        bx.add(f * B.ex); by.add(f * B.ey); bz.add(f * B.ez);
      }
    }
    if (timed_out) break;
    if (valid) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      flag_nan_t(d, kstep, x, y, z);
    }
  }
  PD_TMA_EPILOGUE(NS)
}

// -------------------------------------------------------------------------------------------
// BB (bond_based.jl:125-180), G = 1
// -------------------------------------------------------------------------------------------
template <int CR, int NS, bool MULTI>
__global__ void __launch_bounds__(128, PD_TMA_MINB) k_bb32t(DevBody d, int kstep) {
  PD_TMA_PROLOGUE(CR, NS)
  for (long long s = warp0; s < d.nslices && !timed_out; s += nwarps) {
    const long long i = s * 32 + lane;
    const bool valid = i < d.n;
    const long long sbase = d.soff[s];
    const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
    const int cnt = valid ? (int)(d.off[i + 1] - d.off[i]) : 0;
    const DevParam& P = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float4 hi = valid ? d.uhi[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lo = valid ? d.ulo[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float epsc = P.epscf, bci = P.bcf;
    KSum bx, by, bz;
    int na = 0;
    const int nchunks = rows > 0 ? (rows + CR - 1) / CR : 1;
    for (int c = 0; c < nchunks; c++, t++) {
      PD_TMA_NEXT(CR, NS)
      if (timed_out) break;
      const int nr = min(CR, rows - c * CR);
      const float4* gs = st.geo + stg * CR * 32;
      const int* ns_ = st.nbr + stg * CR * 32;
      float4 hn = make_float4(0.f, 0.f, 0.f, 0.f), ln = hn;
      if (nr > 0 && c * CR < cnt) { const int j0 = ns_[lane]; hn = __ldg(d.uhi + j0); ln = __ldg(d.ulo + j0); }
      for (int q = 0; q < nr; q++) {
        const int r = c * CR + q;
        const long long wi = (sbase >> 5) + r;
        const unsigned word = d.bits[wi];
        const float4 hj = hn, lj = ln;
        const int j = ns_[q * 32 + lane];
        if (q + 1 < nr && r + 1 < cnt) {
          const int j1 = ns_[(q + 1) * 32 + lane];
          hn = __ldg(d.uhi + j1);
          ln = __ldg(d.ulo + j1);
        }
        bool act = false;
        if (r < cnt) {
          const float4 g = gs[q * 32 + lane];
          BondT B;
          bond_t(g, hi, lo, hj, lj, B);
          act = ((word >> lane) & 1u) && !(B.eps > epsc && B.fp);
          if (act) {
            float bc = bci;
            if (MULTI) bc = 0.5f * (bci + d.params[d.meta[j] & META_PID_MASK].bcf);
            const float sc = bc * B.eps * hj.w * B.rl;
            bx.add(sc * B.ex); by.add(sc * B.ey); bz.add(sc * B.ez);
          }
        }
        na += act;
        const unsigned nw = __ballot_sync(0xffffffffu, act);
        if (lane == 0 && nw != word) d.bits[wi] = nw;
      }
    }
    if (timed_out) break;
    if (valid) {
      const float x = bx.value(), y = by.value(), z = bz.value();
      d.b32[3 * i] = x; d.b32[3 * i + 1] = y; d.b32[3 * i + 2] = z;
      d.n_active[i] = na;
      flag_nan_t(d, kstep, x, y, z);
    }
  }
  PD_TMA_EPILOGUE(NS)
}

// ------------------------------------------------------------------------------------------
// launcher: 4 warps per block, one shared-memory stream per warp
// ------------------------------------------------------------------------------------------
template <int CR, int NS>
static int launch_tma_cfg(const DevBody& d, int kstep, int phase, cudaStream_t s, int blocks_per_sm) {
  constexpr int WARPS = 4;
  const size_t smem = (size_t)WARPS * Stream<CR, NS>::BYTES;
  if (smem > 48 * 1024) {  // per device: set on every launch (cheap, capture-safe)
    cudaFuncSetAttribute(k_osb_a32t<CR, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_osb_b32t<CR, NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_osb_b32t<CR, NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_bb32t<CR, NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_bb32t<CR, NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  long long blocks = (d.nslices + WARPS - 1) / WARPS;
  const long long cap = 148LL * blocks_per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  const int grid = (int)blocks, block = WARPS * 32;
  const bool A = phase != 2, B = phase != 1;
  int launches = 0;
  if (d.material == MAT_BB) {
    if (!A) return 0;
    if (d.multi) k_bb32t<CR, NS, true><<<grid, block, smem, s>>>(d, kstep);
    else k_bb32t<CR, NS, false><<<grid, block, smem, s>>>(d, kstep);
    return 1;
  }
  if (A) { k_osb_a32t<CR, NS><<<grid, block, smem, s>>>(d, kstep); launches++; }
  if (B) {
    if (d.multi) k_osb_b32t<CR, NS, true><<<grid, block, smem, s>>>(d, kstep);
    else k_osb_b32t<CR, NS, false><<<grid, block, smem, s>>>(d, kstep);
    launches++;
  }
  return launches;
}

bool tma_supported(const DevBody& d) {
  return d.lg == 1 && d.geo != nullptr && (d.material == MAT_BB || d.material == MAT_OSB);
}

// pipe: 1 = 4 rows x 3 stages, 2 = 4 rows x 4 stages, 3 = 8 rows x 3 stages
int launch_force32_tma(const DevBody& d, int pipe, int kstep, int phase, cudaStream_t s) {
  switch (pipe) {
    case 2: return launch_tma_cfg<4, 4>(d, kstep, phase, s, 8);
    case 3: return launch_tma_cfg<8, 3>(d, kstep, phase, s, 8);
    default: return launch_tma_cfg<4, 3>(d, kstep, phase, s, 8);
  }
}

}  // namespace pd
