// pd_common.cuh -- device-side data layout of one body and small helpers shared by the
// force, integration and neighbour-search kernels of libpdcuda.
//
// HBM layout of one body (n points, B directed bonds, CSR by point):
//   off      int64[n+1]   n_neighbors of point i is off[i+1] - off[i] (the reference's CSR
//                         order: bond k of point i is bond off[i] + k of the reference)
//   Bond arrays are stored in a sliced layout with G lanes per point ("SELL"): the points
//   are cut into slices of P = 32 / G consecutive points; slice s owns rows
//   [soff[s] / 32, soff[s+1] / 32) of 32 bond slots; bond k of the point p of the slice sits
//   in row k / G at lane p * G + k % G. A warp walks one slice row by row, so every
//   bond-array load of a warp is one contiguous 128-byte (int32) or 512-byte (float4)
//   segment, and the 32 bond_active bits of a row are one word owned by that warp.
//   soff     int64[S+1]   slot offset of every slice (multiple of 32)
//   nbr      int32[slots] neighbour index j (padding slots: 0)
//   bits     uint32[slots/32] bond_active, bit (slot & 31) of word slot >> 5 (padding: 0)
//   revk     int32[slots] position k' of i in the bond list of j (only for asymmetric states)
//   FP64 path: len64 double[slots] reference length L, negative when failure is not permitted
//   FP32 path: geo  float4[slots]  {xi_x, xi_y, xi_z, +-L}: reference bond vector X_j - X_i
//              and length, the sign of w carrying fail_permit (negative = not permitted)
//   X0       double4[n]   {X, Y, Z, V}: reference position and volume
//   cur      double4[n]   FP64 path: {x, y, z, V} current position (kept incrementally as the
//                         reference does); FP32 path: {u_x, u_y, u_z, V} displacement
//   FP32 path, gathered by the bond loops: uhi float4[n] {(float)u, V} and ulo float4[n]
//                         {(float)(u - hi), 0}: u_j - u_i = (hi_j - hi_i) + (lo_j - lo_i) in
//                         FP32 carries the FP64 difference to FP32 precision
//   meta     uint32[n]    parameter-set id (bits 0-15) and point flags
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// occupancy bounds of the force kernels: blocks of up to 256 threads, at least PD_MINB
// (PD_MINB_A for the OSB phase-A kernel) resident blocks per SM, which caps the registers per
// thread at 64 (51). Measured on the 8M-point OSB block: these caps beat the uncapped
// allocation by 1.25x (phase B) and 1.2x (phase A).
#ifndef PD_MINB
#define PD_MINB 4
#endif
#ifndef PD_MINB_A
#define PD_MINB_A 5
#endif
#define PD_LB __launch_bounds__(256, PD_MINB)
#define PD_LB_A __launch_bounds__(256, PD_MINB_A)
// FP64 kernels keep more registers (their 3x3 FP64 algebra spills under the FP32 caps)
#define PD_LB64 __launch_bounds__(256, 2)

namespace pd {

constexpr uint32_t META_PID_MASK = 0xFFFFu;
constexpr uint32_t META_KILLED = 1u << 16;  // CMaterial: all bonds killed (too_much_damage!)
constexpr uint32_t META_HAS_BC = 1u << 17;  // point carries boundary conditions
constexpr uint32_t META_HAS_BEXT = 1u << 18; // point has a nonzero or prescribed b_ext
// halo row of a partitioned body: a copy of a point another partition owns, bonded only to
// owned points; its state is overwritten by halo exchanges, and the owner decides its kills
constexpr uint32_t META_HALO = 1u << 19;

enum Material : int { MAT_BB = 0, MAT_OSB = 1, MAT_CMAT = 2 };
enum CModel : int { CM_SVK = 0, CM_NEOHOOKE = 1, CM_NHPENALTY = 2 };
enum Kernel : int { KER_CONST_ONE = 0, KER_LINEAR = 1, KER_CUBIC_BSPLINE = 2 };
// CMat zero-energy mode stabilisation (zem_stabilization.jl)
enum Zem : int { ZEM_SILLING = 0, ZEM_WAN = 1 };

// One parameter set (StandardPointParameters) with the derived per-set constants.
struct DevParam {
  double delta, rho, bc, epsc, G, K, lambda, mu, beta;  // beta = Cs * bc / delta
  double zwa;                                           // (1 - nu) lambda / nu (Hooke diagonal)
  double dt, dth;                                       // integration step of the set
  float deltaf, bcf, epscf, Gf, Kf, lambdaf, muf, betaf, zwaf;
  float inv_delta;  // 1 / delta (FP32 correspondence scaling)
  float vscale;     // 1 / delta^3 (FP32 correspondence scaling)
};

struct Ctrl {
  long long base;        // step number of the first step of the current launch block
  long long table_first; // first step held in the boundary-condition value table
  long long table_n;     // steps held in the table
  int err;               // 1: NaN in b_int; 2: boundary values missing for a step;
                         // 3: a bounded wait gave up; 4: halo row index outside the body
  int pad;
  long long err_step;
};

struct DevBody {
  long long n, nb;
  const long long* off;
  const long long* soff;
  long long nslices;
  int lg;            // lanes per point of the bond layout
  const int* nbr;
  unsigned int* bits;
  const int* rev;    // revk
  const double* len64;
  const float4* geo;
  const double4* X0;
  double4* cur;
  unsigned int* meta;
  const DevParam* params;
  int* n_active;
  double* b64;
  float* b32;
  double4* coef64;   // OSB FP64: {c1, c2, wvol, dil}
  float2* cc32;      // OSB FP32: {c1, c2}
  float2* cm32;      // OSB FP32: {wvol, dil}
  float4* uhi;       // FP32 path: {(float)u, V}
  float4* ulo;       // FP32 path: {(float)(u - hi), 0}
  double* F64;       // CMat FP64: deformation gradient F (9 per point, column-major)
  double* PK64;      // CMat FP64: P K^-1 (9 per point)
  float* H32;        // CMat FP32: displacement gradient H = F - I (9 per point)
  float4* cst32;     // CMat FP32: 3 float4 per point {A (9), beta~, 0, 0}
  // CMat with ZEMWan: the stabilising stiffness C : K^-1 of every point (FP64: 9 per point,
  // column-major; FP32: 2 float4 per point {S00, S11, S22, S01}, {S02, S12, 0, 0}); null with
  // ZEMSilling
  double* C164;
  float4* zw32;
  float* K32;        // CMat FP32: the scaled shape tensor of every point {xx, yy, zz, xy, xz, yz}
  // EnergySurfaceCorrection (BB, OSB): the factor of every bond slot (FP64 / FP32 path) and
  // the per-point multiplication factors {x, y, z} it is made from; null without correction
  const double* sc64;
  const float* sc32;
  double* mf;
  Ctrl* ctrl;
  int material, kernel, cmodel, sym, multi, zem;
  double maxdmg;
  double cs;
};

// ---------------------------------------------------------------------------------------
// influence function (kernels.jl:10-52); evaluated with the horizon of the bond owner
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double omega_of(int kernel, double delta, double L) {
  if (kernel == KER_LINEAR) return delta / L;
  if (kernel == KER_CONST_ONE) return 1.0;
  double xi = L / delta;
  if (0 < xi && xi <= 0.5) return 2.0 / 3.0 - 4 * (xi * xi) + 4 * (xi * xi * xi);
  if (0.5 < xi && xi <= 1) return 4.0 / 3.0 - 4 * xi + 4 * (xi * xi) - 4.0 / 3.0 * (xi * xi * xi);
  return 0.0;
}

__device__ __forceinline__ float omega_of_f(int kernel, float delta, float L) {
  if (kernel == KER_LINEAR) return delta / L;
  if (kernel == KER_CONST_ONE) return 1.0f;
  float xi = L / delta;
  if (0 < xi && xi <= 0.5f) return 2.0f / 3.0f - 4 * (xi * xi) + 4 * (xi * xi * xi);
  if (0.5f < xi && xi <= 1) return 4.0f / 3.0f - 4 * xi + 4 * (xi * xi) - 4.0f / 3.0f * (xi * xi * xi);
  return 0.0f;
}

// slot of bond k of point i in the sliced layout
__device__ __forceinline__ long long bond_slot(const DevBody& d, long long i, int k) {
  const int G = d.lg, P = 32 / G;
  const long long s = i / P;
  const int p = (int)(i - s * P);
  return d.soff[s] + (long long)(k / G) * 32 + p * G + (k % G);
}

// slot of the reverse bond j -> i of the bond in slot b (asymmetric bond states)
__device__ __forceinline__ long long rev_slot(const DevBody& d, long long b, int j) {
  return bond_slot(d, j, __ldg(d.rev + b));
}

__device__ __forceinline__ bool bond_bit(const unsigned int* bits, long long b) {
  return (__ldg(bits + (b >> 5)) >> (b & 31)) & 1u;
}

__device__ __forceinline__ bool bond_bit_live(const unsigned int* bits, long long b) {
  // the word may be cleared by another group while this kernel runs: plain (non-__ldg) load
  return (bits[b >> 5] >> (b & 31)) & 1u;
}

__device__ __forceinline__ void clear_bit(unsigned int* bits, long long b) {
  atomicAnd(bits + (b >> 5), ~(1u << (b & 31)));
}

// Warp-uniform loop over the slices of the bond layout: one warp per slice; all lanes of a
// warp walk the same rows, so ballots and group shuffles always see the full warp.
#define PD_SLICE_LOOP(G)                                                                    \
  constexpr int PPW = 32 / (G);                                                             \
  const int lane = threadIdx.x & 31;                                                        \
  const int sub = lane / (G), gl = lane % (G);                                              \
  (void)sub; (void)gl;                                                                      \
  const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;          \
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;                        \
  for (long long s = warp0; s < d.nslices; s += nwarps)

// point, slice rows and bond count of the lane
#define PD_SLICE_SETUP                                                                      \
  const long long i = s * PPW + sub;                                                        \
  const bool valid = i < d.n;                                                               \
  const long long sbase = d.soff[s];                                                        \
  const int rows = (int)((d.soff[s + 1] - sbase) >> 5);                                     \
  const int cnt = valid ? (int)(d.off[i + 1] - d.off[i]) : 0;

// ---------------------------------------------------------------------------------------
// compensated (Kahan) FP32 accumulation and its lane-group reduction (partners combined with
// TwoSum)
// ---------------------------------------------------------------------------------------
struct KSum {
  float s, c;
  __device__ __forceinline__ KSum() : s(0.f), c(0.f) {}
  // Kahan: c carries the low-order part lost by the previous additions
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s - c; }
};

// lanes [g*G, g*G+G) of a warp form one group; fixed butterfly order => deterministic.
// Partner sums are combined with TwoSum, their compensations added.
template <int G>
__device__ __forceinline__ void group_reduce(KSum& k) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const float s2 = __shfl_down_sync(0xffffffffu, k.s, o, G);
    const float c2 = __shfl_down_sync(0xffffffffu, k.c, o, G);
    const float t = k.s + s2;
    const float z = t - k.s;
    const float e = (k.s - (t - z)) + (s2 - z);
    k.s = t;
    k.c = (k.c + c2) - e;
  }
}

template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, G);
  return v;
}

template <int G, typename T>
__device__ __forceinline__ T group_bcast(T v) {
  return __shfl_sync(0xffffffffu, v, 0, G);
}

template <int G>
__device__ __forceinline__ bool group_any(bool p) {
  unsigned m = __ballot_sync(0xffffffffu, p);
  if (G == 32) return m != 0;
  unsigned lane = threadIdx.x & 31;
  unsigned grp = (lane / G) * G;
  unsigned gm = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << grp);
  return (m & gm) != 0;
}

}  // namespace pd
