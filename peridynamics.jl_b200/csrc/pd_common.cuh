// pd_common.cuh -- device-side data layout of one body and small helpers shared by the
// force, integration and neighbour-search kernels of libpdcuda.
//
// HBM layout of one body (n points, B directed bonds, CSR by point):
//   off      int64[n+1]   bond range of point i is [off[i], off[i+1])
//   nbr      int32[B]     neighbour index j
//   bits     uint32[B/32] bond_active, one bit per bond (bit b&31 of word b>>5)
//   rev      int32[B]     index of the reverse bond j->i (only for asymmetric bond states)
//   FP64 path: len64 double[B] reference length L, negative when failure is not permitted
//   FP32 path: geo  float4[B]  {xi_x, xi_y, xi_z, +-L}: reference bond vector X_j - X_i and
//              length, the sign of w carrying fail_permit (negative = not permitted)
//   X0       double4[n]   {X, Y, Z, V}: reference position and volume
//   cur      double4[n]   FP64 path: {x, y, z, V} current position (kept incrementally as the
//                         reference does); FP32 path: {u_x, u_y, u_z, V} displacement
//   meta     uint32[n]    parameter-set id (bits 0-15) and point flags
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pd {

constexpr uint32_t META_PID_MASK = 0xFFFFu;
constexpr uint32_t META_KILLED = 1u << 16;  // CMaterial: all bonds killed (too_much_damage!)
constexpr uint32_t META_HAS_BC = 1u << 17;  // point carries boundary conditions
constexpr uint32_t META_HAS_BEXT = 1u << 18; // point has a nonzero or prescribed b_ext

enum Material : int { MAT_BB = 0, MAT_OSB = 1, MAT_CMAT = 2 };
enum CModel : int { CM_SVK = 0, CM_NEOHOOKE = 1, CM_NHPENALTY = 2 };
enum Kernel : int { KER_CONST_ONE = 0, KER_LINEAR = 1, KER_CUBIC_BSPLINE = 2 };

// One parameter set (StandardPointParameters) with the derived per-set constants.
struct DevParam {
  double delta, rho, bc, epsc, G, K, lambda, mu, beta;  // beta = Cs * bc / delta
  double dt, dth;                                       // integration step of the set
  float deltaf, bcf, epscf, Gf, Kf, lambdaf, muf, betaf;
  float inv_delta;  // 1 / delta (FP32 correspondence scaling)
  float vscale;     // 1 / delta^3 (FP32 correspondence scaling)
};

struct Ctrl {
  long long base;        // step number of the first step of the current launch block
  long long table_first; // first step held in the boundary-condition value table
  long long table_n;     // steps held in the table
  int err;               // 1: NaN in b_int; 2: boundary values missing for a step
  int pad;
  long long err_step;
};

struct DevBody {
  long long n, nb;
  const long long* off;
  const int* nbr;
  unsigned int* bits;
  const int* rev;
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
  float4* coef32;    // OSB FP32: {c1, c2, wvol, dil}
  double* F64;       // CMat FP64: deformation gradient F (9 per point, column-major)
  double* PK64;      // CMat FP64: P K^-1 (9 per point)
  float* H32;        // CMat FP32: displacement gradient H = F - I (9 per point)
  float4* cst32;     // CMat FP32: 3 float4 per point {A (9), beta~, 0, 0}
  Ctrl* ctrl;
  int material, kernel, cmodel, sym, multi;
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

// ---------------------------------------------------------------------------------------
// compensated (Kahan-Babuska / Neumaier) FP32 accumulation and its lane-group reduction
// ---------------------------------------------------------------------------------------
struct KSum {
  float s, c;
  __device__ __forceinline__ KSum() : s(0.f), c(0.f) {}
  __device__ __forceinline__ void add(float x) {
    float t = s + x;
    // Neumaier: the rounding error of s + x, whichever operand is larger
    c += (fabsf(s) >= fabsf(x)) ? ((s - t) + x) : ((x - t) + s);
    s = t;
  }
  __device__ __forceinline__ float value() const { return s + c; }
};

// lanes [g*G, g*G+G) of a warp form one group; fixed butterfly order => deterministic
template <int G>
__device__ __forceinline__ void group_reduce(KSum& k) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    float s2 = __shfl_down_sync(0xffffffffu, k.s, o, G);
    float c2 = __shfl_down_sync(0xffffffffu, k.c, o, G);
    float t = k.s + s2;
    float e = (fabsf(k.s) >= fabsf(s2)) ? ((k.s - t) + s2) : ((s2 - t) + k.s);
    k.s = t;
    k.c = (k.c + c2) + e;
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
