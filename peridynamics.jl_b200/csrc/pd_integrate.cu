// pd_integrate.cu -- Velocity Verlet kernels and small device helpers of libpdcuda.
//
// Compiled with -fmad=false so that v + a * dt/2 and u + v * dt round like the reference.
//
// One step n of the reference (velocity_verlet.jl:181-197, 239-295) is
//   v_half = v + a dt/2;  BC(t_n);  u += v_half dt, x += v_half dt;  force(t_n);
//   a = (b_int + b_ext) / rho;  v = v_half + a dt/2.
// The device runs it as [kick-drift] [boundary conditions] [force]: the kick-drift kernel of
// step n computes a_{n-1} and v_{n-1} in registers from the previous force (or reads the
// stored v, a at the start of a run), writes v_half_n and moves every point without
// conditions; the condition kernel overwrites v_half / b_ext of the constrained points and
// moves them; a finish kernel stores a and v after the last force of a run. The stored state
// between runs is exactly the reference's (v, a, v_half, u, x).
#include "pd_common.cuh"
#include "pd_launch.h"

namespace pd {

__device__ __forceinline__ double bint(const DevBody& d, const IntDev& g, long long k) {
  return g.fp32 ? (double)d.b32[k] : d.b64[k];
}

__device__ __forceinline__ void drift(const DevBody& d, const IntDev& g, long long i,
                                      const double* vh, double dt) {
  double4 c = d.cur[i];
  const double du0 = vh[0] * dt, du1 = vh[1] * dt, du2 = vh[2] * dt;
  if (!g.fp32) {
    g.u[3 * i] += du0; g.u[3 * i + 1] += du1; g.u[3 * i + 2] += du2;
  }
  c.x += du0; c.y += du1; c.z += du2;
  d.cur[i] = c;
}

__global__ void k_kick_drift(DevBody d, IntDev g, int mode, double dt_override, int kstep) {
  if (d.ctrl->err) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const unsigned meta = d.meta[i];
  const DevParam& P = d.params[meta & META_PID_MASK];
  const double dt = dt_override > 0 ? dt_override : P.dt;
  const double dth = 0.5 * dt;
  double vh[3];
  for (int k = 0; k < 3; k++) {
    const long long q = 3 * i + k;
    if (mode == 1) {
      double b = bint(d, g, q);
      if (meta & META_HAS_BEXT) b = b + g.bext[q];
      const double a = b / P.rho;
      const double v = g.vh[q] + a * dth;
      vh[k] = v + a * dth;
    } else {
      vh[k] = g.v[q] + g.a[q] * dth;
    }
    g.vh[q] = vh[k];
  }
  if (!(meta & META_HAS_BC)) drift(d, g, i, vh, dt);
}

// apply_boundary_conditions! (boundary_conditions.jl:37-51, 98-108, 198-226) at t = n dt for
// the constrained points, then their update_disp_and_pos!
__global__ void k_bc(DevBody d, IntDev g, BCDev bc, double dt_override, int kstep) {
  if (d.ctrl->err) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= bc.n_points) return;
  const long long i = bc.point[p];
  const long long step = d.ctrl->base + kstep;
  const long long row = step - d.ctrl->table_first;
  const DevParam& P = d.params[d.meta[i] & META_PID_MASK];
  const double dt = dt_override > 0 ? dt_override : P.dt;
  for (int e = bc.entry_off[p]; e < bc.entry_off[p + 1]; e++) {
    const BCEntry en = bc.entry[e];
    const BCInfo in = bc.info[en.bc];
    double v;
    if (in.kind == 2) {
      v = bc.data[in.col + en.q];
    } else {
      if (row < 0 || row >= d.ctrl->table_n) {
        atomicExch(&d.ctrl->err, 2);
        d.ctrl->err_step = step;
        return;
      }
      v = bc.table[row * bc.per_step + in.col + (in.kind == 1 ? en.q : 0)];
    }
    if (!isfinite(v)) continue;
    double* field = in.field == 0 ? g.vh : g.bext;
    field[3 * i + in.dim] = v;
  }
  double vh[3] = {g.vh[3 * i], g.vh[3 * i + 1], g.vh[3 * i + 2]};
  drift(d, g, i, vh, dt);
}

__global__ void k_finish(DevBody d, IntDev g, double dt_override) {
  if (d.ctrl->err) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const unsigned meta = d.meta[i];
  const DevParam& P = d.params[meta & META_PID_MASK];
  const double dt = dt_override > 0 ? dt_override : P.dt;
  const double dth = 0.5 * dt;
  for (int k = 0; k < 3; k++) {
    const long long q = 3 * i + k;
    double b = bint(d, g, q);
    if (meta & META_HAS_BEXT) b = b + g.bext[q];
    const double a = b / P.rho;
    g.a[q] = a;
    g.v[q] = g.vh[q] + a * dth;
  }
}

static inline int blocks_for(long long n, int t) {
  long long b = (n + t - 1) / t;
  return (int)(b < 1 ? 1 : b);
}

void launch_kick_drift(const DevBody& d, const IntDev& g, int mode, double dt_override, int kstep,
                       cudaStream_t s) {
  k_kick_drift<<<blocks_for(d.n, 256), 256, 0, s>>>(d, g, mode, dt_override, kstep);
}

void launch_bc(const DevBody& d, const IntDev& g, const BCDev& bc, double dt_override, int kstep,
               cudaStream_t s) {
  if (bc.n_points == 0) return;
  k_bc<<<blocks_for(bc.n_points, 128), 128, 0, s>>>(d, g, bc, dt_override, kstep);
}

void launch_finish(const DevBody& d, const IntDev& g, double dt_override, cudaStream_t s) {
  k_finish<<<blocks_for(d.n, 256), 256, 0, s>>>(d, g, dt_override);
}

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
__global__ void k_pack_bits(const unsigned char* bytes, unsigned int* bits, long long nb) {
  const long long wi = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nw = (nb + 31) / 32;
  if (wi >= nw) return;
  unsigned int w = 0;
  for (int k = 0; k < 32; k++) {
    const long long b = wi * 32 + k;
    if (b < nb && bytes[b]) w |= 1u << k;
  }
  bits[wi] = w;
}

void launch_pack_bits(const unsigned char* bytes, unsigned int* bits, long long nb, cudaStream_t s) {
  const long long nw = (nb + 31) / 32;
  if (nw == 0) return;
  k_pack_bits<<<blocks_for(nw, 256), 256, 0, s>>>(bytes, bits, nb);
}

// bond_active of the reference: the stored bit, and no bond of a killed point
__global__ void k_export_bond_active(DevBody d, unsigned char* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const bool killed = d.meta[i] & META_KILLED;
  for (long long b = d.off[i]; b < d.off[i + 1]; b++)
    out[b] = killed ? 0 : (unsigned char)((d.bits[b >> 5] >> (b & 31)) & 1u);
}

void launch_export_bond_active(const DevBody& d, unsigned char* out, cudaStream_t s) {
  k_export_bond_active<<<blocks_for(d.n, 256), 256, 0, s>>>(d, out);
}

__global__ void k_count_active(DevBody d) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  int na = 0;
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) na += (d.bits[b >> 5] >> (b & 31)) & 1u;
  d.n_active[i] = (d.meta[i] & META_KILLED) ? 0 : na;
}

void launch_count_active(const DevBody& d, cudaStream_t s) {
  k_count_active<<<blocks_for(d.n, 256), 256, 0, s>>>(d);
}

// reverse bond of b = (i -> j): position of i in the bond list of j, or -1.
// flags[0] = 1 if some bond has no reverse.
__global__ void k_reverse(DevBody d, int* rev, int* flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    const int j = d.nbr[b];
    long long lo = d.off[j], hi = d.off[j + 1];
    long long found = -1;
    // lists are sorted in the common case: binary search, then a linear fallback
    long long a = lo, z = hi;
    while (a < z) {
      const long long mid = (a + z) / 2;
      if (d.nbr[mid] < i) a = mid + 1; else z = mid;
    }
    if (a < hi && d.nbr[a] == i) found = a;
    if (found < 0)
      for (long long c = lo; c < hi; c++)
        if (d.nbr[c] == i) { found = c; break; }
    rev[b] = (int)found;
    if (found < 0) flags[0] = 1;
  }
}

void launch_reverse(const DevBody& d, int* rev, int* flags, cudaStream_t s) {
  k_reverse<<<blocks_for(d.n, 256), 256, 0, s>>>(d, rev, flags);
}

// flags[1] = 1 if a bond and its reverse differ in state; flags[2] = 1 if a fail-permitted
// bond joins points of different critical stretch
__global__ void k_check_sym(DevBody d, const int* rev, int* flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam& Pi = d.params[d.meta[i] & META_PID_MASK];
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    const long long r = rev[b];
    if (r < 0) continue;
    const bool a = (d.bits[b >> 5] >> (b & 31)) & 1u;
    const bool c = (d.bits[r >> 5] >> (r & 31)) & 1u;
    if (a != c) flags[1] = 1;
    const int j = d.nbr[b];
    const DevParam& Pj = d.params[d.meta[j] & META_PID_MASK];
    bool permitted = d.len64 ? (d.len64[b] > 0) : (d.geo[b].w > 0);
    if (permitted && (Pi.epsc != Pj.epsc || Pi.epscf != Pj.epscf)) flags[2] = 1;
  }
}

void launch_check_sym(const DevBody& d, const int* rev, int* flags, cudaStream_t s) {
  k_check_sym<<<blocks_for(d.n, 256), 256, 0, s>>>(d, rev, flags);
}

// calc_damage! (bond_system.jl:338-343) from the active-bond count
__global__ void k_export_damage(DevBody d, int valid, double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const long long nn = d.off[i + 1] - d.off[i];
  out[i] = valid ? 1 - (double)d.n_active[i] / (double)nn : 0.0;
}

void launch_export_damage(const DevBody& d, int valid, double* out, cudaStream_t s) {
  k_export_damage<<<blocks_for(d.n, 256), 256, 0, s>>>(d, valid, out);
}

// what = 0: position, 1: displacement
__global__ void k_export_position(DevBody d, IntDev g, double* out, int what) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 c = d.cur[i], X = d.X0[i];
  double r[3];
  if (!g.fp32) {
    if (what == 0) { r[0] = c.x; r[1] = c.y; r[2] = c.z; }
    else { r[0] = g.u[3 * i]; r[1] = g.u[3 * i + 1]; r[2] = g.u[3 * i + 2]; }
  } else {
    if (what == 0) { r[0] = X.x + c.x; r[1] = X.y + c.y; r[2] = X.z + c.z; }
    else { r[0] = c.x; r[1] = c.y; r[2] = c.z; }
  }
  out[3 * i] = r[0]; out[3 * i + 1] = r[1]; out[3 * i + 2] = r[2];
}

void launch_export_position(const DevBody& d, const IntDev& g, double* out, int what, cudaStream_t s) {
  k_export_position<<<blocks_for(d.n, 256), 256, 0, s>>>(d, g, out, what);
}

// calc_timestep_point (bond_system.jl:269-277): sqrt(2 rho / sum_j V_j bc / L)
__global__ void k_timestep(DevBody d, double* dtp) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam& P = d.params[d.meta[i] & META_PID_MASK];
  double dtsum = 0.0;
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    const int j = d.nbr[b];
    double L;
    if (d.len64) {
      L = fabs(d.len64[b]);
    } else {  // FP32 path: the FP64 length from the reference positions, as the bond search
      const double4 Xi = d.X0[i], Xj = d.X0[j];
      const double dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
      L = sqrt((dx * dx + dy * dy) + dz * dz);
    }
    dtsum += d.X0[j].w * P.bc / L;
  }
  dtp[i] = sqrt(2 * P.rho / dtsum);
}

void launch_timestep(const DevBody& d, double* dt_point, cudaStream_t s) {
  k_timestep<<<blocks_for(d.n, 256), 256, 0, s>>>(d, dt_point);
}

}  // namespace pd

namespace pd {

// bond geometry of the FP64 path: L with the sign carrying fail_permit (negative = no failure)
__global__ void k_build_len64(DevBody d, const double* L, const unsigned char* fp, double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 Xi = d.X0[i];
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    double Lb;
    if (L) {
      Lb = L[b];
    } else {
      const double4 Xj = d.X0[d.nbr[b]];
      const double dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
      Lb = sqrt((dx * dx + dy * dy) + dz * dz);
    }
    out[b] = (fp == nullptr || fp[b]) ? Lb : -Lb;
  }
}

// bond geometry of the FP32 path: {xi = X_j - X_i, +-L}
__global__ void k_build_geo(DevBody d, const double* L, const unsigned char* fp, float4* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 Xi = d.X0[i];
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    const double4 Xj = d.X0[d.nbr[b]];
    const double gx = Xj.x - Xi.x, gy = Xj.y - Xi.y, gz = Xj.z - Xi.z;
    double Lb;
    if (L) {
      Lb = L[b];
    } else {
      const double dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
      Lb = sqrt((dx * dx + dy * dy) + dz * dz);
    }
    const float Lf = (float)Lb;
    out[b] = make_float4((float)gx, (float)gy, (float)gz, (fp == nullptr || fp[b]) ? Lf : -Lf);
  }
}

void launch_build_len64(const DevBody& d, const double* L, const unsigned char* fp, double* out, cudaStream_t s) {
  k_build_len64<<<blocks_for(d.n, 256), 256, 0, s>>>(d, L, fp, out);
}

void launch_build_geo(const DevBody& d, const double* L, const unsigned char* fp, float4* out, cudaStream_t s) {
  k_build_geo<<<blocks_for(d.n, 256), 256, 0, s>>>(d, L, fp, out);
}

}  // namespace pd

namespace pd {

// break_bonds! (bond_system.jl:249-267): bonds between a point of set a and a point of set b
// become inactive
__global__ void k_break_sets(DevBody d, const unsigned char* A, const unsigned char* B) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    const int j = d.nbr[b];
    if ((A[i] && B[j]) || (B[i] && A[j])) atomicAnd(d.bits + (b >> 5), ~(1u << (b & 31)));
  }
}

void launch_break_sets(const DevBody& d, const unsigned char* A, const unsigned char* B, cudaStream_t s) {
  k_break_sets<<<blocks_for(d.n, 256), 256, 0, s>>>(d, A, B);
}

// synthetic initial damage: the pair {i, j} is broken when a hash of (min, max, seed) falls
// below the fraction, so both directions of a pair share the state
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27; x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

__global__ void k_break_random(DevBody d, unsigned long long threshold, unsigned long long seed) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  for (long long b = d.off[i]; b < d.off[i + 1]; b++) {
    const unsigned long long j = (unsigned long long)d.nbr[b];
    const unsigned long long lo = j < (unsigned long long)i ? j : (unsigned long long)i;
    const unsigned long long hi = j < (unsigned long long)i ? (unsigned long long)i : j;
    const unsigned long long r = mix64(mix64(lo * 0x9e3779b97f4a7c15ull + seed) ^ hi);
    if (r < threshold) atomicAnd(d.bits + (b >> 5), ~(1u << (b & 31)));
  }
}

void launch_break_random(const DevBody& d, double fraction, unsigned long long seed, cudaStream_t s) {
  const long double t = (long double)fraction * 18446744073709551616.0L;
  const unsigned long long thr = fraction >= 1.0 ? ~0ull : (unsigned long long)t;
  k_break_random<<<blocks_for(d.n, 256), 256, 0, s>>>(d, thr, seed);
}

}  // namespace pd
