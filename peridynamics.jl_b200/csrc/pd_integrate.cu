// pd_integrate.cu -- Velocity Verlet kernels and small device helpers of libpdcuda.
//
// Compiled with -fmad=false so that v + a * dt/2 and u + v * dt round like the reference.
//
// One step n of the reference (velocity_verlet.jl:181-197, 239-295) is
//   v_half = v + a dt/2;  BC(t_n);  u += v_half dt, x += v_half dt;  force(t_n);
//   a = (b_int + b_ext) / rho;  v = v_half + a dt/2.
// The device runs it as [kick-drift with conditions] [force]: the kick-drift kernel of step n
// computes a_{n-1} and v_{n-1} in registers from the previous force (or reads the stored v, a
// at the start of a run), forms v_half_n, applies the point's conditions at t_n (v_half / b_ext
// components of a constrained point, found through the condition slot of the point) and moves
// the point; a finish kernel stores a and v after the last force of a run. The stored state
// between runs is exactly the reference's (v, a, v_half, u, x).
#include "pd_common.cuh"
#include "pd_launch.h"

namespace pd {

__device__ __forceinline__ double bint(const DevBody& d, const IntDev& g, long long k) {
  return g.fp32 ? (double)d.b32[k] : d.b64[k];
}

// FP32 path: the gathered copy of the displacement, {(float)u, V} and {(float)(u - hi), 0}
__device__ __forceinline__ void split_u(const DevBody& d, long long i, const double4& c) {
  const float hx = (float)c.x, hy = (float)c.y, hz = (float)c.z;
  d.uhi[i] = make_float4(hx, hy, hz, (float)c.w);
  d.ulo[i] = make_float4((float)(c.x - (double)hx), (float)(c.y - (double)hy),
                         (float)(c.z - (double)hz), 0.f);
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
  if (g.fp32) split_u(d, i, c);
}

__global__ void k_split_u(DevBody d) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  split_u(d, i, d.cur[i]);
}

__global__ void k_kick_drift(DevBody d, IntDev g, BCDev bc, int mode, double dt_override, int kstep) {
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
    if (mode == 2) {  // dynamic relaxation: drift with the stored v_half
      vh[k] = g.vh[q];
      continue;
    }
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
  if (meta & META_HAS_BC) {
    // apply_boundary_conditions! (boundary_conditions.jl:37-51, 98-108, 198-226) at t = n dt
    const int p = bc.slot[i];
    const long long step = d.ctrl->base + kstep;
    const long long row = step - d.ctrl->table_first;
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
      if (in.field == 0) {
        vh[in.dim] = v;
        g.vh[3 * i + in.dim] = v;
      } else {
        g.bext[3 * i + in.dim] = v;
      }
    }
  }
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

void launch_kick_drift(const DevBody& d, const IntDev& g, const BCDev& bc, int mode,
                       double dt_override, int kstep, cudaStream_t s) {
  k_kick_drift<<<blocks_for(d.n, 256), 256, 0, s>>>(d, g, bc, mode, dt_override, kstep);
}

void launch_split_u(const DevBody& d, cudaStream_t s) {
  if (d.n == 0 || d.uhi == nullptr) return;
  k_split_u<<<blocks_for(d.n, 256), 256, 0, s>>>(d);
}

__global__ void k_split_u_rows(DevBody d, const int* rows, long long n) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const long long i = rows[r];
  if (i < 0 || i >= d.n) return;
  split_u(d, i, d.cur[i]);
}

void launch_split_u_rows(const DevBody& d, const int* rows, long long n, cudaStream_t s) {
  if (n <= 0 || d.uhi == nullptr) return;
  k_split_u_rows<<<blocks_for(n, 256), 256, 0, s>>>(d, rows, n);
}

void launch_finish(const DevBody& d, const IntDev& g, double dt_override, cudaStream_t s) {
  k_finish<<<blocks_for(d.n, 256), 256, 0, s>>>(d, g, dt_override);
}

}  // namespace pd
