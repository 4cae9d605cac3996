// pd_dr.cu -- dynamic relaxation on the device (src/time_solvers/dynamic_relaxation.jl of the
// reference): the adaptive-damping explicit solver for quasi-static problems that runs on the
// same force kernels as Velocity Verlet.
//
// One step n (relaxation_timestep!, :191-211), t = n dt:
//   conditions at t and u += v_half dt, x += v_half dt        (the Velocity Verlet drift kernels,
//                                                               mode 2: no kick)
//   force density at t
//   n > 1: damping cn = 2 sqrt(cn1 / cn2) (clamped to 1.9 above 2, 0 when not positive) with
//          cn1 = sum over dofs with v_half != 0 of -u^2 (b_int - b_int_old) / (dt Lambda v_half_old),
//          cn2 = sum of u^2, both compensated (TwoSum) sums     (damping_terms, :276-317)
//   v_half = 0.5 dt (b_int + b_ext) / Lambda (n = 1), else
//          ((2 - cn dt) v_half_old + 2 dt a) / (2 + cn dt), a = (b_int + b_ext) / Lambda
//   v = (v_half_old + v_half) / 2, v_half_old = v_half, b_int_old = b_int
// with the fictitious density Lambda_i = f / 4 dt^2 n_i 5 pi delta^2 bc (calc_density_matrix!,
// :153-164). With the serial mapping the damping sums run in the reference's order on one
// thread, so the FP64 trajectories equal the serial CPU restatement bit for bit; otherwise
// they are summed over a fixed partition and fixed combination trees (deterministic).
// Compiled with -fmad=false, in the reference's operation order.
#include <cmath>
#include <cstddef>
#include <vector>

#include "pd_handle.h"

namespace pd {

constexpr int DR_NB = 148 * 8;   // blocks of the damping reduction (8 per SM)
constexpr int DR_TPB = 256;

struct DRState {
  double* lam = nullptr;   // [n] Lambda (the same for the three dofs of a point)
  double* vho = nullptr;   // [3n] v_half_old
  double* bo = nullptr;    // [3n] b_int_old
  double* part = nullptr;  // [4 DR_NB] partial (cn1, cn1_c, cn2, cn2_c)
  double* cn = nullptr;    // [1]
  double dt = 0.0, factor = 1.0;
};

void dr_release(pd_handle* h) {
  delete h->dr;  // device arrays are in h->allocs and freed with the handle
  h->dr = nullptr;
}

__device__ __forceinline__ double dr_bint(const DevBody& d, const IntDev& g, long long q) {
  return g.fp32 ? (double)d.b32[q] : d.b64[q];
}

__device__ __forceinline__ double dr_u(const DevBody& d, const IntDev& g, long long q) {
  if (!g.fp32) return g.u[q];
  const double* c = reinterpret_cast<const double*>(d.cur + q / 3);
  return c[q % 3];
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double v = s - a;
  e = (a - (s - v)) + (b - v);
}

__global__ void k_dr_lam(DevBody d, double factor, double dt, double* lam) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam& P = d.params[d.meta[i] & META_PID_MASK];
  const double nb = (double)(d.off[i + 1] - d.off[i]);
  const double k = (5.0 * M_PI) * (P.delta * P.delta) * P.bc;
  lam[i] = factor * 1.0 / 4.0 * (dt * dt) * nb * k;
}

// the damping terms of dofs [q0, q1) in order, accumulated into (s1, c1, s2, c2)
__device__ __forceinline__ void dr_terms(const DevBody& d, const IntDev& g, const double* lam,
                                         const double* vho, const double* bo, double dt, long long q0,
                                         long long q1, double& s1, double& c1, double& s2, double& c2) {
  for (long long q = q0; q < q1; q++) {
    const double u = dr_u(d, g, q);
    double e;
    if (g.vh[q] != 0.0) {
      const double db = dr_bint(d, g, q) - bo[q];
      const double temp = dt * lam[q / 3] * vho[q];
      two_sum(s1, -(u * u) * db / temp, s1, e);
      c1 += e;
    }
    two_sum(s2, u * u, s2, e);
    c2 += e;
  }
}

__device__ __forceinline__ double finish_damping(double cn1, double cn2) {
  double cn = 0.0;
  if (cn2 != 0.0 && cn1 / cn2 > 0.0) cn = 2.0 * sqrt(cn1 / cn2);
  if (cn > 2.0) cn = 1.9;
  return cn;
}

// serial order: one thread, all dofs (the reference with one chunk)
__global__ void k_dr_damping_serial(DevBody d, IntDev g, const double* lam, const double* vho,
                                    const double* bo, double dt, double* cn) {
  if (d.ctrl->err) return;
  double s1 = 0.0, c1 = 0.0, s2 = 0.0, c2 = 0.0;
  dr_terms(d, g, lam, vho, bo, dt, 0, 3 * d.n, s1, c1, s2, c2);
  *cn = finish_damping(s1 + c1, s2 + c2);
}

// combine (a, b) of the reference (:295-301) into a
__device__ __forceinline__ void dr_combine(double* a, const double* b) {
  double s, e1, e2;
  two_sum(a[0], b[0], s, e1);
  a[1] = a[1] + b[1] + e1;
  a[0] = s;
  two_sum(a[2], b[2], s, e2);
  a[3] = a[3] + b[3] + e2;
  a[2] = s;
}

__device__ __forceinline__ void dr_shfl_combine(double* a, int off) {
  double b[4];
  for (int k = 0; k < 4; k++) b[k] = __shfl_down_sync(0xffffffffu, a[k], off);
  dr_combine(a, b);
}

// a fixed tree over the block's threads (deterministic); the result is in thread 0
__device__ __forceinline__ void dr_block_combine(double* acc) {
  __shared__ double sh[DR_TPB / 32][4];
  for (int off = 16; off > 0; off >>= 1) dr_shfl_combine(acc, off);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int k = 0; k < 4; k++) sh[w][k] = acc[k];
  __syncthreads();
  if (w == 0) {
    for (int k = 0; k < 4; k++) acc[k] = l < DR_TPB / 32 ? sh[l][k] : 0.0;
    for (int off = DR_TPB / 64; off > 0; off >>= 1) dr_shfl_combine(acc, off);
  }
}

// fixed partition: thread t of the grid sums the dofs t, t + T, t + 2T, ... (T threads in the
// grid: coalesced), then the block and a last kernel combine the partial sums over fixed trees
__global__ void __launch_bounds__(DR_TPB) k_dr_damping_part(DevBody d, IntDev g, const double* lam,
                                                            const double* vho, const double* bo,
                                                            double dt, double* part) {
  const long long nd = 3 * d.n;
  const long long T = (long long)gridDim.x * blockDim.x;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nd; q += T) {
    const double u = dr_u(d, g, q);
    double e;
    if (g.vh[q] != 0.0) {
      const double db = dr_bint(d, g, q) - bo[q];
      const double temp = dt * lam[q / 3] * vho[q];
      two_sum(acc[0], -(u * u) * db / temp, acc[0], e);
      acc[1] += e;
    }
    two_sum(acc[2], u * u, acc[2], e);
    acc[3] += e;
  }
  dr_block_combine(acc);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) part[4 * blockIdx.x + k] = acc[k];
}

__global__ void __launch_bounds__(DR_TPB) k_dr_damping_finish(DevBody d, const double* part, int nb,
                                                              double* cn) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nb; b += blockDim.x) dr_combine(acc, part + 4 * b);
  dr_block_combine(acc);
  if (threadIdx.x == 0 && !d.ctrl->err) *cn = finish_damping(acc[0] + acc[1], acc[2] + acc[3]);
}

// relaxation_first_step! / relaxation_step! and relaxation_updates! (:337-370)
__global__ void k_dr_update(DevBody d, IntDev g, const double* lam, double* vho, double* bo,
                            const double* cnp, double dt, int first) {
  if (d.ctrl->err) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double L = lam[i];
  const double cn = first ? 0.0 : *cnp;
  for (int k = 0; k < 3; k++) {
    const long long q = 3 * i + k;
    const double bi = dr_bint(d, g, q);
    const double b = bi + g.bext[q];
    double vh;
    if (first) {
      vh = 0.5 * dt * b / L;
    } else {
      const double a = b / L;
      vh = ((2.0 - cn * dt) * vho[q] + 2.0 * dt * a) / (2.0 + cn * dt);
    }
    g.vh[q] = vh;
    g.v[q] = 0.5 * (vho[q] + vh);
    vho[q] = vh;
    bo[q] = bi;
  }
}

static int dr_grid(long long n, int t) {
  long long b = (n + t - 1) / t;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace pd

using namespace pd;

extern "C" pd_status pd_dr_init(pd_handle* h, double dt, double damping_factor) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (!(dt > 0)) return pd_fail(PD_ERR_ARG, "`stepsize` should be larger than zero!");
  if (!(damping_factor > 0)) return pd_fail(PD_ERR_ARG, "`damping_factor` should be larger than zero!");
  PD_CUDA(cudaSetDevice(h->device));
  if (!h->dr) {
    DRState* S = new DRState();
    h->dr = S;
    PD_TRY(dalloc(h, &S->lam, h->n));
    PD_TRY(dalloc(h, &S->vho, 3 * h->n));
    PD_TRY(dalloc(h, &S->bo, 3 * h->n));
    PD_TRY(dalloc(h, &S->part, 4 * DR_NB));
    PD_TRY(dalloc(h, &S->cn, 1));
  }
  DRState* S = h->dr;
  S->dt = dt;
  S->factor = damping_factor;
  PD_CUDA(cudaMemsetAsync(S->vho, 0, sizeof(double) * 3 * h->n, h->stream));
  PD_CUDA(cudaMemsetAsync(S->bo, 0, sizeof(double) * 3 * h->n, h->stream));
  k_dr_lam<<<dr_grid(h->n, 256), 256, 0, h->stream>>>(h->d, damping_factor, dt, S->lam);
  h->launches++;
  PD_CUDA(cudaGetLastError());
  PD_CUDA(cudaStreamSynchronize(h->stream));
  return PD_OK;
}

extern "C" pd_status pd_dr_density_matrix(pd_handle* h, double* out) {
  if (!h || !out) return pd_fail(PD_ERR_ARG, "NULL argument");
  if (!h->dr) return pd_fail(PD_ERR_ARG, "dynamic relaxation not initialised (pd_dr_init)");
  PD_CUDA(cudaSetDevice(h->device));
  // ordered after pd_dr_init's kernels on the handle's (non-blocking) stream
  PD_CUDA(cudaMemcpyAsync(out, h->dr->lam, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
  PD_CUDA(cudaStreamSynchronize(h->stream));
  return PD_OK;
}

// The kernels of steps first_step .. first_step + n_steps - 1 on the handle's stream. With ev
// (3 n_steps + 1 events) it records the start of every step, of its force phase and of its
// damping / update kernels, and the end of the last step.
static void dr_issue(pd_handle* h, long long first_step, long long n_steps, cudaEvent_t* ev) {
  DRState* S = h->dr;
  const double dt = S->dt;
  const int pg = dr_grid(h->n, 256);
  for (long long k = 0; k < n_steps; k++) {
    const long long step = first_step + k;
    if (ev) cudaEventRecord(ev[3 * k], h->stream);
    launch_kick_drift(h->d, h->g, h->bc, 2, dt, (int)k, h->stream);
    h->launches++;
    if (ev) cudaEventRecord(ev[3 * k + 1], h->stream);
    pd_launch_force(h, (int)k, 0);
    if (ev) cudaEventRecord(ev[3 * k + 2], h->stream);
    if (step > 1) {
      if (h->cfg.exact) {
        k_dr_damping_serial<<<1, 1, 0, h->stream>>>(h->d, h->g, S->lam, S->vho, S->bo, dt, S->cn);
        h->launches++;
      } else {
        k_dr_damping_part<<<DR_NB, DR_TPB, 0, h->stream>>>(h->d, h->g, S->lam, S->vho, S->bo, dt, S->part);
        k_dr_damping_finish<<<1, DR_TPB, 0, h->stream>>>(h->d, S->part, DR_NB, S->cn);
        h->launches += 2;
      }
    }
    k_dr_update<<<pg, 256, 0, h->stream>>>(h->d, h->g, S->lam, S->vho, S->bo, S->cn, dt, step == 1);
    h->launches++;
  }
  if (ev) cudaEventRecord(ev[3 * n_steps], h->stream);
}

static pd_status dr_begin(pd_handle* h, int64_t first_step, int64_t n_steps) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (!h->dr) return pd_fail(PD_ERR_ARG, "dynamic relaxation not initialised (pd_dr_init)");
  if (first_step < 1 || n_steps < 0 || n_steps > (1LL << 30))
    return pd_fail(PD_ERR_ARG, "invalid step range");
  PD_CUDA(cudaSetDevice(h->device));
  PD_TRY(pd_clear_error(h));
  const long long base = first_step;
  return pd_set_ctrl(h, offsetof(Ctrl, base), &base, sizeof(long long));
}

extern "C" pd_status pd_run_dr(pd_handle* h, int64_t first_step, int64_t n_steps) {
  PD_TRY(dr_begin(h, first_step, n_steps));
  dr_issue(h, first_step, n_steps, nullptr);
  PD_CUDA(cudaGetLastError());
  h->damage_valid = true;
  return pd_check_err(h);
}

extern "C" pd_status pd_run_dr_timed(pd_handle* h, int64_t first_step, int64_t n_steps,
                                     double* ms_total, double* ms_drift, double* ms_force,
                                     double* ms_relax) {
  if (!ms_total || !ms_drift || !ms_force || !ms_relax) return pd_fail(PD_ERR_ARG, "NULL argument");
  if (n_steps > (1 << 20)) return pd_fail(PD_ERR_ARG, "at most 2^20 timed steps");
  PD_TRY(dr_begin(h, first_step, n_steps));
  std::vector<cudaEvent_t> ev(3 * n_steps + 1);
  for (auto& e : ev) PD_CUDA(cudaEventCreate(&e));
  dr_issue(h, first_step, n_steps, ev.data());
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaEventSynchronize(ev.back());
  double td = 0, tf = 0, tr = 0;
  float x = 0;
  if (err == cudaSuccess) {
    for (long long k = 0; k < n_steps; k++) {
      cudaEventElapsedTime(&x, ev[3 * k], ev[3 * k + 1]); td += x;
      cudaEventElapsedTime(&x, ev[3 * k + 1], ev[3 * k + 2]); tf += x;
      cudaEventElapsedTime(&x, ev[3 * k + 2], ev[3 * k + 3]); tr += x;
    }
    cudaEventElapsedTime(&x, ev[0], ev.back());
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (err != cudaSuccess) return pd_fail(PD_ERR_CUDA, cudaGetErrorString(err));
  *ms_total = x;
  *ms_drift = td;
  *ms_force = tf;
  *ms_relax = tr;
  h->damage_valid = true;
  return pd_check_err(h);
}
