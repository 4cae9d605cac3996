// pd_static.cu -- an ordinary state-based force evaluation that allocates no device memory.
//
// Some callers cannot allocate GPU memory at the moment they need forces: a Julia host that
// manages every device buffer through its own memory pool and forbids the library to call
// cudaMalloc (the reference asserts that its force loop allocates nothing, test/perf/perf.jl),
// a time loop that must not stall on the allocator, or an application that hands the library
// memory it carved out of a fixed arena. For them pd_osb_force_static takes every input and
// output as a device pointer owned by the caller and keeps its one piece of scratch state --
// the weighted volume, dilatation and the two force coefficients of every point, which the
// gather phase reads for the neighbours -- in the file-scope device array below. The array
// is part of the library image: every GPU that loads the library holds it until the process
// exits, which is why it is kept to PD_STATIC_MAX_POINTS points (8 MiB).
//
// The arithmetic is the FP64 serial-order evaluation of pd_force64.cu (one thread per point,
// the reference's order of operations and of the scattered terms), on the reference's CSR
// bond arrays instead of the sliced layout.
#include <cuda.h>

#include <mutex>
#include <string>
#include <vector>

#include "pdcuda.h"
#include "pd_common.cuh"

namespace pd {

constexpr long long PD_STATIC_MAX_POINTS = 1LL << 18;

// {c1, c2, wvol, dil} per point, shared by every call of pd_osb_force_static on this device
static __device__ __align__(256) double4 g_osb_state[PD_STATIC_MAX_POINTS];

struct StaticArgs {
  long long n;
  const double* X;    // [3n] reference positions
  const double* x;    // [3n] current positions
  const double* vol;  // [n]
  const long long* off;
  const int* nbr;
  const double* L;
  const unsigned char* fail_permit;
  unsigned char* bond_active;  // in / out
  double delta, G, K, epsc;
  int kernel;
  double* b_int;      // [3n] out
  long long* n_active; // [n] out
  double4* state;     // g_osb_state, through the address looked up on the host
};

__device__ __forceinline__ double s_omega(int kernel, double delta, double L) {
  if (kernel == KER_LINEAR) return delta / L;
  if (kernel == KER_CONST_ONE) return 1.0;
  const double xi = L / delta;
  if (0 < xi && xi <= 0.5) return 2.0 / 3.0 - 4 * (xi * xi) + 4 * (xi * xi * xi);
  if (0.5 < xi && xi <= 1) return 4.0 / 3.0 - 4 * xi + 4 * (xi * xi) - 4.0 / 3.0 * (xi * xi * xi);
  return 0.0;
}

__device__ __forceinline__ double s_len(const double* p, long long i, long long j, double* d) {
  d[0] = p[3 * j] - p[3 * i];
  d[1] = p[3 * j + 1] - p[3 * i + 1];
  d[2] = p[3 * j + 2] - p[3 * i + 2];
  return sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
}

// calc_failure! (ordinary_state_based.jl:107-126), calc_weighted_volume (:176-189),
// calc_dilatation (:191-204), c1 and c2 (:135-136)
__global__ void k_static_osb_a(StaticArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  long long na = 0;
  double wvol = 0.0;
  for (long long b = a.off[i]; b < a.off[i + 1]; b++) {
    const long long j = a.nbr[b];
    double d[3], D[3];
    const double l = s_len(a.x, i, j, d);
    const double eps = (l - a.L[b]) / a.L[b];
    if (eps > a.epsc && a.fail_permit[b]) a.bond_active[b] = 0;
    na += a.bond_active[b];
    s_len(a.X, i, j, D);
    const double om = a.bond_active[b] ? s_omega(a.kernel, a.delta, a.L[b]) : 0.0;
    wvol += om * 1.0 * ((D[0] * D[0] + D[1] * D[1]) + D[2] * D[2]) * a.vol[j];
  }
  double dil = 0.0, c1 = 0.0, c2 = 0.0;
  if (wvol != 0.0) {
    const double c1d = 3.0 / wvol;
    for (long long b = a.off[i]; b < a.off[i + 1]; b++) {
      const long long j = a.nbr[b];
      double d[3];
      const double l = s_len(a.x, i, j, d);
      const double om = a.bond_active[b] ? s_omega(a.kernel, a.delta, a.L[b]) : 0.0;
      dil += om * 1.0 * c1d * a.L[b] * (l - a.L[b]) * a.vol[j];
    }
    c1 = 15.0 * a.G / wvol;
    c2 = dil * (3.0 * a.K / wvol - c1 / 3.0);
  }
  a.state[i] = make_double4(c1, c2, wvol, dil);
  a.n_active[i] = na;
}

// position of point i in the sorted bond list of point j (the reverse bond j -> i), or -1
__device__ __forceinline__ long long s_reverse(const StaticArgs& a, long long j, long long i) {
  long long lo = a.off[j], hi = a.off[j + 1];
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (a.nbr[mid] < i) lo = mid + 1; else hi = mid;
  }
  return (lo < a.off[j + 1] && a.nbr[lo] == i) ? lo : -1;
}

// force_density_point! (ordinary_state_based.jl:128-149) gathered in the serial order of the
// scattered terms: neighbours j < i, the own bonds, neighbours j > i (sorted bond lists). The
// term of neighbour j is the one its own loop scatters (b_j's bond j -> i: its bond state and
// its length), so bond states need not be the same in both directions.
__global__ void k_static_osb_b(StaticArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 ci = a.state[i];
  double bx = 0.0, by = 0.0, bz = 0.0;
  const long long b0 = a.off[i], b1 = a.off[i + 1];
  auto nbr_term = [&](long long b) {
    const long long j = a.nbr[b];
    const double4 cj = a.state[j];
    if (cj.z == 0.0) return;
    const long long r = s_reverse(a, j, i);
    if (r < 0) return;  // j has no bond to i: nothing is scattered into i
    double d[3];
    const double l = s_len(a.x, j, i, d);
    const double Lr = a.L[r];
    const double om = a.bond_active[r] ? s_omega(a.kernel, a.delta, Lr) : 0.0;
    const double s = om * 1.0 * (cj.y * Lr + cj.x * (l - Lr)) / l;
    bx += -(s * d[0]) * a.vol[j];
    by += -(s * d[1]) * a.vol[j];
    bz += -(s * d[2]) * a.vol[j];
  };
  long long split = b0;
  while (split < b1 && a.nbr[split] < i) split++;
  for (long long b = b0; b < split; b++) nbr_term(b);
  if (ci.z != 0.0)
    for (long long b = b0; b < b1; b++) {
      const long long j = a.nbr[b];
      double d[3];
      const double l = s_len(a.x, i, j, d);
      const double om = a.bond_active[b] ? s_omega(a.kernel, a.delta, a.L[b]) : 0.0;
      const double s = om * 1.0 * (ci.y * a.L[b] + ci.x * (l - a.L[b])) / l;
      bx += s * d[0] * a.vol[j];
      by += s * d[1] * a.vol[j];
      bz += s * d[2] * a.vol[j];
    }
  for (long long b = split; b < b1; b++) nbr_term(b);
  a.b_int[3 * i] = bx;
  a.b_int[3 * i + 1] = by;
  a.b_int[3 * i + 2] = bz;
}

}  // namespace pd

using namespace pd;

static thread_local std::string g_static_err;

// Device address of g_osb_state in each CUDA context that called, looked up once per context
// with it current. The context is read through the driver's cuCtxGetCurrent (taken from the
// runtime's driver entry points, so the library needs no link to libcuda); where that is not
// available the key is the device's primary context, identified by the device index.
struct StaticSlot {
  CUcontext ctx;
  int dev;
  void* ptr;
};
static std::mutex g_static_mutex;
static std::vector<StaticSlot> g_static_slots;
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

static CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrentFn)p;
  }
  return fn;
}

extern "C" const char* pd_static_last_error(void) { return g_static_err.c_str(); }

extern "C" pd_status pd_osb_force_static(int64_t n, const double* ref_position, const double* position,
                                         const double* volume, const int64_t* bond_offsets,
                                         const int32_t* neighbors, const double* bond_length,
                                         const uint8_t* fail_permit, uint8_t* bond_active,
                                         const pd_point_params* params, int32_t kernel,
                                         double* b_int, int64_t* n_active, void* stream) {
  if (n < 0 || !params) { g_static_err = "n < 0 or params is NULL"; return PD_ERR_ARG; }
  if (n > PD_STATIC_MAX_POINTS) {
    g_static_err = "pd_osb_force_static handles at most " + std::to_string(PD_STATIC_MAX_POINTS) +
                   " points (the size of its static scratch array); got " + std::to_string(n);
    return PD_ERR_ARG;
  }
  if (kernel < PD_KERNEL_CONST_ONE || kernel > PD_KERNEL_CUBIC_BSPLINE) {
    g_static_err = "unknown kernel";
    return PD_ERR_ARG;
  }
  if (n == 0) return PD_OK;
  if (!ref_position || !position || !volume || !bond_offsets || !neighbors || !bond_length ||
      !fail_permit || !bond_active || !b_int || !n_active) {
    g_static_err = "every array must be a device pointer";
    return PD_ERR_ARG;
  }
  // an error left by earlier CUDA work of this thread would be reported as this call's after
  // the launches: report it now, launch nothing, and leave it pending for its owner
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    g_static_err = std::string("a CUDA error from before this call is pending (") +
                   cudaGetErrorString(e) + "); no kernel was launched";
    return PD_ERR_CUDA;
  }
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_static_err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return PD_ERR_CUDA;
  }
  CUcontext ctx = nullptr;
  if (CtxGetCurrentFn get = ctx_get_current()) {
    if (get(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  }
  void* state = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_static_mutex);
    for (const StaticSlot& sl : g_static_slots)
      if (sl.dev == dev && sl.ctx == ctx) { state = sl.ptr; break; }
    if (!state) {
      // set-up in this context (the current one): the host-side name of the array is not a
      // device address, so its device address is looked up once
      e = cudaGetSymbolAddress(&state, g_osb_state);
      if (e != cudaSuccess) {
        g_static_err = std::string("cudaGetSymbolAddress of the scratch array on device ") +
                       std::to_string(dev) + ": " + cudaGetErrorString(e);
        return PD_ERR_CUDA;
      }
      if (ctx == nullptr && ctx_get_current() != nullptr) {
        // cudaGetSymbolAddress made the primary context current
        CUcontext now = nullptr;
        if (ctx_get_current()(&now) == CUDA_SUCCESS) ctx = now;
      }
      g_static_slots.push_back({ctx, dev, state});
    }
  }
  StaticArgs a;
  a.n = n;
  a.X = ref_position;
  a.x = position;
  a.vol = volume;
  a.off = reinterpret_cast<const long long*>(bond_offsets);
  a.nbr = neighbors;
  a.L = bond_length;
  a.fail_permit = fail_permit;
  a.bond_active = bond_active;
  a.delta = params->delta;
  a.G = params->G;
  a.K = params->K;
  a.epsc = params->epsilon_c;
  a.kernel = kernel;
  a.b_int = b_int;
  a.n_active = reinterpret_cast<long long*>(n_active);
  a.state = (double4*)state;
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = (int)((n + 127) / 128);
  k_static_osb_a<<<blocks, 128, 0, s>>>(a);
  k_static_osb_b<<<blocks, 128, 0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_static_err = std::string("kernel launch: ") + cudaGetErrorString(e);
    return PD_ERR_CUDA;
  }
  return PD_OK;
}
