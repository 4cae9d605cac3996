// pd_layout.cu -- the sliced bond layout of libpdcuda and the kernels that read or write
// bond arrays outside the force evaluation (setup, state upload, exports, CFL step).
//
// The reference keeps bonds in CSR order (bond_ids ranges, bond_system.jl:167-176); the
// device keeps that order inside every point (bond k of point i is the reference's bond
// off[i] + k) but stores bond k of the points of a slice next to each other (see
// pd_common.cuh). The host API converts between the two with the kernels below.
#include <cub/cub.cuh>

#include "pd_common.cuh"
#include "pd_launch.h"

namespace pd {

static inline int blocks_for(long long n, int t) {
  long long b = (n + t - 1) / t;
  return (int)(b < 1 ? 1 : b);
}

// rows of 32 slots that slice s needs: ceil(max bond count of its points / G), times 32
__global__ void k_slice_slots(long long n, const long long* off, int G, long long nslices,
                              long long* slots) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  const int P = 32 / G;
  long long m = 0;
  for (int p = 0; p < P; p++) {
    const long long i = s * P + p;
    if (i < n) m = max(m, off[i + 1] - off[i]);
  }
  slots[s] = ((m + G - 1) / G) * 32;
}

__global__ void k_set_total(long long* soff, long long nslices, const long long* slots) {
  soff[nslices] = soff[nslices - 1] + slots[nslices - 1];
}

cudaError_t build_slices(long long n, const long long* off, int G, long long** soff_out,
                         long long* nslices_out, long long* nslots_out, cudaStream_t s) {
  const long long P = 32 / G;
  const long long ns = n > 0 ? (n + P - 1) / P : 1;
  long long *slots = nullptr, *soff = nullptr;
  void* tmp = nullptr;
  size_t need = 0;
  cudaError_t e = cudaMalloc(&slots, sizeof(long long) * ns);
  if (e == cudaSuccess) e = cudaMalloc(&soff, sizeof(long long) * (ns + 1));
  if (e == cudaSuccess && n == 0) {
    e = cudaMemsetAsync(soff, 0, sizeof(long long) * (ns + 1), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(slots);
    if (e != cudaSuccess) { cudaFree(soff); return e; }
    *soff_out = soff; *nslices_out = 0; *nslots_out = 0;
    return cudaSuccess;
  }
  if (e == cudaSuccess) {
    k_slice_slots<<<blocks_for(ns, 256), 256, 0, s>>>(n, off, G, ns, slots);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, need, slots, soff, (int)ns, s);
  if (e == cudaSuccess) e = cudaMalloc(&tmp, need > 0 ? need : 1);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, need, slots, soff, (int)ns, s);
  if (e == cudaSuccess) { k_set_total<<<1, 1, 0, s>>>(soff, ns, slots); e = cudaGetLastError(); }
  long long total = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, soff + ns, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(slots);
  cudaFree(tmp);
  if (e != cudaSuccess) { cudaFree(soff); return e; }
  *soff_out = soff;
  *nslices_out = ns;
  *nslots_out = total;
  return cudaSuccess;
}

// CSR -> slots for 4-byte values (neighbour indices, reverse positions)
__global__ void k_scatter_i32(DevBody d, const int* src, int* dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  for (int k = 0; k < cnt; k++) dst[bond_slot(d, i, k)] = src[d.off[i] + k];
}

void launch_scatter_i32(const DevBody& d, const int* src, int* dst, cudaStream_t s) {
  k_scatter_i32<<<blocks_for(d.n, 256), 256, 0, s>>>(d, src, dst);
}

// layout (a) -> layout (b) of one bond array
template <class T>
__global__ void k_relayout(DevBody a, DevBody b, const T* src, T* dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int cnt = (int)(a.off[i + 1] - a.off[i]);
  for (int k = 0; k < cnt; k++) dst[bond_slot(b, i, k)] = src[bond_slot(a, i, k)];
}

void launch_relayout_i32(const DevBody& a, const DevBody& b, const int* src, int* dst, cudaStream_t s) {
  k_relayout<int><<<blocks_for(a.n, 256), 256, 0, s>>>(a, b, src, dst);
}
void launch_relayout_f64(const DevBody& a, const DevBody& b, const double* src, double* dst, cudaStream_t s) {
  k_relayout<double><<<blocks_for(a.n, 256), 256, 0, s>>>(a, b, src, dst);
}
void launch_relayout_f4(const DevBody& a, const DevBody& b, const float4* src, float4* dst, cudaStream_t s) {
  k_relayout<float4><<<blocks_for(a.n, 256), 256, 0, s>>>(a, b, src, dst);
}

// bond geometry of the FP64 path: L with the sign carrying fail_permit (negative = no failure)
__global__ void k_build_len64(DevBody d, const int* nbr_csr, const double* L, const unsigned char* fp,
                              double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 Xi = d.X0[i];
  const long long o = d.off[i];
  const int cnt = (int)(d.off[i + 1] - o);
  for (int k = 0; k < cnt; k++) {
    double Lb;
    if (L) {
      Lb = L[o + k];
    } else {
      const double4 Xj = d.X0[nbr_csr[o + k]];
      const double dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
      Lb = sqrt((dx * dx + dy * dy) + dz * dz);
    }
    out[bond_slot(d, i, k)] = (fp == nullptr || fp[o + k]) ? Lb : -Lb;
  }
}

// bond geometry of the FP32 path: {xi = X_j - X_i, +-L}
__global__ void k_build_geo(DevBody d, const int* nbr_csr, const double* L, const unsigned char* fp,
                            float4* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 Xi = d.X0[i];
  const long long o = d.off[i];
  const int cnt = (int)(d.off[i + 1] - o);
  for (int k = 0; k < cnt; k++) {
    const double4 Xj = d.X0[nbr_csr[o + k]];
    const double gx = Xj.x - Xi.x, gy = Xj.y - Xi.y, gz = Xj.z - Xi.z;
    double Lb;
    if (L) {
      Lb = L[o + k];
    } else {
      const double dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
      Lb = sqrt((dx * dx + dy * dy) + dz * dz);
    }
    const float Lf = (float)Lb;
    out[bond_slot(d, i, k)] =
        make_float4((float)gx, (float)gy, (float)gz, (fp == nullptr || fp[o + k]) ? Lf : -Lf);
  }
}

void launch_build_len64(const DevBody& d, const int* nbr_csr, const double* L, const unsigned char* fp,
                        double* out, cudaStream_t s) {
  k_build_len64<<<blocks_for(d.n, 256), 256, 0, s>>>(d, nbr_csr, L, fp, out);
}

void launch_build_geo(const DevBody& d, const int* nbr_csr, const double* L, const unsigned char* fp,
                      float4* out, cudaStream_t s) {
  k_build_geo<<<blocks_for(d.n, 256), 256, 0, s>>>(d, nbr_csr, L, fp, out);
}

// bond_active bytes in the reference's order (or all active when bytes is null) -> bits;
// one warp per slice, one ballot per row
__global__ void k_pack_bits(DevBody d, const unsigned char* bytes) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= d.nslices) return;
  const int lane = threadIdx.x & 31, G = d.lg, P = 32 / G;
  const int sub = lane / G, gl = lane % G;
  const long long s = warp;
  const long long i = s * P + sub;
  const bool valid = i < d.n;
  const long long sbase = d.soff[s];
  const int rows = (int)((d.soff[s + 1] - sbase) >> 5);
  const int cnt = valid ? (int)(d.off[i + 1] - d.off[i]) : 0;
  for (int r = 0; r < rows; r++) {
    const int k = r * G + gl;
    const bool on = k < cnt && (bytes == nullptr || bytes[d.off[i] + k] != 0);
    const unsigned w = __ballot_sync(0xffffffffu, on);
    if (lane == 0) d.bits[(sbase >> 5) + r] = w;
  }
}

void launch_pack_bits(const DevBody& d, const unsigned char* bytes, cudaStream_t s) {
  if (d.nslices == 0) return;
  k_pack_bits<<<blocks_for(d.nslices * 32, 256), 256, 0, s>>>(d, bytes);
}

// bond_active of the reference: the stored bit, and no bond of a killed point
__global__ void k_export_bond_active(DevBody d, unsigned char* out, int raw) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const bool killed = !raw && (d.meta[i] & META_KILLED);
  const long long o = d.off[i];
  const int cnt = (int)(d.off[i + 1] - o);
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    out[o + k] = killed ? 0 : (unsigned char)((d.bits[b >> 5] >> (b & 31)) & 1u);
  }
}

void launch_export_bond_active(const DevBody& d, unsigned char* out, int raw, cudaStream_t s) {
  k_export_bond_active<<<blocks_for(d.n, 256), 256, 0, s>>>(d, out, raw);
}

__global__ void k_count_active(DevBody d) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  int na = 0;
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    na += (d.bits[b >> 5] >> (b & 31)) & 1u;
  }
  d.n_active[i] = (d.meta[i] & META_KILLED) ? 0 : na;
}

void launch_count_active(const DevBody& d, cudaStream_t s) {
  k_count_active<<<blocks_for(d.n, 256), 256, 0, s>>>(d);
}

// reverse bonds on the CSR lists: position k' of i in the list of j (binary search in the
// common sorted case, linear search otherwise); flags[0] = 1 if a bond has no reverse. One warp
// per point, its lanes taking consecutive bonds (coalesced reads of nbr, writes of revk).
__global__ void k_reverse(long long n, const long long* off, const int* nbr, int* revk, int* flags) {
  const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  for (long long b = off[i] + (threadIdx.x & 31); b < off[i + 1]; b += 32) {
    const int j = nbr[b];
    const long long lo = off[j], hi = off[j + 1];
    long long found = -1, a = lo, z = hi;
    while (a < z) {
      const long long mid = (a + z) / 2;
      if (nbr[mid] < i) a = mid + 1; else z = mid;
    }
    if (a < hi && nbr[a] == i) found = a;
    if (found < 0)
      for (long long c = lo; c < hi; c++)
        if (nbr[c] == i) { found = c; break; }
    revk[b] = found < 0 ? 0 : (int)(found - lo);
    if (found < 0) flags[0] = 1;
  }
}

void launch_reverse(long long n, const long long* off, const int* nbr, int* revk, int* flags, cudaStream_t s) {
  k_reverse<<<blocks_for(n * 32, 256), 256, 0, s>>>(n, off, nbr, revk, flags);
}

// flags[1] = 1 if a bond and its reverse differ in state; flags[2] = 1 if a fail-permitted
// bond joins points of different critical stretch
__global__ void k_check_sym(DevBody d, int* flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam& Pi = d.params[d.meta[i] & META_PID_MASK];
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    const int j = d.nbr[b];
    const long long r = bond_slot(d, j, d.rev[b]);
    const bool a = (d.bits[b >> 5] >> (b & 31)) & 1u;
    const bool c = (d.bits[r >> 5] >> (r & 31)) & 1u;
    if (a != c) flags[1] = 1;
    const DevParam& Pj = d.params[d.meta[j] & META_PID_MASK];
    const bool permitted = d.len64 ? (d.len64[b] > 0) : (d.geo[b].w > 0);
    if (permitted && (Pi.epsc != Pj.epsc || Pi.epscf != Pj.epscf)) flags[2] = 1;
  }
}

void launch_check_sym(const DevBody& d, int* flags, cudaStream_t s) {
  k_check_sym<<<blocks_for(d.n, 256), 256, 0, s>>>(d, flags);
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
  if (d.meta[i] & META_HALO) {  // its owner's partition gives the step of a halo row
    dtp[i] = INFINITY;
    return;
  }
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  double dtsum = 0.0;
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
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

// bonds that may fail and whose current stretch lies within tol of the owner's critical
// stretch (FP64 from the current state in both precisions): the failure decisions that the
// rounding of a summation order can flip
__global__ void k_near_critical(DevBody d, IntDev g, double tol, unsigned long long* count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam& P = d.params[d.meta[i] & META_PID_MASK];
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  const double4 Xi = d.X0[i], ci = d.cur[i];
  unsigned long long c = 0;
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    const int j = d.nbr[b];
    const double4 Xj = d.X0[j], cj = d.cur[j];
    double L, dx, dy, dz;
    bool permitted;
    if (d.len64) {
      L = fabs(d.len64[b]);
      permitted = d.len64[b] > 0;
      dx = cj.x - ci.x; dy = cj.y - ci.y; dz = cj.z - ci.z;
    } else {  // FP32 path: cur holds the displacement
      const double ex = Xi.x - Xj.x, ey = Xi.y - Xj.y, ez = Xi.z - Xj.z;
      L = sqrt((ex * ex + ey * ey) + ez * ez);
      permitted = d.geo[b].w > 0;
      dx = (Xj.x + cj.x) - (Xi.x + ci.x);
      dy = (Xj.y + cj.y) - (Xi.y + ci.y);
      dz = (Xj.z + cj.z) - (Xi.z + ci.z);
    }
    const double l = sqrt((dx * dx + dy * dy) + dz * dz);
    if (permitted && fabs((l - L) / L - P.epsc) <= tol) c++;
  }
  (void)g;
  if (c) atomicAdd(count, c);
}

void launch_near_critical(const DevBody& d, const IntDev& g, double tol, unsigned long long* count,
                          cudaStream_t s) {
  k_near_critical<<<blocks_for(d.n, 256), 256, 0, s>>>(d, g, tol, count);
}

// break_bonds! (bond_system.jl:249-267): bonds between a point of set a and a point of set b
// become inactive
__global__ void k_break_sets(DevBody d, const unsigned char* A, const unsigned char* B) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
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

// gid (may be null): the point numbers the pair hash uses (a partition passes the body's)
__global__ void k_break_random(DevBody d, unsigned long long threshold, unsigned long long seed,
                               const long long* gid) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  const unsigned long long gi = gid ? (unsigned long long)gid[i] : (unsigned long long)i;
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    const int jl = d.nbr[b];
    const unsigned long long j = gid ? (unsigned long long)gid[jl] : (unsigned long long)jl;
    const unsigned long long lo = j < gi ? j : gi;
    const unsigned long long hi = j < gi ? gi : j;
    const unsigned long long r = mix64(mix64(lo * 0x9e3779b97f4a7c15ull + seed) ^ hi);
    if (r < threshold) atomicAnd(d.bits + (b >> 5), ~(1u << (b & 31)));
  }
}

void launch_break_random(const DevBody& d, double fraction, unsigned long long seed,
                         const long long* gid, cudaStream_t s) {
  const long double t = (long double)fraction * 18446744073709551616.0L;
  const unsigned long long thr = fraction >= 1.0 ? ~0ull : (unsigned long long)t;
  k_break_random<<<blocks_for(d.n, 256), 256, 0, s>>>(d, thr, seed, gid);
}

}  // namespace pd
