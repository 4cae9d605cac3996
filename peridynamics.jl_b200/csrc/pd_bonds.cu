// pd_bonds.cu -- device neighbour search of libpdcuda (replaces find_bonds / find_bonds! /
// filter_bonds!, src/discretization/bond_system.jl:96-165, which the reference runs on the
// CPU through PointNeighbors' grid search).
//
// Cell list with cells of edge delta_max: points are sorted by cell (CUB radix sort, stable,
// so points keep ascending index inside a cell), every point counts and then writes its
// neighbours j != i with |X_i - X_j|^2 <= delta_i^2 (the squared distance summed
// (dx^2 + dy^2) + dz^2 without FMA, as the CPU), filter-mode pre-cracks drop the bonds
// between their two point sets, and every bond list is put in ascending j order (one warp per
// list for lists of up to 1024 bonds, CUB's segmented sort beyond).
#include <cub/cub.cuh>

#include <climits>

#include "pd_common.cuh"
#include "pd_bonds.h"

namespace pd {

struct Grid {
  double lo[3];
  double h;
  long long nc[3];
};

__device__ __forceinline__ long long cell_coord(double x, double lo, double h, long long nc) {
  long long c = (long long)floor((x - lo) / h);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_cell_id(long long n, const double* X, Grid g, unsigned long long* key, int* val) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long cx = cell_coord(X[3 * i], g.lo[0], g.h, g.nc[0]);
  const long long cy = cell_coord(X[3 * i + 1], g.lo[1], g.h, g.nc[1]);
  const long long cz = cell_coord(X[3 * i + 2], g.lo[2], g.h, g.nc[2]);
  key[i] = (unsigned long long)(cx + g.nc[0] * (cy + g.nc[1] * cz));
  val[i] = (int)i;
}

__global__ void k_cell_ranges(long long n, const unsigned long long* key, int* start, int* end) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const unsigned long long c = key[k];
  if (k == 0 || key[k - 1] != c) start[c] = (int)k;
  if (k == n - 1 || key[k + 1] != c) end[c] = (int)k + 1;
}

// pass 0: count (cnt[i]); pass 1: write into nbr[off[i]...]
template <int PASS>
__global__ void k_search(long long n, const double* X, const double* delta, const unsigned short* cmask,
                         const unsigned char* owned, Grid g, const int* start, const int* end, const int* sorted, long long* cnt,
                         const long long* off, int* nbr, int* flags) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
  const double di = delta[i];
  const double r2 = di * di;
  const unsigned short mi = cmask ? cmask[i] : 0;
  const bool own_i = owned ? owned[i] != 0 : true;
  const long long cx = cell_coord(xi, g.lo[0], g.h, g.nc[0]);
  const long long cy = cell_coord(yi, g.lo[1], g.h, g.nc[1]);
  const long long cz = cell_coord(zi, g.lo[2], g.h, g.nc[2]);
  long long r = (long long)ceil(di / g.h);
  if (r < 1) r = 1;
  long long c = 0;
  const long long o = PASS ? off[i] : 0;
  for (long long z = cz - r; z <= cz + r; z++) {
    if (z < 0 || z >= g.nc[2]) continue;
    for (long long y = cy - r; y <= cy + r; y++) {
      if (y < 0 || y >= g.nc[1]) continue;
      for (long long x = cx - r; x <= cx + r; x++) {
        if (x < 0 || x >= g.nc[0]) continue;
        const long long cell = x + g.nc[0] * (y + g.nc[1] * z);
        for (int k = start[cell]; k < end[cell]; k++) {
          const int j = sorted[k];
          if (j == i) continue;
          const double dx = xi - X[3 * (long long)j], dy = yi - X[3 * (long long)j + 1],
                       dz = zi - X[3 * (long long)j + 2];
          const double d2 = (dx * dx + dy * dy) + dz * dz;
          if (!(d2 <= r2)) continue;
          if (!own_i && !owned[j]) continue;
          if (cmask) {
            // crack k: point in set a -> bit 2k, in set b -> bit 2k+1
            const unsigned short mj = cmask[j];
            const unsigned short ai = mi & 0x5555, bi = (mi >> 1) & 0x5555;
            const unsigned short aj = mj & 0x5555, bj = (mj >> 1) & 0x5555;
            if ((ai & bj) || (bi & aj)) continue;
          }
          if (sqrt(d2) < 2.220446049250313e-16) flags[0] = 1;  // check_point_duplicates
          if (PASS) nbr[o + c] = j;
          c++;
        }
      }
    }
  }
  if (!PASS) cnt[i] = c;
}

__global__ void k_set_last(long long* off, long long n, const long long* cnt) {
  off[n] = off[n - 1] + cnt[n - 1];
}

// reference length L = sqrt(dot(X_i - X_j)) and fail_permit = fp_i & fp_j of every bond; one
// warp per point, its lanes taking consecutive bonds (coalesced reads of nbr, writes of L, fpb)
__global__ void k_bond_props(long long n, const double* X, const unsigned char* fp, const long long* off,
                             const int* nbr, double* L, unsigned char* fpb) {
  const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  for (long long b = off[i] + (threadIdx.x & 31); b < off[i + 1]; b += 32) {
    const long long j = nbr[b];
    const double dx = X[3 * i] - X[3 * j], dy = X[3 * i + 1] - X[3 * j + 1], dz = X[3 * i + 2] - X[3 * j + 2];
    L[b] = sqrt((dx * dx + dy * dy) + dz * dz);
    fpb[b] = (unsigned char)((fp ? fp[i] : 1) & (fp ? fp[j] : 1));
  }
}

// cnt_max[0] = max_i cnt[i] (one atomic per block)
__global__ void k_max_count(long long n, const long long* __restrict__ cnt, int* cnt_max) {
  __shared__ int red[8];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int c = i < n ? (int)cnt[i] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int m = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = max(m, red[w]);
    atomicMax(cnt_max, m);
  }
}

// ascending order of every point's bond list (in[off[i] .. off[i+1]) -> out, at most 32 E
// entries), one warp per list: a bitonic network over 32 E keys, E per lane at positions
// e * 32 + lane, padded with INT_MAX (no point index reaches it). The keys of a list are
// distinct, so the result is the unique ascending order.
template <int E>
__global__ void __launch_bounds__(256) k_sort_lists(long long n, const long long* __restrict__ off,
                                                    const int* __restrict__ in, int* __restrict__ out) {
  constexpr int N = 32 * E;
  const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // the whole warp
  const long long b = off[i];
  const int m = (int)(off[i + 1] - b);
  int v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = e * 32 + lane < m ? in[b + e * 32 + lane] : INT_MAX;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {  // partner in this lane: v[e ^ (j / 32)]
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int e2 = e ^ (j >> 5);
          if (e2 > e) {
            const bool asc = ((e * 32) & k) == 0;
            const int a = v[e], c = v[e2];
            if ((a > c) == asc) { v[e] = c; v[e2] = a; }
          }
        }
      } else {  // partner in lane ^ j, same e
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int o = __shfl_xor_sync(0xffffffffu, v[e], j);
          const bool asc = ((e * 32 + lane) & k) == 0, lower = (lane & j) == 0;
          v[e] = lower == asc ? min(v[e], o) : max(v[e], o);
        }
      }
    }
  }
#pragma unroll
  for (int e = 0; e < E; e++)
    if (e * 32 + lane < m) out[b + e * 32 + lane] = v[e];
}

static inline int nblk(long long n, int t) { return (int)((n + t - 1) / t < 1 ? 1 : (n + t - 1) / t); }

#define CK(x)                                        \
  do {                                               \
    cudaError_t e_ = (x);                            \
    if (e_ != cudaSuccess) { err = e_; goto done; }  \
  } while (0)

cudaError_t device_find_bonds_grid(long long n, const double* dX, const double* ddelta,
                                   const unsigned short* dmask, const unsigned char* downed,
                                   const double lo[3], double h,
                                   const long long nc[3], long long* d_off, int** d_nbr_out,
                                   long long* nb_out, int* dup_out, cudaStream_t s) {
  cudaError_t err = cudaSuccess;
  Grid g;
  unsigned long long *key = nullptr, *key2 = nullptr;
  int *val = nullptr, *val2 = nullptr, *start = nullptr, *end = nullptr, *flags = nullptr;
  int *nbr = nullptr, *nbr2 = nullptr;
  long long* cnt = nullptr;
  void* tmp = nullptr;
  size_t tmpb = 0, need = 0;
  long long ncell = 1, nb = 0;
  int hflags[2] = {0, 0};
  *d_nbr_out = nullptr;
  *nb_out = 0;
  *dup_out = 0;
  g.h = h;
  for (int k = 0; k < 3; k++) { g.lo[k] = lo[k]; g.nc[k] = nc[k]; ncell *= nc[k]; }
  if (n == 0) {
    CK(cudaMemsetAsync(d_off, 0, sizeof(long long), s));
    CK(cudaStreamSynchronize(s));
    return cudaSuccess;
  }
  CK(cudaMalloc(&key, sizeof(unsigned long long) * n));
  CK(cudaMalloc(&key2, sizeof(unsigned long long) * n));
  CK(cudaMalloc(&val, sizeof(int) * n));
  CK(cudaMalloc(&val2, sizeof(int) * n));
  CK(cudaMalloc(&start, sizeof(int) * ncell));
  CK(cudaMalloc(&end, sizeof(int) * ncell));
  CK(cudaMalloc(&flags, sizeof(int) * 4));
  CK(cudaMalloc(&cnt, sizeof(long long) * n));
  CK(cudaMemsetAsync(start, 0, sizeof(int) * ncell, s));
  CK(cudaMemsetAsync(end, 0, sizeof(int) * ncell, s));
  CK(cudaMemsetAsync(flags, 0, sizeof(int) * 4, s));
  k_cell_id<<<nblk(n, 256), 256, 0, s>>>(n, dX, g, key, val);
  CK(cudaGetLastError());
  {
    int bits = 1;
    while (bits < 64 && (1ull << bits) < (unsigned long long)ncell) bits++;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, need, key, key2, val, val2, (int)n, 0, bits, s));
    if (need > tmpb) { cudaFree(tmp); tmp = nullptr; CK(cudaMalloc(&tmp, need)); tmpb = need; }
    CK(cub::DeviceRadixSort::SortPairs(tmp, need, key, key2, val, val2, (int)n, 0, bits, s));
  }
  k_cell_ranges<<<nblk(n, 256), 256, 0, s>>>(n, key2, start, end);
  CK(cudaGetLastError());
  k_search<0><<<nblk(n, 128), 128, 0, s>>>(n, dX, ddelta, dmask, downed, g, start, end, val2, cnt, nullptr,
                                           nullptr, flags);
  CK(cudaGetLastError());
  CK(cub::DeviceScan::ExclusiveSum(nullptr, need, cnt, d_off, (int)n, s));
  if (need > tmpb) { cudaFree(tmp); tmp = nullptr; CK(cudaMalloc(&tmp, need)); tmpb = need; }
  CK(cub::DeviceScan::ExclusiveSum(tmp, need, cnt, d_off, (int)n, s));
  k_set_last<<<1, 1, 0, s>>>(d_off, n, cnt);
  CK(cudaMemcpyAsync(&nb, d_off + n, sizeof(long long), cudaMemcpyDeviceToHost, s));
  k_max_count<<<nblk(n, 256), 256, 0, s>>>(n, cnt, flags + 1);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(hflags, flags, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hflags[0]) { *dup_out = 1; goto done; }
  if (nb > 0x7fffffffLL) { err = cudaErrorInvalidValue; goto done; }
  CK(cudaMalloc(&nbr, sizeof(int) * (nb > 0 ? nb : 1)));
  CK(cudaMalloc(&nbr2, sizeof(int) * (nb > 0 ? nb : 1)));
  k_search<1><<<nblk(n, 128), 128, 0, s>>>(n, dX, ddelta, dmask, downed, g, start, end, val2, nullptr, d_off,
                                           nbr, flags);
  CK(cudaGetLastError());
  if (nb > 0 && hflags[1] <= 1024) {
    // lists of up to 1024 bonds: one warp per list (the library's segmented sort took 0.53 s
    // for the 956.5M bonds of an 8M-point block)
    const int mc = hflags[1], grid = nblk(n * 32, 256);
    if (mc <= 32) k_sort_lists<1><<<grid, 256, 0, s>>>(n, d_off, nbr, nbr2);
    else if (mc <= 64) k_sort_lists<2><<<grid, 256, 0, s>>>(n, d_off, nbr, nbr2);
    else if (mc <= 128) k_sort_lists<4><<<grid, 256, 0, s>>>(n, d_off, nbr, nbr2);
    else if (mc <= 256) k_sort_lists<8><<<grid, 256, 0, s>>>(n, d_off, nbr, nbr2);
    else if (mc <= 512) k_sort_lists<16><<<grid, 256, 0, s>>>(n, d_off, nbr, nbr2);
    else k_sort_lists<32><<<grid, 256, 0, s>>>(n, d_off, nbr, nbr2);
    CK(cudaGetLastError());
  } else if (nb > 0) {
    CK(cub::DeviceSegmentedSort::SortKeys(nullptr, need, nbr, nbr2, (int)nb, (int)n, d_off, d_off + 1, s));
    if (need > tmpb) { cudaFree(tmp); tmp = nullptr; CK(cudaMalloc(&tmp, need)); tmpb = need; }
    CK(cub::DeviceSegmentedSort::SortKeys(tmp, need, nbr, nbr2, (int)nb, (int)n, d_off, d_off + 1, s));
  }
  CK(cudaStreamSynchronize(s));
  *d_nbr_out = nbr2;
  nbr2 = nullptr;
  *nb_out = nb;
done:
  cudaFree(key); cudaFree(key2); cudaFree(val); cudaFree(val2); cudaFree(start); cudaFree(end);
  cudaFree(flags); cudaFree(cnt); cudaFree(tmp); cudaFree(nbr); cudaFree(nbr2);
  return err;
}

void launch_bond_props(long long n, const double* dX, const unsigned char* dfp, const long long* doff,
                       const int* dnbr, double* dL, unsigned char* dfpb, cudaStream_t s) {
  k_bond_props<<<nblk(n * 32, 256), 256, 0, s>>>(n, dX, dfp, doff, dnbr, dL, dfpb);
}

}  // namespace pd
