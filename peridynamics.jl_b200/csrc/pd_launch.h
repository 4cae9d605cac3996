// pd_launch.h -- host-side launchers exported by each kernel translation unit of libpdcuda.
#pragma once
#include <cuda_runtime.h>
#include "pd_common.cuh"

// Upper bound of a force kernel's grid in blocks per SM (148 SMs; 0: no bound, one warp per
// slice). Every warp loops over slices with the grid's stride, so a bounded grid gives each warp
// several slices. Measured on the 8M-point OSB block (packed kernels, blocks of 128 threads, one
// B200): bound 64 (9,472 blocks): step 8.76 ms, phase A 4.15 ms, phase B 4.46 ms; no bound
// (62,500 blocks): 8.18 ms, 3.92 ms, 4.12 ms at a lower SM clock; bounds 32, 16 and 8: 8.81,
// 9.15 and 10.26 ms (phase B 4.51, 5.04 and 6.26 ms).
#ifndef PD_GRID_BLOCKS_PER_SM
#define PD_GRID_BLOCKS_PER_SM 0
#endif

namespace pd {

struct LaunchCfg {
  int group;  // lanes per point: 1, 2, 4, 8, 16, 32
  int block;  // threads per block
  bool exact; // FP64: one lane per point in the reference's serial summation order
  int pipe;   // FP32: 0 = plain loads, 1-3 = TMA-staged bond stream (pd_force32_tma.cu),
              // 4 = two rows of neighbour gathers in flight (BB, OSB), 5 = OSB / CMat with
              // packed x/y pairs and the next row pair's stream in flight (one lane per point)
  int fullk;  // FP32 OSB / CMat: sum the weighted volumes / shape tensors in full (else
              // update the stored ones)
};

// boundary conditions as the integration kernels see them
struct BCInfo {
  int field;  // 0 velocity_half, 1 b_ext
  int dim;
  int kind;   // 0 time table, 1 per point per step, 2 constant data
  int col;    // column in the per-step table (kinds 0, 1) or offset into the data (kind 2)
};
struct BCEntry {
  int bc;     // index into BCInfo
  int q;      // position of the point in the condition's point list
};
struct BCDev {
  int n_points;          // points that carry conditions
  const int* point;      // [n_points]
  const int* slot;       // [n]: position of the point in point[] (read for flagged points only)
  const int* entry_off;  // [n_points + 1]
  const BCEntry* entry;
  const BCInfo* info;
  const double* table;   // [table_n][per_step]
  long long per_step;
  const double* data;
};

// integration state (FP64 in both precision modes)
struct IntDev {
  double* u;    // FP64 path displacement [3n] (FP32 path: displacement lives in cur)
  double* vh;
  double* v;
  double* a;
  double* bext;
  int fp32;     // 1: FP32 force output b32, displacement in cur
};

// force evaluation; phase 0 = all kernels, 1 = the first (BB: the only) kernel, 2 = the
// second kernel of the state-based materials. Returns the number of kernels launched.
int launch_force64(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s);
int launch_force32(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s);
bool tma_supported(const DevBody& d);
int launch_force32_tma(const DevBody& d, int pipe, int kstep, int phase, cudaStream_t s);
// packed-pair OSB kernels (pipe 5, pd_force32_pk.cu): phase 1 = A, 2 = B, 0 = both
bool pk_supported(const DevBody& d, int phase);
// the packed kernels of OSB (pd_force32_pk.cu) or CMat (pd_force32.cu) apply to this phase
bool packed_supported(const DevBody& d, int phase);
int launch_force32_pk(const DevBody& d, const LaunchCfg& c, int kstep, int phase, cudaStream_t s);
void launch_cauchy64(const DevBody& d, const double* F, int from_h32, double* out, cudaStream_t s);

// integration with the boundary conditions, one launch per step: mode 0 = kick from the stored
// (v, a), mode 1 = kick from the last force, mode 2 = no kick (dynamic relaxation: drift with
// the stored v_half)
void launch_kick_drift(const DevBody& d, const IntDev& g, const BCDev& bc, int mode,
                       double dt_override, int kstep, cudaStream_t s);
void launch_finish(const DevBody& d, const IntDev& g, double dt_override, cudaStream_t s);
void launch_split_u(const DevBody& d, cudaStream_t s);
// the split of rows[0 .. n) (halo rows that received a displacement)
void launch_split_u_rows(const DevBody& d, const int* rows, long long n, cudaStream_t s);

// sliced bond layout and bond-array helpers (pd_layout.cu)
cudaError_t build_slices(long long n, const long long* off, int G, long long** soff_out,
                         long long* nslices_out, long long* nslots_out, cudaStream_t s);
void launch_scatter_i32(const DevBody& d, const int* src, int* dst, cudaStream_t s);
void launch_relayout_i32(const DevBody& a, const DevBody& b, const int* src, int* dst, cudaStream_t s);
void launch_relayout_f64(const DevBody& a, const DevBody& b, const double* src, double* dst, cudaStream_t s);
void launch_relayout_f4(const DevBody& a, const DevBody& b, const float4* src, float4* dst, cudaStream_t s);
void launch_build_len64(const DevBody& d, const int* nbr_csr, const double* L, const unsigned char* fp,
                        double* out, cudaStream_t s);
void launch_build_geo(const DevBody& d, const int* nbr_csr, const double* L, const unsigned char* fp,
                      float4* out, cudaStream_t s);
void launch_pack_bits(const DevBody& d, const unsigned char* bytes, cudaStream_t s);
void launch_export_bond_active(const DevBody& d, unsigned char* out, int raw, cudaStream_t s);
void launch_count_active(const DevBody& d, cudaStream_t s);
void launch_reverse(long long n, const long long* off, const int* nbr, int* revk, int* flags, cudaStream_t s);
void launch_check_sym(const DevBody& d, int* flags, cudaStream_t s);
void launch_export_damage(const DevBody& d, int valid, double* out, cudaStream_t s);
void launch_export_position(const DevBody& d, const IntDev& g, double* out, int what, cudaStream_t s);
void launch_timestep(const DevBody& d, double* dt_point, cudaStream_t s);
void launch_break_sets(const DevBody& d, const unsigned char* A, const unsigned char* B, cudaStream_t s);
void launch_near_critical(const DevBody& d, const IntDev& g, double tol, unsigned long long* count,
                          cudaStream_t s);
void launch_break_random(const DevBody& d, double fraction, unsigned long long seed,
                         const long long* gid, cudaStream_t s);

}  // namespace pd
