// pd_handle.h -- the body handle of libpdcuda and the error helpers shared by the
// translation units that implement the C ABI (pd_api.cu, pd_nk.cu).
#pragma once
#include <algorithm>
#include <string>
#include <vector>

#include "pdcuda.h"
#include "pd_common.cuh"
#include "pd_launch.h"

namespace pd {
struct NKState;  // quasi-static Newton-Krylov solver state (pd_nk.cu)
void nk_release(pd_handle* h);
struct DRState;  // dynamic relaxation state (pd_dr.cu)
void dr_release(pd_handle* h);
}

// sets the thread's last error message and returns code
pd_status pd_fail(pd_status code, const std::string& msg);

#define PD_CUDA(x)                                                                            \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess)                                                                    \
      return pd_fail(e_ == cudaErrorMemoryAllocation ? PD_ERR_OOM : PD_ERR_CUDA,              \
                     std::string(#x) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

#define PD_TRY(x)                  \
  do {                             \
    pd_status s_ = (x);            \
    if (s_ != PD_OK) return s_;    \
  } while (0)

using pd::BCDev;
using pd::BCInfo;
using pd::DevBody;
using pd::DevParam;
using pd::IntDev;
using pd::LaunchCfg;

struct GraphKey {
  int steps = 0, group = 0, block = 0, exact = 0, bcpts = 0, pipe = 0;
  double dt = 0;
  long long version = -1;
  bool operator==(const GraphKey& o) const {
    return steps == o.steps && group == o.group && block == o.block && exact == o.exact &&
           bcpts == o.bcpts && dt == o.dt && version == o.version && pipe == o.pipe;
  }
};

struct pd_handle {
  int device = 0;
  cudaStream_t stream = nullptr;      // the stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the stream the handle created (destroyed with it)
  long long n = 0, nb = 0;
  int material = 0, kernel = 1, cmodel = 0, precision = 0, multi = 0, zem = 0;
  double cs = 0.5, maxdmg = 0.85;
  std::vector<DevParam> hp;
  std::vector<unsigned> hmeta;
  std::vector<void*> allocs;
  DevBody d{};
  IntDev g{};
  BCDev bc{};
  DevParam* dparams = nullptr;
  int* rev = nullptr;
  int* flags = nullptr;
  LaunchCfg cfg{1, 256, false, 0, 0};
  // FP32 OSB / CMat: the stored weighted volumes / shape tensors are stale (bond states
  // changed outside the kernels)
  bool kfull = true;
  bool damage_valid = false;
  bool has_bext_state = false;
  // boundary conditions (host side)
  std::vector<BCInfo> bcinfo;
  std::vector<int> bcn;
  long long per_step = 0;
  bool needs_table = false;
  double* table = nullptr;
  long long table_cap = 0;
  std::vector<unsigned char> bext_pt;  // points with b_ext conditions
  long long version = 0;
  // graphs
  int graph_steps = 0;
  cudaGraphExec_t gexec = nullptr;
  int graph_nodes = 0;
  GraphKey gkey;
  long long launches = 0;
  long long nan_step = -1;
  long long nslots = 0;
  pd::NKState* nk = nullptr;  // created by the first pd_nk_* call
  pd::DRState* dr = nullptr;  // created by pd_dr_init
  // staged Velocity Verlet run (pd_vv_begin .. pd_vv_end)
  long long stage_n = 0;
  double stage_dto = -1.0;
  // device staging for host transfers of point fields (pd_set_state, pd_get_field): grown on
  // demand and kept, so that a state upload or a field read allocates nothing
  void* xfer = nullptr;
  size_t xfer_bytes = 0;
};

template <class T>
inline pd_status dalloc(pd_handle* h, T** p, size_t count) {
  void* q = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * count);
  if (e != cudaSuccess)
    return pd_fail(e == cudaErrorMemoryAllocation ? PD_ERR_OOM : PD_ERR_CUDA,
                std::string("cudaMalloc of ") + std::to_string(sizeof(T) * count) + " bytes: " +
                    cudaGetErrorString(e));
  h->allocs.push_back(q);
  *p = (T*)q;
  return PD_OK;
}

inline void dfree(pd_handle* h, void* p) {
  if (!p) return;
  auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
  if (it != h->allocs.end()) h->allocs.erase(it);
  cudaFree(p);
}

// helpers implemented in pd_api.cu
pd_status pd_set_ctrl(pd_handle* h, size_t off, const void* src, size_t bytes);
pd_status pd_clear_error(pd_handle* h);
pd_status pd_check_err(pd_handle* h);
int pd_launch_force(pd_handle* h, int kstep, int phase);
