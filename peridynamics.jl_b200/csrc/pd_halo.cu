// pd_halo.cu -- partitioned bodies: Velocity Verlet in stages and the halo data that
// partitions exchange between the stages (the MPI data handler of the reference,
// src/core/mpi_body_data_handler.jl, re-expressed for one GPU per partition).
//
// A partition is a body whose rows are its owned points and its halo rows: copies of the
// points of other partitions that are bonded to an owned point, carrying only those bonds
// (pd_create_partition). Rows are numbered in the body's point order, so every owned point
// keeps the bond order of the undivided body and sums in the same order. One step is
//   stage 0  half kick, conditions, drift                        -> exchange kind 0
//   stage 1  first force kernel (BB: the whole force)            -> exchange kind 1 (OSB, CMat)
//   stage 2  second force kernel (OSB, CMat)
// and a run ends with the closing half kick (pd_vv_end). Kind 0 is the point state the force
// kernels gather from neighbours (current position, or displacement whose FP32 split is
// recomputed on arrival); kind 1 is the state the first kernel leaves for the second
// (OSB: the weighted volume / dilatation terms; CMat: F and P K^-1, or their FP32 products,
// and the killed flag, with which the halo row's bonds are cleared when bond states are
// directed). Halo rows evaluate their bonds' failure with the same positions and parameters
// as the owner, so their bond states agree with the owner's without an exchange.
#include <cmath>
#include <cstddef>

#include "pd_handle.h"

namespace pd {

struct HaloSeg {
  unsigned* base;  // row r holds words [r * words, (r + 1) * words)
  int words;
  int kill_only;   // the point-flag word: only the killed flag is taken over
};

struct HaloKind {
  HaloSeg seg[4];
  int nseg;
  int row_words;
};

static HaloKind halo_kind(const pd_handle* h, int kind) {
  HaloKind k{};
  auto add = [&](void* base, int words, int kill_only) {
    k.seg[k.nseg++] = HaloSeg{static_cast<unsigned*>(base), words, kill_only};
    k.row_words += words;
  };
  const DevBody& d = h->d;
  if (kind == 0) {
    add(d.cur, 8, 0);
  } else if (kind == 2) {
    add(d.mf, 6, 0);  // the row size holds before pd_esc_init allocates the array
  } else if (h->material == PD_MAT_OSB) {
    if (h->precision == PD_PREC_FP64) {
      add(d.coef64, 8, 0);
    } else {
      add(d.cc32, 2, 0);
      add(d.cm32, 2, 0);
    }
  } else if (h->material == PD_MAT_CMAT) {
    if (h->precision == PD_PREC_FP64) {
      add(d.F64, 18, 0);
      add(d.PK64, 18, 0);
      if (d.C164) add(d.C164, 18, 0);
    } else {
      add(d.cst32, 12, 0);
      if (d.zw32) add(d.zw32, 8, 0);
    }
    add(d.meta, 1, 1);
  }
  return k;
}

__device__ __forceinline__ int halo_seg_of(const HaloKind& k, int& w) {
  int s = 0;
  while (s + 1 < k.nseg && w >= k.seg[s].words) {
    w -= k.seg[s].words;
    s++;
  }
  return s;
}

// buf word t = word (t mod row_words) of row rows[t / row_words]; an index outside the body
// records error 4 and is skipped
__global__ void k_halo_pack(HaloKind k, long long n_body, const int* rows, long long n,
                            unsigned* buf, Ctrl* ctrl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k.row_words) return;
  const long long r = t / k.row_words;
  int w = (int)(t - r * k.row_words);
  const long long row = rows[r];
  if (row < 0 || row >= n_body) {
    ctrl->err = 4;
    return;
  }
  const int s = halo_seg_of(k, w);
  buf[t] = k.seg[s].base[row * k.seg[s].words + w];
}

// row rows[t / row_words] = buf word t; an index outside the body records error 4 and is skipped
__global__ void k_halo_unpack(HaloKind k, long long n_body, const int* rows, long long n,
                              const unsigned* buf, Ctrl* ctrl) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * k.row_words) return;
  const long long r = t / k.row_words;
  int w = (int)(t - r * k.row_words);
  const long long row = rows[r];
  if (row < 0 || row >= n_body) {
    ctrl->err = 4;
    return;
  }
  const int s = halo_seg_of(k, w);
  unsigned* dst = k.seg[s].base + row * k.seg[s].words + w;
  const unsigned v = buf[t];
  *dst = k.seg[s].kill_only ? ((*dst & ~META_KILLED) | (v & META_KILLED)) : v;
}

// directed bond states: a halo row its owner killed loses all its bonds (correspondence.jl:293)
__global__ void k_halo_kill_bonds(DevBody d, const int* rows, long long n) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const long long i = rows[r];
  if (i < 0 || i >= d.n || !(d.meta[i] & META_KILLED)) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  for (int k = 0; k < cnt; k++) clear_bit(d.bits, bond_slot(d, i, k));
}

static unsigned halo_blocks(long long work) { return (unsigned)((work + 255) / 256); }

}  // namespace pd

using namespace pd;

extern "C" pd_status pd_set_stream(pd_handle* h, void* stream) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  PD_CUDA(cudaSetDevice(h->device));
  PD_CUDA(cudaStreamSynchronize(h->stream));
  h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
  return PD_OK;
}

extern "C" pd_status pd_halo_row_bytes(pd_handle* h, int32_t kind, int64_t* bytes) {
  if (!h || !bytes) return pd_fail(PD_ERR_ARG, "NULL argument");
  if (kind < 0 || kind > 2) return pd_fail(PD_ERR_ARG, "kind must be 0, 1 or 2");
  *bytes = 4 * (int64_t)halo_kind(h, kind).row_words;
  return PD_OK;
}

extern "C" pd_status pd_halo_pack(pd_handle* h, int32_t kind, const int32_t* d_rows, int64_t n_rows,
                                  void* d_buf) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (kind < 0 || kind > 2) return pd_fail(PD_ERR_ARG, "kind must be 0, 1 or 2");
  if (n_rows < 0 || n_rows > h->n) return pd_fail(PD_ERR_ARG, "n_rows out of range");
  const HaloKind k = halo_kind(h, kind);
  if (n_rows == 0 || k.row_words == 0) return PD_OK;
  if (!d_rows || !d_buf) return pd_fail(PD_ERR_ARG, "NULL device array");
  if (kind == 2 && !h->d.mf) return pd_fail(PD_ERR_ARG, "no surface correction factors (pd_esc_init)");
  PD_CUDA(cudaSetDevice(h->device));
  k_halo_pack<<<halo_blocks(n_rows * k.row_words), 256, 0, h->stream>>>(
      k, h->n, d_rows, n_rows, static_cast<unsigned*>(d_buf), h->d.ctrl);
  h->launches++;
  PD_CUDA(cudaGetLastError());
  return PD_OK;
}

extern "C" pd_status pd_halo_unpack(pd_handle* h, int32_t kind, const int32_t* d_rows, int64_t n_rows,
                                    const void* d_buf) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (kind < 0 || kind > 2) return pd_fail(PD_ERR_ARG, "kind must be 0, 1 or 2");
  if (n_rows < 0 || n_rows > h->n) return pd_fail(PD_ERR_ARG, "n_rows out of range");
  const HaloKind k = halo_kind(h, kind);
  if (n_rows == 0 || k.row_words == 0) return PD_OK;
  if (!d_rows || !d_buf) return pd_fail(PD_ERR_ARG, "NULL device array");
  if (kind == 2 && !h->d.mf) return pd_fail(PD_ERR_ARG, "no surface correction factors (pd_esc_init)");
  PD_CUDA(cudaSetDevice(h->device));
  k_halo_unpack<<<halo_blocks(n_rows * k.row_words), 256, 0, h->stream>>>(
      k, h->n, d_rows, n_rows, static_cast<const unsigned*>(d_buf), h->d.ctrl);
  h->launches++;
  if (kind == 0 && h->precision != PD_PREC_FP64) {
    launch_split_u_rows(h->d, d_rows, n_rows, h->stream);
    h->launches++;
  }
  if (kind == 1 && h->material == PD_MAT_CMAT && !h->d.sym) {
    k_halo_kill_bonds<<<halo_blocks(n_rows), 256, 0, h->stream>>>(h->d, d_rows, n_rows);
    h->launches++;
  }
  PD_CUDA(cudaGetLastError());
  return PD_OK;
}

extern "C" pd_status pd_vv_begin(pd_handle* h, int64_t first_step, int64_t n_steps, double dt) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (first_step < 1 || n_steps < 1 || n_steps > (1LL << 30)) return pd_fail(PD_ERR_ARG, "invalid step range");
  PD_CUDA(cudaSetDevice(h->device));
  const double dto = dt > 0 ? dt : -1.0;
  if (dto < 0)
    for (auto& p : h->hp)
      if (!(p.dt > 0)) return pd_fail(PD_ERR_ARG, "dt <= 0 and no per-parameter time steps set");
  if (h->needs_table) {
    Ctrl c;
    // ordered after the handle's pending work (its stream is non-blocking)
    PD_CUDA(cudaMemcpyAsync(&c, h->d.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
    PD_CUDA(cudaStreamSynchronize(h->stream));
    if (c.table_first > first_step || c.table_first + c.table_n < first_step + n_steps)
      return pd_fail(PD_ERR_ARG, "boundary condition values do not cover steps " + std::to_string(first_step) +
                                     ".." + std::to_string(first_step + n_steps - 1));
  }
  PD_TRY(pd_clear_error(h));
  const long long base = first_step;
  PD_TRY(pd_set_ctrl(h, offsetof(Ctrl, base), &base, sizeof(long long)));
  h->stage_n = n_steps;
  h->stage_dto = dto;
  return PD_OK;
}

extern "C" pd_status pd_vv_stage(pd_handle* h, int32_t stage, int64_t kstep) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (h->stage_n <= 0) return pd_fail(PD_ERR_ARG, "no staged run open (pd_vv_begin)");
  if (kstep < 0 || kstep >= h->stage_n) return pd_fail(PD_ERR_ARG, "kstep outside the staged run");
  PD_CUDA(cudaSetDevice(h->device));
  const int k = (int)kstep;
  switch (stage) {
    case 0:
      launch_kick_drift(h->d, h->g, h->bc, k == 0 ? 0 : 1, h->stage_dto, k, h->stream);
      h->launches++;
      break;
    case 1:
      pd_launch_force(h, k, 1);
      break;
    case 2:
      pd_launch_force(h, k, 2);
      break;
    default:
      return pd_fail(PD_ERR_ARG, "stage must be 0, 1 or 2");
  }
  PD_CUDA(cudaGetLastError());
  return PD_OK;
}

extern "C" pd_status pd_vv_end(pd_handle* h) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (h->stage_n <= 0) return pd_fail(PD_ERR_ARG, "no staged run open (pd_vv_begin)");
  PD_CUDA(cudaSetDevice(h->device));
  launch_finish(h->d, h->g, h->stage_dto, h->stream);
  h->launches++;
  h->stage_n = 0;
  PD_CUDA(cudaGetLastError());
  h->damage_valid = true;
  return pd_check_err(h);
}

extern "C" pd_status pd_force_phase(pd_handle* h, int32_t phase, double t, double dt) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (phase != 1 && phase != 2) return pd_fail(PD_ERR_ARG, "phase must be 1 or 2");
  PD_CUDA(cudaSetDevice(h->device));
  if (phase == 1) {
    PD_TRY(pd_clear_error(h));
    const long long step = (t > 0 && dt > 0) ? (long long)std::floor(t / dt) : 0;
    PD_TRY(pd_set_ctrl(h, offsetof(Ctrl, base), &step, sizeof(long long)));
    pd_launch_force(h, 0, 1);
    PD_CUDA(cudaGetLastError());
    return PD_OK;
  }
  pd_launch_force(h, 0, 2);
  PD_CUDA(cudaGetLastError());
  h->damage_valid = true;
  return pd_check_err(h);
}

