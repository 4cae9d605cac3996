// pd_nk.h -- state of the device Newton-Krylov solve and the helpers that the learned
// preconditioner (pd_mpnn.cu) shares with it (pd_nk.cu).
#pragma once
#include "pd_handle.h"

namespace pd {

constexpr int NK_NB = 592;   // blocks of the reduction kernels: 148 SMs x 4
constexpr int NK_TPB = 256;

// device scalars (doubles) of the solver
enum { SC_WW = 0, SC_UU = 1, SC_VV = 2, SC_EPS = 3, SC_RR = 4, SC_N = 8 };

struct NKState {
  long long ndof = 0, ld = 0;   // 3 n and the padded stride of the basis vectors
  int m = 0;                    // basis capacity (restart length)
  bool zbasis = false;
  int n_cond = 0;
  long long* cdof = nullptr;
  double* cval = nullptr;
  int* cfield = nullptr;
  unsigned char* cmask = nullptr;  // [3n] 1: dof carries a displacement condition
  double *Fu = nullptr, *Fp = nullptr, *r = nullptr, *x = nullptr, *t = nullptr, *s = nullptr;
  double *V = nullptr, *Z = nullptr;
  float* P = nullptr;           // [9n] block-Jacobi inverse blocks (column-major)
  float* D = nullptr;           // [9n] learned corrections
  bool have_D = false;
  float4* kx = nullptr;         // [2n] per point {X, Y, Z, V} (FP32 reference position) and
                                //      {v_x, v_y, v_z, 0}: the vector K0 is applied to
  double *part = nullptr, *h1 = nullptr, *h2 = nullptr, *hc = nullptr, *sc = nullptr,
         *y = nullptr;
  double* hpin = nullptr;       // pinned host copy of hc
  float* rec = nullptr;         // recorded residual directions
  long long rec_cap = 0, rec_n = 0;
};

// host helpers of pd_nk.cu
pd_status nk_ensure(pd_handle* h, int m);                 // solver state with a basis of m
void nk_dots_dev(pd_handle* h, const double* V, int k, const double* w, double* out);
void nk_apply_k0(pd_handle* h, const double* v, double* out);          // out = K0 v
void nk_compute_blocks(pd_handle* h);                                  // P = J_ii^-1 (BB)
// z = P (I + D) (a v + b s), constrained rows 0 (D null: P; s null: a v)
void nk_apply_blocks(pd_handle* h, const float* D, const double* v, double a, const double* s,
                     double b, double* z);

}  // namespace pd
