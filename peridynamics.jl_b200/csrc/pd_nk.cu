// pd_nk.cu -- quasi-static Jacobian-free Newton-Krylov solve on the device
// (src/time_solvers/newton_krylov.jl of the reference).
//
// One load increment (pd_nk_step) follows newton_krylov_step! (:298-332):
//   apply_incr_boundary_conditions! (boundary_conditions.jl:229-236): value = beta f(p) into
//     the displacement (and the position of that dof, update_position! :349-357) or b_ext;
//   Newton loop: force density at u, r = (b_int + b_ext) V with r = 0 at constrained dofs
//     (calc_residual! :371-387), ||r|| against the tolerance, then J du = -r by restarted
//     (flexible) GMRES and u += du, x += du on the free dofs (update_displacement_from_du!
//     :673-686).
// J v is a finite-difference Frechet derivative of the same force kernels as the dynamic
// path: the reference's central rule (:504-567, 603-671) or the forward rule with
// eps = sqrt(eps_mach) |u| / |v| (one force evaluation, F(u) is the Newton residual's).
// Constrained rows of J v are v. The Krylov basis, the Gram-Schmidt products and the
// update of du are FP64 device vectors; the small Hessenberg least-squares problem runs on
// the host, which reads one column of h per Arnoldi step.
//
// Preconditioners (right preconditioning: FGMRES stores the preconditioned basis Z):
//   block Jacobi   z_i = P_i v_i, P_i = J_ii^-1 from the analytic bond-based tangent;
//   block poly     z = P (2v - K0 P v): one step of the Neumann series of (K0 P)^-1 with K0
//                  the small-strain bond stiffness of the reference configuration, applied
//                  as an FP32 bond sweep (one gather of v per bond);
//   learned        B_i = P_i (I + D_i) with per-point corrections D from the message-passing
//                  network, used alone or in the polynomial.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "pd_nk.h"

namespace pd {

void nk_release(pd_handle* h) {
  if (!h->nk) return;
  if (h->nk->hpin) cudaFreeHost(h->nk->hpin);
  delete h->nk;  // device arrays are in h->allocs and freed with the handle
  h->nk = nullptr;
}

// ------------------------------------------------------------------------------------------
// reductions and basis updates (deterministic: fixed partition, fixed reduction order)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// part[q * gridDim.x + block] = sum over the block's rows of V_q[r] w[r], q < k
__global__ void __launch_bounds__(NK_TPB) k_mdot(const double* __restrict__ V, int k, long long ld,
                                                 const double* __restrict__ w, long long n,
                                                 double* __restrict__ part) {
  __shared__ double red[NK_TPB / 32][4];
  const long long chunk = ((n + gridDim.x - 1) / gridDim.x + 31) / 32 * 32;
  const long long r0 = (long long)blockIdx.x * chunk;
  const long long r1 = r0 + chunk < n ? r0 + chunk : n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q0 = 0; q0 < k; q0 += 4) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const double wr = w[r];
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (q0 + u < k) acc[u] += V[(long long)(q0 + u) * ld + r] * wr;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const double s = warp_sum(acc[u]);
      if (lane == 0) red[warp][u] = s;
    }
    __syncthreads();
    if (threadIdx.x < 4 && q0 + (int)threadIdx.x < k) {
      double s = 0.0;
      for (int wp = 0; wp < NK_TPB / 32; wp++) s += red[wp][threadIdx.x];
      part[(long long)(q0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

// out[q] = sum_b part[q * nb + b], one warp per q
__global__ void k_reduce(const double* __restrict__ part, int k, int nb, double* __restrict__ out) {
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (q >= k) return;
  double s = 0.0;
  for (int b = lane; b < nb; b += 32) s += part[(long long)q * nb + b];
  s = warp_sum(s);
  if (lane == 0) out[q] = s;
}

// w = w + sgn * sum_q c[q] V_q
__global__ void __launch_bounds__(NK_TPB) k_mupd(double* __restrict__ w, const double* __restrict__ V,
                                                 int k, long long ld, const double* __restrict__ c,
                                                 double sgn, long long n) {
  extern __shared__ double cs[];
  for (int q = threadIdx.x; q < k; q += blockDim.x) cs[q] = c[q];
  __syncthreads();
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int q = 0; q < k; q++) acc += cs[q] * V[(long long)q * ld + r];
    w[r] = w[r] + sgn * acc;
  }
}

// hc[q] = h1[q] + h2[q] (q <= j), hc[j + 1] = sqrt(ww)
__global__ void k_column(const double* h1, const double* h2, const double* sc, int j, double* hc) {
  const int q = threadIdx.x;
  if (q <= j) hc[q] = h1[q] + h2[q];
  if (q == j + 1) hc[q] = sqrt(sc[SC_WW]);
}

__global__ void k_sqrt(const double* src, double* dst) { *dst = sqrt(*src); }

// v = v / *den (den == 0: v unchanged)
__global__ void k_scale(double* v, long long n, const double* den) {
  const double h = *den;
  if (!(h > 0.0)) return;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    v[r] = v[r] / h;
}

// dst = a * x + b * y (y may be null)
__global__ void k_axpby(double* dst, double a, const double* x, double b, const double* y, long long n) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    dst[r] = y ? a * x[r] + b * y[r] : a * x[r];
}

__global__ void k_to_f32(float* dst, const double* src, long long n) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    dst[r] = (float)src[r];
}

// compute_perturbation (newton_krylov.jl:537-567) and the forward rule
__global__ void k_eps(double* sc, int rule, double scale, double root_eps) {
  const double un = sqrt(sc[SC_UU]);
  double vn = sqrt(sc[SC_VV]);
  if (vn < DBL_EPSILON) vn = 1.0;
  sc[SC_EPS] = rule == 0 ? scale * root_eps * (un + 1.0) / vn
                         : scale * root_eps * (un > 0.0 ? un : 1.0) / vn;
}

// ------------------------------------------------------------------------------------------
// state kernels
// ------------------------------------------------------------------------------------------
// apply_psdbc! with beta (boundary_conditions.jl:154-163); displacement dofs also move their
// position (update_position!, newton_krylov.jl:349-357)
__global__ void k_cond(DevBody d, double* u, double* bext, const long long* cdof, const double* cval,
                       const int* cfield, int nc, double beta) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double value = beta * cval[c];
  const long long q = cdof[c];
  if (cfield[c] == 0) {
    if (isfinite(value)) u[q] = value;
    const long long i = q / 3;
    const int k = (int)(q - 3 * i);
    double* cp = reinterpret_cast<double*>(d.cur + i);
    const double* Xp = reinterpret_cast<const double*>(d.X0 + i);
    cp[k] = Xp[k] + u[q];
  } else if (isfinite(value)) {
    bext[q] = value;
  }
}

// position = X + (u + sgn eps v) (store_state_and_apply_perturbation!, :569-586,
// store_pos_force_and_apply_neg_perturbation! :588-601); v == null: position = X + u
// (compute_jvp_and_restore!, :646-671)
__global__ void k_pos(DevBody d, const double* __restrict__ u, const double* __restrict__ v,
                      const double* sc, double sgn) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 X = d.X0[i];
  double u0 = u[3 * i], u1 = u[3 * i + 1], u2 = u[3 * i + 2];
  if (v) {
    const double e = sgn * sc[SC_EPS];
    u0 = u0 + e * v[3 * i];
    u1 = u1 + e * v[3 * i + 1];
    u2 = u2 + e * v[3 * i + 2];
  }
  double4 c = d.cur[i];
  c.x = X.x + u0; c.y = X.y + u1; c.z = X.z + u2;
  d.cur[i] = c;
}

// r = (b_int + b_ext) V, 0 at constrained dofs; Fu = b_int V
__global__ void k_residual(DevBody d, const double* __restrict__ bext,
                           const unsigned char* __restrict__ cmask, double* __restrict__ r,
                           double* __restrict__ Fu) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * d.n) return;
  const double V = d.X0[q / 3].w;
  const double b = d.b64[q];
  Fu[q] = b * V;
  r[q] = cmask[q] ? 0.0 : (b + bext[q]) * V;
}

// mode 0: out = b_int V; mode 1 (forward): out = (b_int V - base) / eps; mode 2 (central):
// out = (base - b_int V) / (2 eps); constrained rows of modes 1, 2: out = v
__global__ void k_jv(DevBody d, const double* __restrict__ base, const double* __restrict__ v,
                     const unsigned char* __restrict__ cmask, const double* sc, int mode,
                     double* __restrict__ out) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * d.n) return;
  const double f = d.b64[q] * d.X0[q / 3].w;
  if (mode == 0) { out[q] = f; return; }
  if (cmask[q]) { out[q] = v[q]; return; }
  const double e = sc[SC_EPS];
  out[q] = mode == 1 ? (f - base[q]) / e : (base[q] - f) / (2.0 * e);
}

// u += du, x += du on the free dofs
__global__ void k_update(DevBody d, double* __restrict__ u, const double* __restrict__ du,
                         const unsigned char* __restrict__ cmask) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  double4 c = d.cur[i];
  double* cp = reinterpret_cast<double*>(&c);
  for (int k = 0; k < 3; k++) {
    const long long q = 3 * i + k;
    if (!cmask[q]) {
      u[q] += du[q];
      cp[k] += du[q];
    }
  }
  d.cur[i] = c;
}

// ------------------------------------------------------------------------------------------
// preconditioner kernels (bond-based material)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double bb_c(const DevBody& d, const DevParam& Pi, int j) {
  return d.multi ? 0.5 * (Pi.bc + d.params[d.meta[j] & META_PID_MASK].bc) : Pi.bc;
}

// P_i = J_ii^-1 with J_ii = -V_i sum_j V_j c [(1/L - 1/l) I + d d^T / l^3] over the active
// bonds (the derivative of the bond force of bond_based.jl:146-180 with respect to u_i);
// rows and columns of constrained dofs are the identity.
__global__ void k_bj_blocks(DevBody d, const unsigned char* __restrict__ cmask, float* __restrict__ P) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  const double4 xi = d.cur[i];
  const DevParam& Pi = d.params[d.meta[i] & META_PID_MASK];
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    if (!bond_bit(d.bits, b)) continue;
    const int j = d.nbr[b];
    const double L = fabs(d.len64[b]);
    const double4 xj = d.cur[j];
    const double dv[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
    const double l = sqrt((dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2]);
    const double s = bb_c(d, Pi, j) * xj.w * xi.w;
    const double a = s * (1.0 / L - 1.0 / l), g = s / (l * l * l);
    for (int c = 0; c < 3; c++)
      for (int r = 0; r < 3; r++) J[r + 3 * c] -= (r == c ? a : 0.0) + g * dv[r] * dv[c];
  }
  for (int a = 0; a < 3; a++) {
    if (!cmask[3 * i + a]) continue;
    for (int b = 0; b < 3; b++) J[a + 3 * b] = J[b + 3 * a] = (a == b) ? 1.0 : 0.0;
  }
  // inverse by cofactors
  const double c00 = J[4] * J[8] - J[7] * J[5], c01 = J[7] * J[2] - J[1] * J[8],
               c02 = J[1] * J[5] - J[4] * J[2];
  const double det = J[0] * c00 + J[3] * c01 + J[6] * c02;
  float* out = P + 9 * i;
  if (!(fabs(det) > 0.0) || !isfinite(det)) {
    for (int k = 0; k < 9; k++) out[k] = (k % 4) == 0 ? 1.0f : 0.0f;
    return;
  }
  const double id = 1.0 / det;
  double R[9];
  R[0] = c00 * id; R[1] = c01 * id; R[2] = c02 * id;
  R[3] = (J[6] * J[5] - J[3] * J[8]) * id;
  R[4] = (J[0] * J[8] - J[6] * J[2]) * id;
  R[5] = (J[3] * J[2] - J[0] * J[5]) * id;
  R[6] = (J[3] * J[7] - J[6] * J[4]) * id;
  R[7] = (J[6] * J[1] - J[0] * J[7]) * id;
  R[8] = (J[0] * J[4] - J[3] * J[1]) * id;
  for (int k = 0; k < 9; k++) out[k] = (float)R[k];
}

// z_i = B_i (a v_i + b s_i), B_i = P_i (I + D_i) (D null: P_i); constrained dofs 0
__global__ void k_block(const float* __restrict__ P, const float* __restrict__ D,
                        const double* __restrict__ v, double a, const double* __restrict__ s,
                        double b, const unsigned char* __restrict__ cmask, double* __restrict__ z,
                        long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double w[3];
  for (int k = 0; k < 3; k++) w[k] = s ? a * v[3 * i + k] + b * s[3 * i + k] : a * v[3 * i + k];
  if (D) {
    const float* Di = D + 9 * i;
    double t[3];
    for (int r = 0; r < 3; r++) t[r] = w[r] + ((Di[r] * w[0] + Di[r + 3] * w[1]) + Di[r + 6] * w[2]);
    for (int r = 0; r < 3; r++) w[r] = t[r];
  }
  const float* Pi = P + 9 * i;
  for (int r = 0; r < 3; r++) {
    const long long q = 3 * i + r;
    z[q] = cmask[q] ? 0.0 : (Pi[r] * w[0] + Pi[r + 3] * w[1]) + Pi[r + 6] * w[2];
  }
}

__global__ void k_init_kx(DevBody d, float4* __restrict__ kx) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double4 X = d.X0[i];
  kx[2 * i] = make_float4((float)X.x, (float)X.y, (float)X.z, (float)X.w);
}

__global__ void k_pack4(float4* __restrict__ kx, const double* __restrict__ v, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  kx[2 * i + 1] = make_float4((float)v[3 * i], (float)v[3 * i + 1], (float)v[3 * i + 2], 0.f);
}

// out_i = V_i sum_j c V_j / L^3 (xi . (v_j - v_i)) xi over the active bonds: the small-strain
// stiffness K0 of the reference configuration, in FP32 from FP32 copies of the reference
// positions (xi = X_j - X_i, L = |xi|: the bond arrays are read for the neighbour and the
// bond bit only, one 32-byte gather per bond); constrained rows 0
template <int G>
__global__ void __launch_bounds__(256) k_k0(DevBody d, const float4* __restrict__ kx,
                                            const unsigned char* __restrict__ cmask,
                                            double* __restrict__ out) {
  PD_SLICE_LOOP(G) {
    PD_SLICE_SETUP
    float ax = 0.f, ay = 0.f, az = 0.f;
    const float4 Xi = valid ? kx[2 * i] : make_float4(0, 0, 0, 0);
    const float4 vi = valid ? kx[2 * i + 1] : make_float4(0, 0, 0, 0);
    const DevParam& Pi = d.params[valid ? (d.meta[i] & META_PID_MASK) : 0];
    const float ci = (float)Pi.bc;
    const int self = valid ? (int)i : 0;
    // two rows per iteration: two independent neighbour gathers in flight per lane
    for (int r = 0; r < rows; r += 2) {
      const int k0 = r * G + gl, k1 = k0 + G;
      const long long b0 = sbase + (long long)r * 32 + lane, b1 = b0 + 32;
      const bool a0 = k0 < cnt && bond_bit(d.bits, b0);
      const bool a1 = r + 1 < rows && k1 < cnt && bond_bit(d.bits, b1);
      const int j0 = a0 ? __ldg(d.nbr + b0) : self;
      const int j1 = a1 ? __ldg(d.nbr + b1) : self;
      const float4 X0 = __ldg(kx + 2 * j0), v0 = __ldg(kx + 2 * j0 + 1);
      const float4 X1 = __ldg(kx + 2 * j1), v1 = __ldg(kx + 2 * j1 + 1);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const bool a = u ? a1 : a0;
        if (!a) continue;
        const float4 Xj = u ? X1 : X0, vj = u ? v1 : v0;
        const float ex = Xj.x - Xi.x, ey = Xj.y - Xi.y, ez = Xj.z - Xi.z;
        const float L2 = (ex * ex + ey * ey) + ez * ez;
        const float c = d.multi ? (float)bb_c(d, Pi, u ? j1 : j0) : ci;
        const float kk = c * Xj.w / (L2 * sqrtf(L2));
        const float pr = kk * (ex * (vj.x - vi.x) + ey * (vj.y - vi.y) + ez * (vj.z - vi.z));
        ax += pr * ex; ay += pr * ey; az += pr * ez;
      }
    }
    if (G > 1) { ax = group_sum<G>(ax); ay = group_sum<G>(ay); az = group_sum<G>(az); }
    if (valid && gl == 0) {
      const double V = Xi.w;
      out[3 * i] = cmask[3 * i] ? 0.0 : (double)ax * V;
      out[3 * i + 1] = cmask[3 * i + 1] ? 0.0 : (double)ay * V;
      out[3 * i + 2] = cmask[3 * i + 2] ? 0.0 : (double)az * V;
    }
  }
}

static int nk_grid(long long n, int t) {
  long long b = (n + t - 1) / t;
  if (b < 1) b = 1;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)b;
}

}  // namespace pd

using namespace pd;

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
static pd_status nk_state(pd_handle* h, int m) {
  if (!h->nk) {
    if (h->precision != PD_PREC_FP64)
      return pd_fail(PD_ERR_ARG, "the Newton-Krylov solve needs an FP64 handle (finite-difference "
                                 "Jacobian-vector products)");
    NKState* S = new NKState();
    h->nk = S;
    S->ndof = 3 * h->n;
    S->ld = (S->ndof + 31) / 32 * 32;
    const long long nd = S->ndof;
    PD_TRY(dalloc(h, &S->cmask, nd));
    PD_CUDA(cudaMemsetAsync(S->cmask, 0, nd, h->stream));
    PD_TRY(dalloc(h, &S->Fu, nd));
    PD_TRY(dalloc(h, &S->Fp, nd));
    PD_TRY(dalloc(h, &S->r, nd));
    PD_TRY(dalloc(h, &S->x, nd));
    PD_TRY(dalloc(h, &S->t, nd));
    PD_TRY(dalloc(h, &S->s, nd));
    PD_TRY(dalloc(h, &S->P, 9 * h->n));
    PD_TRY(dalloc(h, &S->kx, 2 * h->n));
    k_init_kx<<<nk_grid(h->n, 256), 256, 0, h->stream>>>(h->d, S->kx);
    PD_TRY(dalloc(h, &S->sc, SC_N));
    PD_CUDA(cudaMemsetAsync(S->sc, 0, SC_N * sizeof(double), h->stream));
  }
  NKState* S = h->nk;
  if (m > S->m) {
    dfree(h, S->V); dfree(h, S->Z); dfree(h, S->part); dfree(h, S->h1); dfree(h, S->h2);
    dfree(h, S->hc); dfree(h, S->y);
    S->V = S->Z = S->part = S->h1 = S->h2 = S->hc = S->y = nullptr;
    S->zbasis = false;
    if (S->hpin) { cudaFreeHost(S->hpin); S->hpin = nullptr; }
    PD_TRY(dalloc(h, &S->V, (size_t)(m + 1) * S->ld));
    PD_TRY(dalloc(h, &S->part, (size_t)(m + 1) * NK_NB));
    PD_TRY(dalloc(h, &S->h1, m + 2));
    PD_TRY(dalloc(h, &S->h2, m + 2));
    PD_TRY(dalloc(h, &S->hc, m + 2));
    PD_TRY(dalloc(h, &S->y, m + 2));
    PD_CUDA(cudaMallocHost(&S->hpin, sizeof(double) * (m + 2)));
    S->m = m;
  }
  return PD_OK;
}

static pd_status nk_zbasis(pd_handle* h) {
  NKState* S = h->nk;
  if (!S->zbasis) {
    PD_TRY(dalloc(h, &S->Z, (size_t)S->m * S->ld));
    S->zbasis = true;
  }
  return PD_OK;
}

// out[0..k) = V_q . w (V_q = V + q ld)
static void nk_dots(pd_handle* h, const double* V, int k, const double* w, double* out) {
  NKState* S = h->nk;
  k_mdot<<<NK_NB, NK_TPB, 0, h->stream>>>(V, k, S->ld, w, S->ndof, S->part);
  k_reduce<<<(k + 7) / 8, 256, 0, h->stream>>>(S->part, k, NK_NB, out);
  h->launches += 2;
}

static void nk_mupd(pd_handle* h, double* w, const double* V, int k, const double* c, double sgn) {
  NKState* S = h->nk;
  k_mupd<<<nk_grid(S->ndof, NK_TPB), NK_TPB, sizeof(double) * k, h->stream>>>(w, V, k, S->ld, c, sgn,
                                                                               S->ndof);
  h->launches++;
}

static void nk_force(pd_handle* h) { pd_launch_force(h, 0, 0); }

// J v into out (the current position is X + u on entry and on exit)
static void nk_matvec(pd_handle* h, const pd_nk_params& p, const double* v, double* out,
                      pd_nk_stats* st) {
  NKState* S = h->nk;
  const int pg = nk_grid(h->n, 256), qg = (int)((S->ndof + 255) / 256);
  nk_dots(h, v, 1, v, S->sc + SC_VV);
  const double root = p.frechet == PD_NK_CENTRAL ? std::cbrt(DBL_EPSILON) : std::sqrt(DBL_EPSILON);
  k_eps<<<1, 1, 0, h->stream>>>(S->sc, p.frechet == PD_NK_CENTRAL ? 0 : 1, p.perturbation_scale, root);
  k_pos<<<pg, 256, 0, h->stream>>>(h->d, h->g.u, v, S->sc, 1.0);
  nk_force(h);
  if (p.frechet == PD_NK_CENTRAL) {
    k_jv<<<qg, 256, 0, h->stream>>>(h->d, nullptr, v, S->cmask, S->sc, 0, S->Fp);
    k_pos<<<pg, 256, 0, h->stream>>>(h->d, h->g.u, v, S->sc, -1.0);
    nk_force(h);
    k_jv<<<qg, 256, 0, h->stream>>>(h->d, S->Fp, v, S->cmask, S->sc, 2, out);
    h->launches += 3;
    if (st) st->force_evals += 2;
  } else {
    k_jv<<<qg, 256, 0, h->stream>>>(h->d, S->Fu, v, S->cmask, S->sc, 1, out);
    h->launches += 1;
    if (st) st->force_evals += 1;
  }
  k_pos<<<pg, 256, 0, h->stream>>>(h->d, h->g.u, nullptr, S->sc, 0.0);
  h->launches += 3;
  if (st) st->matvecs++;
}

static void nk_k0(pd_handle* h, const double* v, double* out) {
  NKState* S = h->nk;
  k_pack4<<<nk_grid(h->n, 256), 256, 0, h->stream>>>(S->kx, v, h->n);
  long long blocks = (h->d.nslices + 7) / 8;
  if (blocks < 1) blocks = 1;
  if (PD_GRID_BLOCKS_PER_SM > 0 && blocks > 148LL * PD_GRID_BLOCKS_PER_SM)
    blocks = 148LL * PD_GRID_BLOCKS_PER_SM;
  const int grid = (int)blocks;
  switch (h->d.lg) {
    case 1: k_k0<1><<<grid, 256, 0, h->stream>>>(h->d, S->kx, S->cmask, out); break;
    case 2: k_k0<2><<<grid, 256, 0, h->stream>>>(h->d, S->kx, S->cmask, out); break;
    case 4: k_k0<4><<<grid, 256, 0, h->stream>>>(h->d, S->kx, S->cmask, out); break;
    case 8: k_k0<8><<<grid, 256, 0, h->stream>>>(h->d, S->kx, S->cmask, out); break;
    case 16: k_k0<16><<<grid, 256, 0, h->stream>>>(h->d, S->kx, S->cmask, out); break;
    default: k_k0<32><<<grid, 256, 0, h->stream>>>(h->d, S->kx, S->cmask, out); break;
  }
  h->launches += 2;
}

static pd_status nk_check_pc(pd_handle* h, int pc) {
  if (pc == PD_PC_NONE) return PD_OK;
  if (pc < 0 || pc > PD_PC_LEARNED)
    return pd_fail(PD_ERR_ARG, "unknown preconditioner " + std::to_string(pc));
  if (h->material != PD_MAT_BB)
    return pd_fail(PD_ERR_UNSUPPORTED, "block preconditioners need the bond-based material");
  if ((pc == PD_PC_LEARNED || pc == PD_PC_LEARNED_POLY) && !h->nk->have_D)
    return pd_fail(PD_ERR_ARG, "learned preconditioner without corrections (pd_nk_set_corrections)");
  return PD_OK;
}

static pd_status nk_prepare_pc(pd_handle* h, int pc) {
  NKState* S = h->nk;
  PD_TRY(nk_check_pc(h, pc));
  if (pc == PD_PC_NONE) return PD_OK;
  k_bj_blocks<<<nk_grid(h->n, 128), 128, 0, h->stream>>>(h->d, S->cmask, S->P);
  h->launches++;
  return PD_OK;
}

// z = M v
static void nk_precond(pd_handle* h, int pc, const double* v, double* z, pd_nk_stats* st) {
  NKState* S = h->nk;
  const int g = nk_grid(h->n, 256);
  const float* D = (pc == PD_PC_LEARNED || pc == PD_PC_LEARNED_POLY) ? S->D : nullptr;
  if (pc == PD_PC_BLOCK_JACOBI || pc == PD_PC_LEARNED) {
    k_block<<<g, 256, 0, h->stream>>>(S->P, D, v, 1.0, nullptr, 0.0, S->cmask, z, h->n);
    h->launches++;
  } else {
    k_block<<<g, 256, 0, h->stream>>>(S->P, D, v, 1.0, nullptr, 0.0, S->cmask, S->t, h->n);
    nk_k0(h, S->t, S->s);
    k_block<<<g, 256, 0, h->stream>>>(S->P, D, v, 2.0, S->s, -1.0, S->cmask, z, h->n);
    h->launches += 2;
  }
  if (st) st->precond_applies++;
}

static void nk_record(pd_handle* h, const double* v) {
  NKState* S = h->nk;
  if (S->rec_n >= S->rec_cap) return;
  k_to_f32<<<nk_grid(S->ndof, 256), 256, 0, h->stream>>>(S->rec + S->rec_n * S->ndof, v, S->ndof);
  h->launches++;
  S->rec_n++;
}

// force density at the current state, r and Fu; returns ||r||
static pd_status nk_residual(pd_handle* h, double* rnorm) {
  NKState* S = h->nk;
  nk_force(h);
  k_residual<<<(int)((S->ndof + 255) / 256), 256, 0, h->stream>>>(h->d, h->g.bext, S->cmask, S->r, S->Fu);
  h->launches++;
  nk_dots(h, S->r, 1, S->r, S->sc + SC_RR);
  double rr = 0.0;
  PD_CUDA(cudaMemcpyAsync(&rr, S->sc + SC_RR, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  PD_TRY(pd_check_err(h));  // synchronises
  *rnorm = std::sqrt(rr);
  return PD_OK;
}

// restarted (flexible) GMRES for J du = -r from du = 0 (gmres! of IterativeSolvers.jl as
// called at newton_krylov.jl:448-450); du in S->x
static pd_status nk_linear(pd_handle* h, const pd_nk_params& p, double rnorm, pd_nk_stats* st) {
  NKState* S = h->nk;
  const long long nd = S->ndof, ld = S->ld;
  const int m = p.gmres_restart;
  const int pc = p.precond;
  const int vg = nk_grid(nd, 256);
  PD_CUDA(cudaMemsetAsync(S->x, 0, sizeof(double) * nd, h->stream));
  double beta = rnorm;
  const double tol = std::max(p.gmres_reltol * beta, p.gmres_abstol);
  if (beta <= tol) return PD_OK;
  PD_TRY(nk_prepare_pc(h, pc));
  if (pc != PD_PC_NONE) PD_TRY(nk_zbasis(h));
  // u_norm of the Frechet step: fixed during the solve
  nk_dots(h, h->g.u, 1, h->g.u, S->sc + SC_UU);
  k_axpby<<<vg, 256, 0, h->stream>>>(S->V, -1.0 / beta, S->r, 0.0, nullptr, nd);
  h->launches++;
  nk_record(h, S->V);
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
  long long it = 0;
  double res = beta;
  for (;;) {
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int cols = 0;
    bool stop = false;
    for (int j = 0; j < m; j++) {
      double* vj = S->V + (size_t)j * ld;
      double* zj = vj;
      if (pc != PD_PC_NONE) {
        zj = S->Z + (size_t)j * ld;
        nk_precond(h, pc, vj, zj, st);
      }
      double* w = S->V + (size_t)(j + 1) * ld;
      nk_matvec(h, p, zj, w, st);
      it++;
      st->gmres_iters++;
      // classical Gram-Schmidt with one re-orthogonalisation
      nk_dots(h, S->V, j + 1, w, S->h1);
      nk_mupd(h, w, S->V, j + 1, S->h1, -1.0);
      nk_dots(h, S->V, j + 1, w, S->h2);
      nk_mupd(h, w, S->V, j + 1, S->h2, -1.0);
      nk_dots(h, w, 1, w, S->sc + SC_WW);
      k_column<<<1, ((j + 2 + 31) / 32) * 32, 0, h->stream>>>(S->h1, S->h2, S->sc, j, S->hc);
      k_scale<<<vg, 256, 0, h->stream>>>(w, nd, S->hc + j + 1);
      h->launches += 2;
      PD_CUDA(cudaMemcpyAsync(S->hpin, S->hc, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost,
                              h->stream));
      PD_TRY(pd_check_err(h));  // synchronises
      double* col = &H[(size_t)j * (m + 1)];
      for (int q = 0; q <= j + 1; q++) col[q] = S->hpin[q];
      for (int q = 0; q < j; q++) {
        const double a = cs[q] * col[q] + sn[q] * col[q + 1];
        col[q + 1] = -sn[q] * col[q] + cs[q] * col[q + 1];
        col[q] = a;
      }
      const double rho = std::hypot(col[j], col[j + 1]);
      if (rho == 0.0) { cs[j] = 1.0; sn[j] = 0.0; }
      else { cs[j] = col[j] / rho; sn[j] = col[j + 1] / rho; }
      col[j] = rho;
      col[j + 1] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      res = std::fabs(g[j + 1]);
      cols = j + 1;
      const bool breakdown = !(S->hpin[j + 1] > 0.0);
      if (res <= tol || it >= p.gmres_maxiter || breakdown) { stop = true; break; }
    }
    // y = H^-1 g (upper triangular), du += Z y
    for (int q = cols - 1; q >= 0; q--) {
      double s = g[q];
      for (int c = q + 1; c < cols; c++) s -= H[(size_t)c * (m + 1) + q] * y[c];
      const double dq = H[(size_t)q * (m + 1) + q];
      y[q] = dq != 0.0 ? s / dq : 0.0;
    }
    PD_CUDA(cudaMemcpyAsync(S->y, y.data(), sizeof(double) * cols, cudaMemcpyHostToDevice, h->stream));
    nk_mupd(h, S->x, pc != PD_PC_NONE ? S->Z : S->V, cols, S->y, 1.0);
    if (stop) break;
    // restart from the true residual -r - J du
    nk_matvec(h, p, S->x, S->t, st);
    k_axpby<<<vg, 256, 0, h->stream>>>(S->V, -1.0, S->r, -1.0, S->t, nd);
    h->launches++;
    nk_dots(h, S->V, 1, S->V, S->sc + SC_WW);
    k_sqrt<<<1, 1, 0, h->stream>>>(S->sc + SC_WW, S->hc);
    h->launches++;
    PD_CUDA(cudaMemcpyAsync(S->hpin, S->hc, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PD_TRY(pd_check_err(h));  // synchronises
    beta = S->hpin[0];
    if (beta <= tol) break;
    k_scale<<<vg, 256, 0, h->stream>>>(S->V, nd, S->hc);
    h->launches++;
    nk_record(h, S->V);
  }
  PD_CUDA(cudaGetLastError());
  return PD_OK;
}

static pd_status nk_check_params(const pd_nk_params* p) {
  if (!p) return pd_fail(PD_ERR_ARG, "parameters are NULL");
  if (p->maxiter <= 0) return pd_fail(PD_ERR_ARG, "maxiter has to be larger than zero: maxiter > 0");
  if (!(p->tol > 0)) return pd_fail(PD_ERR_ARG, "tolerance has to be larger than zero: tol > 0");
  if (!(p->gmres_reltol > 0))
    return pd_fail(PD_ERR_ARG, "gmres_reltol has to be larger than zero: gmres_reltol > 0");
  if (!(p->gmres_abstol > 0))
    return pd_fail(PD_ERR_ARG, "gmres_abstol has to be larger than zero: gmres_abstol > 0");
  if (p->gmres_maxiter <= 0)
    return pd_fail(PD_ERR_ARG, "gmres_maxiter has to be larger than zero: gmres_maxiter > 0");
  if (p->gmres_restart <= 0 || p->gmres_restart > 1000)
    return pd_fail(PD_ERR_ARG, "gmres_restart has to be in 1..1000");
  if (!(p->perturbation_scale > 0))
    return pd_fail(PD_ERR_ARG, "perturbation_scale has to be larger than zero: perturbation_scale > 0");
  if (p->frechet != PD_NK_CENTRAL && p->frechet != PD_NK_FORWARD)
    return pd_fail(PD_ERR_ARG, "unknown Frechet rule");
  return PD_OK;
}

extern "C" pd_status pd_nk_set_conditions(pd_handle* h, int32_t n, const pd_nk_condition* conds) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (n < 0 || (n > 0 && !conds)) return pd_fail(PD_ERR_ARG, "invalid condition list");
  PD_CUDA(cudaSetDevice(h->device));
  PD_TRY(nk_state(h, 1));
  NKState* S = h->nk;
  std::vector<long long> dof;
  std::vector<double> val;
  std::vector<int> fld;
  std::vector<unsigned char> mask(S->ndof, 0);
  for (int c = 0; c < n; c++) {
    const pd_nk_condition& k = conds[c];
    if (k.field < 0 || k.field > 1 || k.dim < 0 || k.dim > 2 || k.n_points < 0 ||
        (k.n_points > 0 && (!k.points || !k.values)))
      return pd_fail(PD_ERR_ARG, "invalid condition " + std::to_string(c));
    for (long long q = 0; q < k.n_points; q++) {
      const long long i = k.points[q];
      if (i < 0 || i >= h->n) return pd_fail(PD_ERR_ARG, "condition point index out of range");
      dof.push_back(3 * i + k.dim);
      val.push_back(k.values[q]);
      fld.push_back(k.field);
      if (k.field == 0) mask[3 * i + k.dim] = 1;
    }
  }
  dfree(h, S->cdof); dfree(h, S->cval); dfree(h, S->cfield);
  S->cdof = nullptr; S->cval = nullptr; S->cfield = nullptr;
  S->n_cond = (int)dof.size();
  PD_TRY(dalloc(h, &S->cdof, dof.size()));
  PD_TRY(dalloc(h, &S->cval, val.size()));
  PD_TRY(dalloc(h, &S->cfield, fld.size()));
  if (!dof.empty()) {
    PD_CUDA(cudaMemcpyAsync(S->cdof, dof.data(), sizeof(long long) * dof.size(), cudaMemcpyHostToDevice, h->stream));
    PD_CUDA(cudaMemcpyAsync(S->cval, val.data(), sizeof(double) * val.size(), cudaMemcpyHostToDevice, h->stream));
    PD_CUDA(cudaMemcpyAsync(S->cfield, fld.data(), sizeof(int) * fld.size(), cudaMemcpyHostToDevice, h->stream));
  }
  PD_CUDA(cudaMemcpyAsync(S->cmask, mask.data(), S->ndof, cudaMemcpyHostToDevice, h->stream));
  PD_CUDA(cudaStreamSynchronize(h->stream));
  return PD_OK;
}

extern "C" pd_status pd_nk_set_corrections(pd_handle* h, const float* D) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  PD_CUDA(cudaSetDevice(h->device));
  PD_TRY(nk_state(h, 1));
  NKState* S = h->nk;
  if (!D) { S->have_D = false; return PD_OK; }
  if (!S->D) PD_TRY(dalloc(h, &S->D, 9 * h->n));
  PD_CUDA(cudaMemcpyAsync(S->D, D, sizeof(float) * 9 * h->n, cudaMemcpyHostToDevice, h->stream));
  PD_CUDA(cudaStreamSynchronize(h->stream));
  S->have_D = true;
  return PD_OK;
}

extern "C" pd_status pd_nk_record(pd_handle* h, int64_t capacity) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (capacity < 0) return pd_fail(PD_ERR_ARG, "capacity < 0");
  PD_CUDA(cudaSetDevice(h->device));
  PD_TRY(nk_state(h, 1));
  NKState* S = h->nk;
  dfree(h, S->rec);
  S->rec = nullptr;
  S->rec_cap = S->rec_n = 0;
  if (capacity > 0) {
    PD_TRY(dalloc(h, &S->rec, (size_t)capacity * S->ndof));
    S->rec_cap = capacity;
  }
  return PD_OK;
}

extern "C" pd_status pd_nk_recorded(pd_handle* h, int64_t* n) {
  if (!h || !n) return pd_fail(PD_ERR_ARG, "NULL argument");
  *n = h->nk ? h->nk->rec_n : 0;
  return PD_OK;
}

extern "C" pd_status pd_nk_recorded_vector(pd_handle* h, int64_t k, float* out) {
  if (!h || !out) return pd_fail(PD_ERR_ARG, "NULL argument");
  if (!h->nk || k < 0 || k >= h->nk->rec_n) return pd_fail(PD_ERR_ARG, "recorded index out of range");
  PD_CUDA(cudaSetDevice(h->device));
  PD_CUDA(cudaMemcpyAsync(out, h->nk->rec + k * h->nk->ndof, sizeof(float) * h->nk->ndof,
                          cudaMemcpyDeviceToHost, h->stream));
  PD_CUDA(cudaStreamSynchronize(h->stream));
  return PD_OK;
}

extern "C" pd_status pd_nk_apply(pd_handle* h, int32_t op, const pd_nk_params* p, const double* v,
                                 double* out) {
  if (!h || !out || (op != 3 && !v)) return pd_fail(PD_ERR_ARG, "NULL argument");
  if (op < 0 || op > 3) return pd_fail(PD_ERR_ARG, "unknown operator");
  PD_TRY(nk_check_params(p));
  PD_CUDA(cudaSetDevice(h->device));
  PD_TRY(pd_clear_error(h));
  PD_TRY(nk_state(h, p->gmres_restart));
  NKState* S = h->nk;
  const size_t bytes = sizeof(double) * S->ndof;
  if (op == 3) {
    double rn;
    PD_TRY(nk_residual(h, &rn));
    PD_CUDA(cudaMemcpyAsync(out, S->r, bytes, cudaMemcpyDeviceToHost, h->stream));
    PD_CUDA(cudaStreamSynchronize(h->stream));
    return PD_OK;
  }
  double* dv = S->V;
  double* dout = S->V + S->ld;
  PD_CUDA(cudaMemcpyAsync(dv, v, bytes, cudaMemcpyHostToDevice, h->stream));
  if (op == 0) {
    double rn;
    PD_TRY(nk_residual(h, &rn));  // F(u) for the forward rule
    nk_dots(h, h->g.u, 1, h->g.u, S->sc + SC_UU);
    nk_matvec(h, *p, dv, dout, nullptr);
  } else if (op == 1) {
    nk_k0(h, dv, dout);
  } else {
    PD_TRY(nk_prepare_pc(h, p->precond));
    if (p->precond == PD_PC_NONE)
      PD_CUDA(cudaMemcpyAsync(dout, dv, bytes, cudaMemcpyDeviceToDevice, h->stream));
    else
      nk_precond(h, p->precond, dv, dout, nullptr);
  }
  PD_CUDA(cudaGetLastError());
  PD_CUDA(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, h->stream));
  return pd_check_err(h);
}

extern "C" pd_status pd_nk_step(pd_handle* h, int64_t step, double beta, const pd_nk_params* p,
                                pd_nk_stats* st) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  PD_TRY(nk_check_params(p));
  pd_nk_stats local{};
  if (!st) st = &local;
  *st = pd_nk_stats{};
  PD_CUDA(cudaSetDevice(h->device));
  PD_TRY(pd_clear_error(h));
  PD_TRY(nk_state(h, p->gmres_restart));
  PD_TRY(nk_check_pc(h, p->precond));
  NKState* S = h->nk;
  const long long base = step;
  PD_TRY(pd_set_ctrl(h, offsetof(Ctrl, base), &base, sizeof(long long)));
  if (S->n_cond > 0) {
    k_cond<<<(S->n_cond + 127) / 128, 128, 0, h->stream>>>(h->d, h->g.u, h->g.bext, S->cdof, S->cval,
                                                          S->cfield, S->n_cond, beta);
    h->launches++;
  }
  for (int iter = 1; iter <= p->maxiter; iter++) {
    double rn = 0.0;
    PD_TRY(nk_residual(h, &rn));
    st->force_evals++;
    st->newton_iters = iter;
    st->residual = rn;
    if (iter == 1) st->residual_first = rn;
    const bool conv = p->tol_relative ? rn <= p->tol * st->residual_first : rn < p->tol;
    if (conv) { st->converged = 1; break; }
    if (iter == p->maxiter) break;
    PD_TRY(nk_linear(h, *p, rn, st));
    k_update<<<nk_grid(h->n, 256), 256, 0, h->stream>>>(h->d, h->g.u, S->x, S->cmask);
    h->launches++;
  }
  h->damage_valid = true;
  PD_CUDA(cudaGetLastError());
  PD_CUDA(cudaStreamSynchronize(h->stream));
  if (!st->converged)
    return pd_fail(PD_ERR_NOCONV, "Newton-Krylov solver did not converge after max iterations!\n"
                                  "Consider increasing `maxiter` or `tol`.");
  return PD_OK;
}

// helpers shared with pd_mpnn.cu
namespace pd {
pd_status nk_ensure(pd_handle* h, int m) { return nk_state(h, m); }
void nk_dots_dev(pd_handle* h, const double* V, int k, const double* w, double* out) {
  nk_dots(h, V, k, w, out);
}
void nk_apply_k0(pd_handle* h, const double* v, double* out) { nk_k0(h, v, out); }
void nk_compute_blocks(pd_handle* h) {
  k_bj_blocks<<<nk_grid(h->n, 128), 128, 0, h->stream>>>(h->d, h->nk->cmask, h->nk->P);
  h->launches++;
}
void nk_apply_blocks(pd_handle* h, const float* D, const double* v, double a, const double* s,
                     double b, double* z) {
  k_block<<<nk_grid(h->n, 256), 256, 0, h->stream>>>(h->nk->P, D, v, a, s, b, h->nk->cmask, z, h->n);
  h->launches++;
}
}  // namespace pd
