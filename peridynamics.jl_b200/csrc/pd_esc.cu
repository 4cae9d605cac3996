// pd_esc.cu -- EnergySurfaceCorrection (src/discretization/bond_system_corrections.jl of the
// reference, the energy based surface correction of Le and Bobaru 2018) on the device, for
// BBMaterial and OSBMaterial.
//
// Set-up, once after the pre-cracks (initialize!, :78-94):
//   mfactor[d, i] = Psi_theory(i) / Psi_pd(i, d)        calc_mfactor!, :96-124
//     Psi_pd: the strain energy density of point i (scfactor 1) with the reference positions
//     stretched by lambda = 1.001 along dimension d (BB: bond_based.jl:183-201; OSB:
//     ordinary_state_based.jl:206-234), Psi_theory = (lambda_L / 2 + mu) (lambda - 1)^2 with
//     the point's Lame parameters, averaged over its active bonds with several parameter sets
//     (get_averaged_lame_parameters, :126-152);
//   scfactor of bond i -> j from (mfactor_i + mfactor_j) / 2 along the bond's directions
//                                                       calc_scfactor!, :156-204
// One thread per point (per bond) in the reference's operation order; the FP64 set-up is the
// same for both precisions (the FP32 path stores the factor as float). The force kernels then
// multiply every bond by its factor (their ESC variants). The factor of a bond equals that of
// its reverse bond (both are made from |X_j - X_i| and the symmetric mean).
#include <cmath>

#include "pd_handle.h"

namespace pd {

__device__ __forceinline__ double esc_stretched(const double4& X, int k, int dim, double lam) {
  const double v = k == 0 ? X.x : (k == 1 ? X.y : X.z);
  return k == dim ? lam * v : v;
}

// reference bond length of slot b (the bond search's L)
__device__ __forceinline__ double esc_length(const DevBody& d, long long b, const double4& Xi,
                                             const double4& Xj) {
  if (d.len64) return fabs(d.len64[b]);
  const double dx = Xi.x - Xj.x, dy = Xi.y - Xj.y, dz = Xi.z - Xj.z;
  return sqrt((dx * dx + dy * dy) + dz * dz);
}

__global__ void k_esc_mfactor(DevBody d, int dim, double lam) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const DevParam& P = d.params[d.meta[i] & META_PID_MASK];
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  const double4 Xi = d.X0[i];
  const double xi[3] = {esc_stretched(Xi, 0, dim, lam), esc_stretched(Xi, 1, dim, lam),
                        esc_stretched(Xi, 2, dim, lam)};
  // get_averaged_lame_parameters
  double la = P.lambda, mu = P.mu;
  if (d.multi) {
    double sl = 0.0, sm = 0.0;
    long long na = 0;
    for (int k = 0; k < cnt; k++) {
      const long long b = bond_slot(d, i, k);
      if (!bond_bit(d.bits, b)) continue;
      const DevParam& Pj = d.params[d.meta[d.nbr[b]] & META_PID_MASK];
      sl += (P.lambda + Pj.lambda) / 2;
      sm += (P.mu + Pj.mu) / 2;
      na++;
    }
    la = sl / (double)na;
    mu = sm / (double)na;
  }
  const double psi_theory = (0.5 * la + mu) * ((lam - 1) * (lam - 1));
  double psi = 0.0;
  if (d.material == MAT_BB) {
    for (int k = 0; k < cnt; k++) {
      const long long b = bond_slot(d, i, k);
      const int j = d.nbr[b];
      const double4 Xj = d.X0[j];
      const double L = esc_length(d, b, Xi, Xj);
      const double dx = esc_stretched(Xj, 0, dim, lam) - xi[0], dy = esc_stretched(Xj, 1, dim, lam) - xi[1],
                   dz = esc_stretched(Xj, 2, dim, lam) - xi[2];
      const double l = sqrt((dx * dx + dy * dy) + dz * dz);
      const double eps = (l - L) / L;
      const double om = bond_bit(d.bits, b) ? 1.0 : 0.0;
      const double bc = (P.bc + d.params[d.meta[j] & META_PID_MASK].bc) / 2;
      psi += 0.25 * om * bc * eps * eps * L * Xj.w;
    }
  } else {
    double wvol = 0.0;
    for (int k = 0; k < cnt; k++) {
      const long long b = bond_slot(d, i, k);
      const double4 Xj = d.X0[d.nbr[b]];
      const double L = esc_length(d, b, Xi, Xj);
      const double DX = Xj.x - Xi.x, DY = Xj.y - Xi.y, DZ = Xj.z - Xi.z;
      const double om = bond_bit(d.bits, b) ? omega_of(d.kernel, P.delta, L) : 0.0;
      wvol += om * 1.0 * ((DX * DX + DY * DY) + DZ * DZ) * Xj.w;
    }
    if (wvol != 0.0) {  // otherwise the density keeps its cleared value 0
      double dil = 0.0;
      const double c1d = 3.0 / wvol;
      for (int k = 0; k < cnt; k++) {
        const long long b = bond_slot(d, i, k);
        const double4 Xj = d.X0[d.nbr[b]];
        const double L = esc_length(d, b, Xi, Xj);
        const double dx = esc_stretched(Xj, 0, dim, lam) - xi[0], dy = esc_stretched(Xj, 1, dim, lam) - xi[1],
                     dz = esc_stretched(Xj, 2, dim, lam) - xi[2];
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        const double om = bond_bit(d.bits, b) ? omega_of(d.kernel, P.delta, L) : 0.0;
        dil += om * 1.0 * c1d * L * (l - L) * Xj.w;
      }
      const double psivol = 0.5 * P.K * (dil * dil);
      double psidev = 0.0;
      for (int k = 0; k < cnt; k++) {
        const long long b = bond_slot(d, i, k);
        const int j = d.nbr[b];
        const double4 Xj = d.X0[j];
        const double L = esc_length(d, b, Xi, Xj);
        const double dx = esc_stretched(Xj, 0, dim, lam) - xi[0], dy = esc_stretched(Xj, 1, dim, lam) - xi[1],
                     dz = esc_stretched(Xj, 2, dim, lam) - xi[2];
        const double l = sqrt((dx * dx + dy * dy) + dz * dz);
        const double e = l - L;
        const double edev = e - 1.0 / 3.0 * dil * L;
        const double om = bond_bit(d.bits, b) ? omega_of(d.kernel, P.delta, L) : 0.0;
        const double G = (P.G + d.params[d.meta[j] & META_PID_MASK].G) / 2;
        const double cdev = 15.0 * G / (2 * wvol);
        psidev += cdev * om * 1.0 * edev * edev * Xj.w;
      }
      psi = psivol + psidev;
    }
  }
  d.mf[3 * i + dim] = psi_theory / psi;
}

// calc_scfactor! (:156-204), one thread per point over its bonds
__global__ void k_esc_scfactor(DevBody d, double* sc64, float* sc32) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const int cnt = (int)(d.off[i + 1] - d.off[i]);
  const double4 Xi = d.X0[i];
  const double half_pi = 90 * M_PI / 180;
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    const int j = d.nbr[b];
    const double4 Xj = d.X0[j];
    const double L = esc_length(d, b, Xi, Xj);
    const double ax = fabs(Xj.x - Xi.x), ay = fabs(Xj.y - Xi.y), az = fabs(Xj.z - Xi.z);
    const double scx = (d.mf[3 * i] + d.mf[3 * (long long)j]) / 2;
    const double scy = (d.mf[3 * i + 1] + d.mf[3 * (long long)j + 1]) / 2;
    const double scz = (d.mf[3 * i + 2] + d.mf[3 * (long long)j + 2]) / 2;
    double scr;
    if (!(az <= 1e-10) && ax <= 1e-10 && ay <= 1e-10) {
      scr = scz;
    } else {
      double th, ph;
      if (az <= 1e-10) {
        if (ay <= 1e-10) th = 0.0;
        else if (ax <= 1e-10) th = half_pi;
        else th = atan(ay / ax);
        ph = half_pi;
      } else {
        th = atan(ay / ax);
        ph = acos(az / L);
      }
      const double a = cos(th) * sin(ph), c = sin(th) * sin(ph), e = cos(ph);
      scr = sqrt(1 / ((a * a / (scx * scx) + c * c / (scy * scy)) + e * e / (scz * scz)));
    }
    if (sc64) sc64[b] = scr;
    else sc32[b] = (float)scr;
  }
}

// the factors of the bonds in CSR order
__global__ void k_esc_export(DevBody d, double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const long long o = d.off[i];
  const int cnt = (int)(d.off[i + 1] - o);
  for (int k = 0; k < cnt; k++) {
    const long long b = bond_slot(d, i, k);
    out[o + k] = d.sc64 ? d.sc64[b] : (double)d.sc32[b];
  }
}

static unsigned esc_blocks(long long n) { return (unsigned)((n + 127) / 128 > 0 ? (n + 127) / 128 : 1); }

}  // namespace pd

using namespace pd;

extern "C" pd_status pd_esc_init(pd_handle* h, int32_t what) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (what < 0 || what > 2) return pd_fail(PD_ERR_ARG, "what must be 0, 1 or 2");
  if (h->material != PD_MAT_BB && h->material != PD_MAT_OSB)
    return pd_fail(PD_ERR_UNSUPPORTED, "EnergySurfaceCorrection needs BBMaterial or OSBMaterial");
  PD_CUDA(cudaSetDevice(h->device));
  if (h->n == 0) return PD_OK;
  if (!h->d.mf) {
    double* mf = nullptr;
    PD_TRY(dalloc(h, &mf, 3 * h->n));
    h->d.mf = mf;
  }
  if (what != 2)
    for (int dim = 0; dim < 3; dim++) {
      k_esc_mfactor<<<esc_blocks(h->n), 128, 0, h->stream>>>(h->d, dim, 1.001);
      h->launches++;
    }
  if (what != 1) {
    double* sc64 = const_cast<double*>(h->d.sc64);
    float* sc32 = const_cast<float*>(h->d.sc32);
    if (h->precision == PD_PREC_FP64 && !sc64) PD_TRY(dalloc(h, &sc64, h->nslots));
    if (h->precision != PD_PREC_FP64 && !sc32) PD_TRY(dalloc(h, &sc32, h->nslots));
    k_esc_scfactor<<<esc_blocks(h->n), 128, 0, h->stream>>>(h->d, sc64, sc32);
    h->launches++;
    h->d.sc64 = sc64;
    h->d.sc32 = sc32;
    h->version++;     // cached step graphs hold the previous kernels
    h->kfull = true;  // stored weighted volumes hold the previous factors
  }
  PD_CUDA(cudaGetLastError());
  PD_CUDA(cudaStreamSynchronize(h->stream));
  return PD_OK;
}

extern "C" pd_status pd_esc_get(pd_handle* h, double* mfactor, double* scfactor) {
  if (!h) return pd_fail(PD_ERR_ARG, "handle is NULL");
  if (!h->d.mf) return pd_fail(PD_ERR_ARG, "no surface correction (pd_esc_init)");
  PD_CUDA(cudaSetDevice(h->device));
  PD_CUDA(cudaStreamSynchronize(h->stream));
  if (mfactor) PD_CUDA(cudaMemcpy(mfactor, h->d.mf, sizeof(double) * 3 * h->n, cudaMemcpyDeviceToHost));
  if (scfactor) {
    if (!h->d.sc64 && !h->d.sc32) return pd_fail(PD_ERR_ARG, "bond factors not computed (pd_esc_init 0 or 2)");
    double* tmp = nullptr;
    PD_CUDA(cudaMalloc(&tmp, sizeof(double) * (h->nb > 0 ? h->nb : 1)));
    k_esc_export<<<esc_blocks(h->n), 128, 0, h->stream>>>(h->d, tmp);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaMemcpy(scfactor, tmp, sizeof(double) * h->nb, cudaMemcpyDeviceToHost);
    cudaFree(tmp);
    if (e != cudaSuccess) return pd_fail(PD_ERR_CUDA, cudaGetErrorString(e));
  }
  return PD_OK;
}
