// k-omega SST node-level model updates as one fused node kernel: turbulent
// viscosity, F1 blending, production, and the steady k / omega node terms.
//
// Reference: src/model/turbulence/RANS/shearStressTransport/shearStressTransportModel.cpp
// (updateTurbulentDynamicViscosity :597-678, updateFOneBlending :95-174,
// updateTurbulentProduction :176-420) and src/assemble/turbulence/RANS/
// shearStressTransport/segregatedShearStressTransport/{turbulentKineticEnergy/
// turbulentKineticEnergySSTAssemblerNodeTerms.cpp:13-127, turbulentEddyFrequency/
// turbulentEddyFrequencySSTAssemblerNodeTerms.cpp:13-218}. The fusion is exact:
// the omega node terms read k only through k_prev and grad k, which the k solve
// does not change before the omega assembly.
#include <cuda_runtime.h>

#include <string>

#include "oa_internal.h"

namespace oa {
namespace {

constexpr double SMALL = 2.220446049250313e-16;  // src/basic/types.h:179

struct SstArgs {
  oa_sst_constants c;
  oa_sst_fields f;
  double dt, mut_urf;
  int nn;
};

// One thread per node; every input is read once and every output written once
// (about 200 B in, 56 B out per node), so the kernel is HBM-bound.
__global__ void __launch_bounds__(256) k_sst_nodes(SstArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nn) return;
  const oa_sst_fields& f = a.f;
  const oa_sst_constants& C = a.c;
  const double k = __ldg(f.k + i), w = __ldg(f.omega + i), rho = __ldg(f.rho + i), mu = __ldg(f.mu + i),
               y = __ldg(f.ymin + i), vol = __ldg(f.vol + i), div = __ldg(f.div + i);
  double du[9], gk[3], gw[3];
#pragma unroll
  for (int q = 0; q < 9; ++q) du[q] = __ldg(f.gradU + 9L * i + q);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    gk[q] = __ldg(f.gradK + 3L * i + q);
    gw[q] = __ldg(f.gradW + 3L * i + q);
  }
  const double betaStar = C.beta_star, a1 = C.a1, sigmaWTwo = C.sigma_w2;

  // turbulent viscosity (F2-limited strain)
  double sijMag = 0.0;
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double s = 0.5 * (du[3 * p + q] + du[3 * q + p]);
      sijMag += s * s;
    }
  sijMag = sqrt(2.0 * sijMag);
  const double minDSq = y * y;
  const double trbDiss = sqrt(k) / betaStar / (w + SMALL) / (y + SMALL);
  const double lamDiss = 500.0 * mu / rho / (w + SMALL) / (minDSq + SMALL);
  const double fArgTwo = fmax(2.0 * trbDiss, lamDiss);
  const double fTwo = tanh(fArgTwo * fArgTwo);
  const double mut_val = a1 * rho * k / (fmax(a1 * w, sijMag * fTwo) + SMALL);
  const double mut = a.mut_urf * mut_val + (1.0 - a.mut_urf) * f.mut_old[i];
  f.mut[i] = mut;

  // F1 blending
  double crossDiff = 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) crossDiff += gk[q] * gw[q];
  const double CDkw = fmax(2.0 * rho * sigmaWTwo * crossDiff / (w + SMALL), 1.0e-10);
  const double fArgOne = fmin(fmax(trbDiss, lamDiss), 4.0 * rho * sigmaWTwo * k / (CDkw + SMALL) / (minDSq + SMALL));
  const double F1 = tanh(fArgOne * fArgOne * fArgOne * fArgOne);
  f.F1[i] = F1;

  // production (incompressible, fixed frame); wall nodes take the supplied
  // wall production
  double PkByMut = 0.0;
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) PkByMut += du[3 * p + q] * (du[3 * p + q] + du[3 * q + p]);
  PkByMut = fmax(PkByMut, 0.0);
  double Pk = fmax(mut * PkByMut, 0.0);
  if (__ldg(f.wall_node + i)) Pk = f.pk_wall ? __ldg(f.pk_wall + i) : 0.0;
  f.Pk[i] = Pk;

  // k node terms
  {
    double lhs = rho * vol / a.dt, rhs = 0.0;
    if (div < 0) lhs += -div;
    rhs -= -div * k;
    const double Dk = betaStar * rho * w * k;
    const double P = Pk > C.prod_limit * Dk ? C.prod_limit * Dk : Pk;
    rhs += (P - Dk) * vol;
    lhs += betaStar * rho * w * vol;
    f.k_diag[i] = lhs;
    f.k_rhs[i] = rhs;
  }
  // omega node terms
  {
    double lhs = rho * vol / a.dt, rhs = 0.0;
    if (div < 0) lhs += -div;
    rhs -= -div * w;
    const double kPre = __ldg(f.k_prev + i);
    const double arg2 = fmin(fmax(2 * sqrt(kPre) / (C.cmu * w * y + SMALL), 500 * mu / (pow(y, 2.0) * rho * w + SMALL)),
                             100.0);
    const double F2_old = tanh(pow(arg2, 2.0));
    const double P = fmin(PkByMut, ((C.prod_limit * betaStar) / a1) * w * fmax(a1 * w, F2_old * sqrt(2.0) * sijMag));
    const double om = 1.0 - F1;
    const double beta = F1 * C.beta1 + om * C.beta2;
    const double gamma = F1 * C.gamma1 + om * C.gamma2;
    const double sigmaD = 2.0 * om * sigmaWTwo;
    const double Pw = gamma * rho * P;
    const double Dw = beta * rho * w * w;
    const double Sw = sigmaD * rho * crossDiff / (w + SMALL);
    rhs += (Pw - Dw + Sw) * vol;
    lhs += (2.0 * beta * rho * w + fmax(Sw / (w + SMALL), 0.0)) * vol;
    f.w_diag[i] = lhs;
    f.w_rhs[i] = rhs;
  }
}

// The driver's viscosity updates after the node update, one thread per node:
// mu_eff = mu + mu_t (turbulenceModel::updateEffectiveDynamicViscosity,
// src/model/turbulence/turbulenceModel.cpp:121-150) and the k and omega
// diffusivities mu + mu_t (F1 sigma_1 + (1 - F1) sigma_2)
// (turbulentKineticEnergySSTEquation.cpp:55-75,
// turbulentEddyFrequencySSTEquation.cpp:55-75).
__global__ void k_sst_diffusivities(int nn, double sk1, double sk2, double sw1, double sw2,
                                    const double* __restrict__ mu, const double* __restrict__ mut,
                                    const double* __restrict__ F1, double* mu_eff, double* gk, double* gw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const double m = mu[i], t = mut[i], f1 = F1[i];
  const double ck = f1 * sk1 + (1.0 - f1) * sk2;
  const double cw = f1 * sw1 + (1.0 - f1) * sw2;
  gk[i] = m + t * ck;
  gw[i] = m + t * cw;
  mu_eff[i] = m + t;
}

}  // namespace
}  // namespace oa

using namespace oa;

extern "C" {

void oa_sst_default_constants(oa_sst_constants* c) {
  if (!c) return;
  c->sigma_k1 = 0.85;
  c->sigma_k2 = 1.0;
  c->sigma_w1 = 0.5;
  c->sigma_w2 = 0.856;
  c->beta1 = 0.075;
  c->beta2 = 0.0828;
  c->gamma1 = 0.5532;
  c->gamma2 = 0.4403;
  c->a1 = 0.31;
  c->beta_star = 0.09;
  c->prod_limit = 10.0;
  c->cmu = 0.09;
}

int oa_sst_node_update(int nn, const oa_sst_constants* c, double dt, double mut_urf, const oa_sst_fields* f,
                       void* stream) {
  if (nn < 0 || !c || !f || !(dt > 0.0)) return fail(OA_ERR_ARG, "oa_sst_node_update: bad arguments");
  const void* need[] = {f->k,   f->omega, f->k_prev, f->rho, f->mu,   f->ymin,   f->gradU,  f->gradK,  f->gradW,
                        f->div, f->vol,   f->mut_old, f->wall_node, f->mut, f->F1, f->Pk, f->k_diag, f->k_rhs,
                        f->w_diag, f->w_rhs};
  for (const void* p : need)
    if (!p) return fail(OA_ERR_ARG, "oa_sst_node_update: null field pointer");
  if (nn == 0) return OA_OK;
  SstArgs a{*c, *f, dt, mut_urf, nn};
  k_sst_nodes<<<(nn + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

int oa_sst_diffusivities(int nn, const oa_sst_constants* c, const double* mu, const double* mut, const double* F1,
                         double* mu_eff, double* gamma_k, double* gamma_w, void* stream) {
  if (nn < 0 || !c || !mu || !mut || !F1 || !mu_eff || !gamma_k || !gamma_w)
    return fail(OA_ERR_ARG, "oa_sst_diffusivities: bad arguments");
  if (nn == 0) return OA_OK;
  k_sst_diffusivities<<<(nn + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nn, c->sigma_k1, c->sigma_k2, c->sigma_w1, c->sigma_w2, mu, mut, F1, mu_eff, gamma_k, gamma_w);
  count_launches(1);
  OA_CUDA(cudaGetLastError());
  return OA_OK;
}

}  // extern "C"
