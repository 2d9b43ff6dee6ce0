// Oracle (test infrastructure only): CPU FP64 restatement of the node-level
// k-omega SST model updates and the steady k / omega node terms. Only tests
// use it, as the checker.
//
// Reference routines restated (paths relative to the reference project root):
//   - mu_t                src/model/turbulence/RANS/shearStressTransport/shearStressTransportModel.cpp:597-678
//                         (updateTurbulentDynamicViscosity)
//   - F1                  shearStressTransportModel.cpp:95-174 (updateFOneBlending)
//   - P_k                 shearStressTransportModel.cpp:176-420 (updateTurbulentProduction: the
//                         interior formula, incompressible, no rotating frame; wall nodes are
//                         zeroed and receive the wall production the caller supplies)
//   - k node terms        src/assemble/turbulence/RANS/shearStressTransport/segregatedShearStressTransport/
//                         turbulentKineticEnergy/turbulentKineticEnergySSTAssemblerNodeTerms.cpp:13-127
//   - omega node terms    .../turbulentEddyFrequency/turbulentEddyFrequencySSTAssemblerNodeTerms.cpp:13-218
//   - constants           shearStressTransportModel.h:21-37, RANSModel.h:20-22, turbulenceModel.h:20
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace {
constexpr double SMALL = 2.220446049250313e-16;  // src/basic/types.h:179
}

extern "C" {

void orc_sst_default_constants(orc_sst_constants* c) {
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

void orc_sst_nodes(int nn, const orc_sst_constants* C, double dt, double mut_urf, const orc_sst_in* in,
                   orc_sst_out* out) {
  const double betaStar = C->beta_star, a1 = C->a1, sigmaWTwo = C->sigma_w2;
  for (int i = 0; i < nn; ++i) {
    const double k = in->k[i], w = in->omega[i], rho = in->rho[i], mu = in->mu[i], y = in->ymin[i];
    const double* dudx = &in->gradU[9L * i];
    const double* gk = &in->gradK[3L * i];
    const double* gw = &in->gradW[3L * i];
    const double vol = in->vol[i], div = in->div[i];

    // updateTurbulentDynamicViscosity
    double sijMag = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        const double s = 0.5 * (dudx[3 * a + b] + dudx[3 * b + a]);
        sijMag += s * s;
      }
    sijMag = std::sqrt(2.0 * sijMag);
    double minDSq = y * y;
    double trbDiss = std::sqrt(k) / betaStar / (w + SMALL) / (y + SMALL);
    double lamDiss = 500.0 * mu / rho / (w + SMALL) / (minDSq + SMALL);
    const double fArgTwo = std::max(2.0 * trbDiss, lamDiss);
    const double fTwo = std::tanh(fArgTwo * fArgTwo);
    const double mut_val = a1 * rho * k / (std::max(a1 * w, sijMag * fTwo) + SMALL);
    const double mut = mut_urf * mut_val + (1.0 - mut_urf) * in->mut_old[i];
    out->mut[i] = mut;

    // updateFOneBlending
    double crossDiff = 0.0;
    for (int j = 0; j < 3; ++j) crossDiff += gk[j] * gw[j];
    const double CDkw = std::max(2.0 * rho * sigmaWTwo * crossDiff / (w + SMALL), 1.0e-10);
    const double fArgOne = std::min(std::max(trbDiss, lamDiss), 4.0 * rho * sigmaWTwo * k / (CDkw + SMALL) / (minDSq + SMALL));
    const double F1 = std::tanh(fArgOne * fArgOne * fArgOne * fArgOne);
    out->F1[i] = F1;

    // updateTurbulentProduction (incompressible, fixed frame)
    double PkByMut = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) PkByMut += dudx[3 * a + b] * (dudx[3 * a + b] + dudx[3 * b + a]);
    PkByMut = std::max(PkByMut, 0.0);
    double divergence = 0.0;
    for (int a = 0; a < 3; ++a) divergence += dudx[4 * a];
    PkByMut = std::max(PkByMut - 2.0 / 3.0 * divergence * divergence * 0.0, 0.0);
    double Pk = mut * PkByMut;
    Pk = std::max(std::max(Pk, 0.0) - 2.0 / 3.0 * divergence * rho * k * 0.0, 0.0);
    if (in->wall_node[i] != 0) Pk = in->pk_wall ? in->pk_wall[i] : 0.0;
    out->Pk[i] = Pk;

    // k node terms (steady)
    {
      double lhs = 0.0, rhs = 0.0;
      lhs += rho * vol / dt;
      if (div < 0) lhs += -div;
      rhs -= -div * k;
      const double Dk = betaStar * rho * w * k;
      double P = Pk;
      if (P > C->prod_limit * Dk) P = C->prod_limit * Dk;
      rhs += (P - Dk) * vol;
      lhs += betaStar * rho * w * vol;
      out->k_diag[i] = lhs;
      out->k_rhs[i] = rhs;
    }
    // omega node terms (steady)
    {
      double lhs = 0.0, rhs = 0.0;
      lhs += rho * vol / dt;
      if (div < 0) lhs += -div;
      rhs -= -div * w;
      double P = 0.0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) P += dudx[3 * a + b] * (dudx[3 * a + b] + dudx[3 * b + a]);
      P = std::max(P, 0.0);
      double dv = 0.0;
      for (int a = 0; a < 3; ++a) dv += dudx[4 * a];
      P += -2.0 / 3.0 * dv * dv * 0.0;
      const double kPre = in->k_prev[i];
      const double arg2 = std::min(std::max(2 * std::sqrt(kPre) / (C->cmu * w * y + SMALL),
                                            500 * mu / (std::pow(y, 2.0) * rho * w + SMALL)),
                                   100.0);
      const double F2_old = std::tanh(std::pow(arg2, 2.0));
      P = std::min(P, ((C->prod_limit * betaStar) / a1) * w * std::max(a1 * w, F2_old * std::sqrt(2.0) * sijMag));
      const double om = 1.0 - F1;
      const double beta = F1 * C->beta1 + om * C->beta2;
      const double gamma = F1 * C->gamma1 + om * C->gamma2;
      const double sigmaD = 2.0 * om * sigmaWTwo;
      const double Pw = gamma * rho * P;
      const double Dw = beta * rho * w * w;
      const double Sw = sigmaD * rho * crossDiff / (w + SMALL);
      rhs += (Pw - Dw + Sw) * vol;
      lhs += (2.0 * beta * rho * w + std::max(Sw / (w + SMALL), 0.0)) * vol;
      out->w_diag[i] = lhs;
      out->w_rhs[i] = rhs;
    }
  }
}

// turbulenceModel::updateEffectiveDynamicViscosity
// (src/model/turbulence/turbulenceModel.cpp:121-150): mu_eff = mu + mu_t; the
// diffusivity setup of turbulentKineticEnergySSTEquation.cpp:55-75 and
// turbulentEddyFrequencySSTEquation.cpp:55-75: mu + mu_t times the constant
// blended by F1 between the inner (1) and outer (2) values.
void orc_sst_diffusivities(int nn, const orc_sst_constants* C, const double* mu, const double* mut, const double* F1,
                           double* mu_eff, double* gamma_k, double* gamma_w) {
  for (int i = 0; i < nn; ++i) {
    const double bk = F1[i] * C->sigma_k1 + (1.0 - F1[i]) * C->sigma_k2;
    const double bw = F1[i] * C->sigma_w1 + (1.0 - F1[i]) * C->sigma_w2;
    gamma_k[i] = mu[i] + mut[i] * bk;
    gamma_w[i] = mu[i] + mut[i] * bw;
    mu_eff[i] = mu[i] + mut[i];
  }
}

}  // extern "C"
