// Deck-level constants for hosts that hold only the input decks: the
// influence-function parameters and the bond-law constants that the
// reference's material constructors derive from a MaterialDeck.  Host code
// only (no device work), in the reference's evaluation order, so that a
// binding needs neither the materials' private members nor a copy of these
// formulas.
//
//   influence functions: influenceFn.cpp:13-85 (defaults), 25-27, 59-61,
//                        90-121 (moments)
//   RnpMaterial:  material.h:541-620 (C, beta, rbar, invFactor)
//   PmbMaterial:  material.h:919-997 (c, s0)
//   PdElastic:    material.h:1257-1305 (c)
//   PdState:      material.h:1579-1700 (K, G, s0)
//   internal contact stiffness of broken bonds: baseParticle.cpp:156-179
#include <cmath>
#include <cstdint>

#include "pdgpu_internal.h"

namespace {

double moment(int type, const double p[2], int i) {
  if (type == PDGPU_INF_CONST) return p[0] / double(i + 1);
  if (type == PDGPU_INF_LINEAR) return (p[0] / double(i + 1)) + (p[1] / double(i + 2));
  const double a = p[0], b = p[1];
  const double sq1 = std::sqrt(b), sq2 = std::sqrt(M_PI);
  if (i == 0) return 0.5 * a * sq1 * sq2 * std::erf(1. / sq1);
  if (i == 1) return 0.5 * a * b * (1. - std::exp(-1. / b));
  if (i == 2) return 0.5 * a * b * sq1 * (0.5 * sq2 * std::erf(1. / sq1) - (1. / sq1) * std::exp(-1. / b));
  return 0.5 * a * b * b * (1. - (1. + 1. / b) * std::exp(-1. / b));
}

double toK(double E, double nu) { return E / (3. * (1. - 2. * nu)); }
double toLambdaE(double E, double nu) { return E * nu / ((1. + nu) * (1. - 2. * nu)); }
double toGE(double E, double nu) { return E / (2. * (1. + nu)); }
double toELambda(double l, double nu) { return l * (1. + nu) * (1. - 2. * nu) / nu; }

}  // namespace

extern "C" {

PDGPU_API int pdgpu_influence_params(int32_t type, int32_t n_params, const double *params, int32_t dim,
                                     double out[2]) {
  if (!out || dim < 1 || dim > 3 || n_params < 0 || (n_params > 0 && !params)) return PDGPU_ERR_ARG;
  out[0] = out[1] = 0.;
  if (type == PDGPU_INF_CONST) {
    out[0] = n_params > 0 ? params[0] : double(dim + 1);
  } else if (type == PDGPU_INF_LINEAR) {
    if (n_params == 0) {
      out[0] = dim == 1 ? 6. : (dim == 2 ? 12. : 20.);
      out[1] = -out[0];
    } else {
      out[0] = params[0];
      out[1] = n_params < 2 ? -params[0] : params[1];
    }
  } else if (type == PDGPU_INF_GAUSSIAN) {
    if (n_params >= 2) {
      out[0] = params[0];
      out[1] = params[1];
    } else {
      const double b = 0.2;
      out[1] = b;
      if (dim == 1)
        out[0] = 2. / (b * (1. - std::exp(-1. / b)));
      else if (dim == 2)
        out[0] = (4.0 / b) * 1.0 / (std::sqrt(M_PI * b) * std::erf(1.0 / std::sqrt(b)) - 2.0 * std::exp(-1.0 / b));
      else
        out[0] = (2.0 / b) * 1.0 / (b - (b + 1.) * std::exp(-1.0 / b));
    }
  } else {
    return PDGPU_ERR_ARG;
  }
  return PDGPU_OK;
}

PDGPU_API int pdgpu_material_constants(const pdgpu_material_deck *deck, int32_t dim, double horizon,
                                       int32_t inf_type, const double inf_params[2], double mat[6],
                                       double *bulk_modulus) {
  if (!deck || !inf_params || !mat || dim < 2 || dim > 3 || !(horizon > 0)) return PDGPU_ERR_ARG;
  double E = deck->E, K = deck->K, G = deck->G, nu = deck->nu;
  const double Gc = deck->Gc;
  for (int q = 0; q < 6; q++) mat[q] = 0.;
  double Kp = 0.;
  if (deck->law == PDGPU_MAT_RNP || deck->law == PDGPU_MAT_PMB || deck->law == PDGPU_MAT_PDELASTIC) {
    // bond-based laws fix Poisson's ratio at 1/4
    nu = 0.25;
    if (E > 0.) K = toK(E, nu);
    if (K > 0. && E < 0.) E = K * (3. * (1. - 2. * nu));
    const double lam = toLambdaE(E, nu);
    const double M = moment(inf_type, inf_params, dim);
    if (deck->law == PDGPU_MAT_RNP) {
      double C, beta, inv;
      if (dim == 2) {
        C = M_PI * Gc / (4. * M);
        beta = 4. * lam / (C * M);
        inv = std::pow(horizon, 3) * M_PI;
      } else {
        C = 2. * Gc / (3. * M);
        beta = 5. * lam / (C * M);
        inv = std::pow(horizon, 4) * 4. * M_PI / 3.;
      }
      mat[0] = C;
      mat[1] = beta;
      mat[2] = std::sqrt(0.5 / beta);
      mat[3] = inv;
      mat[4] = deck->check_sc_factor;
      mat[5] = deck->irreversible ? 1. : 0.;
      const double lam2 = dim == 2 ? C * M * beta / 4. : C * M * beta / 5.;
      Kp = toK(toELambda(lam2, 0.25), 0.25);
    } else if (deck->law == PDGPU_MAT_PMB) {
      double c;
      if (dim == 2)
        c = 24.0 * E / (M_PI * std::pow(horizon, 3.0) * (1. - nu));
      else
        c = 24.0 * lam / (M_PI * std::pow(horizon, 3.0));
      mat[0] = c;
      mat[1] = std::sqrt(5.0 * M_PI * Gc / (9.0 * E * horizon));
      const double lam2 = c * (M_PI * std::pow(horizon, 3.0)) / 24.0;
      Kp = toK(toELambda(lam2, 0.25), 0.25);
    } else {
      const double c = 24.0 * lam / (M_PI * std::pow(horizon, 3.0));
      mat[0] = c;
      const double lam2 = c * (M_PI * std::pow(horizon, 3.0)) / 24.0;
      Kp = toK(toELambda(lam2, 0.25), 0.25);
    }
  } else if (deck->law == PDGPU_MAT_PDSTATE) {
    // exactly two of E, K, G, nu given
    const bool fE = E > 0, fK = K > 0, fG = G > 0, fnu = nu > 0;
    if (!fnu) {
      if (fE && fG) nu = (0.5 * E / G) - 1.;
      if (fE && fK) nu = (3. * K - E) / (6. * K);
      if (fG && fK) nu = (3. * K - 2. * G) / (2. * (3. * K + G));
    }
    if (!fE) {
      if (fK) E = K * (3. * (1. - 2. * nu));
      if (fG) E = 2. * G * (1. + nu);
    }
    if (!fK) K = toK(E, nu);
    if (!fG) G = toGE(E, nu);
    const double dd = (3. * G + std::pow(3. / 4., 4) * (K - 5. * G / 3.)) * horizon;
    mat[0] = K;
    mat[1] = G;
    mat[2] = std::sqrt(Gc / dd);
    Kp = K;
  } else {
    return PDGPU_ERR_ARG;
  }
  if (bulk_modulus) *bulk_modulus = Kp;
  return PDGPU_OK;
}

}  // extern "C"
