// Semi-numerical Hessian: central differences of analytic gradients, the
// reference's only Hessian (GenericMethodWrapper::calculate falls back to
// Utils::NumericalHessianCalculator because canCalculateAnalyticalHessian()
// is false: src/Sparrow/Sparrow/Implementations/GenericMethodWrapper.cpp:58-88,
// 339-341).  The 6 N displaced geometries are independent molecules, so they
// run as batches through the batched SCF and gradient kernels: one launch
// sequence per batch instead of 6 N serial single points.
#pragma once
#include <string>
#include <vector>

#include "engine.h"

namespace sgb {

// Displacement of the reference's numerical Hessian (bohr).
constexpr double kHessianStep = 1e-2;

struct HessianRequest {
  Method method = kPM6;
  std::string parameters;  // as Batch::set_parameters
  bool unrestricted = false;
  MoleculeInput molecule;
  ScfParams scf;
  double step = kHessianStep;
  size_t device_budget_bytes = 16ull << 30;  // per batch of displaced geometries
};

// H[i][j] = (g_j(x + h e_i) - g_j(x - h e_i)) / 2h, then (H + H^T) / 2
// (Hartree/bohr^2, 3 n_atoms x 3 n_atoms row-major).  not_converged counts
// displaced geometries whose SCF did not converge (their gradients are still
// used, as the reference does).
int numerical_hessian(const HessianRequest& req, std::vector<double>& H, int& not_converged, std::string& err);

}  // namespace sgb
