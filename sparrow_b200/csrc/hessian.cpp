#include "hessian.h"

#include <algorithm>
#include <cmath>

#include "params.h"

namespace sgb {

namespace {

// Device bytes of one displaced copy of the molecule in a batch (pair data,
// N x N matrices, DIIS rings; an upper estimate).
size_t bytes_per_copy(const HessianRequest& req, int nao) {
  const size_t nat = req.molecule.Z.size();
  const size_t npairs = nat * (nat - 1) / 2;
  const size_t mats = (req.unrestricted ? 12 : 8) + (req.unrestricted ? 4 : 2) * (size_t)kDiisMax;
  const size_t dftb = is_dftb(req.method) ? 3 : 0;
  return 8 * (npairs * 180 + (size_t)nao * nao * (mats + dftb)) + 4096;
}

}  // namespace

int numerical_hessian(const HessianRequest& req, std::vector<double>& H, int& not_converged, std::string& err) {
  const MoleculeInput& mol = req.molecule;
  const int nat = (int)mol.Z.size();
  if (nat == 0) {
    err = "empty molecular structure";
    return kErrEmptyStructure;
  }
  if (!(req.step > 0) || req.step > 0.5) {
    err = "the Hessian displacement must lie in (0, 0.5] bohr";
    return kErrInvalidArgument;
  }
  const int n3 = 3 * nat;
  // AO count for the memory estimate (elements are validated by setup)
  int nao = 0;
  for (int z : mol.Z) nao += std::max(1, z == 1 ? 1 : 4);
  const size_t per_copy = bytes_per_copy(req, nao);
  const int chunk = (int)std::max<size_t>(2, std::min<size_t>((size_t)2 * n3, req.device_budget_bytes / per_copy) & ~size_t(1));

  Batch batch(req.method);
  batch.set_parameters(req.parameters);
  batch.set_unrestricted(req.unrestricted);
  H.assign((size_t)n3 * n3, 0.0);
  not_converged = 0;
  std::vector<MoleculeInput> copies;
  std::vector<MoleculeOutput> out;
  // displacement k of coordinate c = k / 2, sign + for even k
  for (int k0 = 0; k0 < 2 * n3; k0 += chunk) {
    const int k1 = std::min(2 * n3, k0 + chunk);
    copies.assign(k1 - k0, mol);
    for (int k = k0; k < k1; ++k) copies[k - k0].xyz[k / 2] += (k & 1) ? -req.step : req.step;
    int rc = batch.setup(copies, err);
    if (rc) return rc;
    rc = batch.run(req.scf, true, err);
    if (rc) return rc;
    rc = batch.fetch(out, true, err);
    if (rc) return rc;
    for (int k = k0; k < k1; ++k) {
      const MoleculeOutput& o = out[k - k0];
      if (o.status != 0) {
        err = "device SCF failure at displacement " + std::to_string(k);
        return kErrDevice;
      }
      if (!o.converged) ++not_converged;
      const double s = ((k & 1) ? -1.0 : 1.0) / (2.0 * req.step);
      double* row = H.data() + (size_t)(k / 2) * n3;
      for (int j = 0; j < n3; ++j) row[j] += s * o.gradient[j];
    }
  }
  for (int i = 0; i < n3; ++i)
    for (int j = i + 1; j < n3; ++j) {
      const double v = 0.5 * (H[(size_t)i * n3 + j] + H[(size_t)j * n3 + i]);
      H[(size_t)i * n3 + j] = H[(size_t)j * n3 + i] = v;
    }
  return kOk;
}

}  // namespace sgb
