// C-ABI and the C++ Calculator facade (see include/sparrow_b200.h).
//
// Calculator mirrors the reference's GenericMethodWrapper behaviour
// (src/Sparrow/Sparrow/Implementations/GenericMethodWrapper.cpp:58-282):
// settings are applied at calculate(), results are invalidated by a new
// structure or new positions, non-convergence is reported but the energy is
// still returned, and the state is the density matrix.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/sparrow_b200.h"
#include "dftb_params.h"
#include "engine.h"
#include "hessian.h"
#include "params.h"
#include "server.h"

namespace sgb {

// "METHOD" or "METHOD:parameters": for DFTB an embedded set name or a
// directory of Slater-Koster files (e.g. "DFTB3:3ob-2-1"), for NDDO the path
// of a parameters.json file (e.g. "PM6:/data/pm6-refit.json").
bool parse_method_spec(const char* spec, Method& m, std::string& set) {
  std::string s(spec);
  const size_t c = s.find(':');
  set.clear();
  if (c != std::string::npos) {
    set = s.substr(c + 1);
    s = s.substr(0, c);
  }
  return parse_method(s, m);
}

struct Settings {
  int charge = 0;
  int multiplicity = 1;
  std::string spin_mode = "any";
  double scc = 1e-7;
  double rmsd = 1e-5;
  int max_iter = 100;
  std::string mixer = "diis";
  std::string parameters;
  std::string scf_path = "auto";  // auto | batched | large | large_mixed
};

class Calculator {
 public:
  explicit Calculator(Method m) : method_(m), batch_(new Batch(m)) {}
  Method method() const { return method_; }
  Settings& settings() { return settings_; }
  const Settings& settings() const { return settings_; }
  std::string error;

  int set_structure(int n, const int* Z, const double* xyz) {
    if (n <= 0 || !Z || !xyz) {
      error = "empty molecular structure";
      return kErrEmptyStructure;
    }
    Z_.assign(Z, Z + n);
    xyz_.assign(xyz, xyz + 3 * n);
    invalidate(true);
    return kOk;
  }
  int modify_positions(const double* xyz) {
    if (Z_.empty()) {
      error = "no structure set";
      return kErrEmptyStructure;
    }
    xyz_.assign(xyz, xyz + xyz_.size());
    invalidate(false);
    return kOk;
  }
  int n_atoms() const { return (int)Z_.size(); }
  const std::vector<double>& positions() const { return xyz_; }
  void set_required(uint32_t mask) { required_ = mask; }

  int calculate() {
    if (Z_.empty()) {
      error = "empty molecular structure";
      return kErrEmptyStructure;
    }
    // DFTB: an embedded set name or a Slater-Koster directory; NDDO: a
    // parameters.json path; empty = the method's embedded default
    batch_->set_parameters(settings_.parameters);
    // spin mode as the reference's NDDOMethodWrapper::applySettings
    // (Implementations/Nddo/NDDOMethodWrapper.cpp:68-92): "any" is unrestricted
    // for multiplicities other than 1
    if (settings_.spin_mode == "restricted_open_shell") {
      error = "restricted open-shell SCF is not supported (use unrestricted)";
      return kErrInvalidArgument;
    }
    const bool uhf = settings_.spin_mode == "unrestricted" ||
                     (settings_.spin_mode == "any" && settings_.multiplicity != 1);
    if (!uhf && settings_.multiplicity != 1) {
      error = "a restricted calculation needs spin multiplicity 1";
      return kErrInvalidArgument;
    }
    batch_->set_unrestricted(uhf);
    ScfParams sp;
    sp.scc = settings_.scc;
    sp.rmsd = settings_.rmsd;
    sp.max_iter = settings_.max_iter;
    sp.diis_size = settings_.mixer == "diis" ? kDiisMax : 1;
    sp.canonical = 1;  // results report orbital energies
    std::vector<MoleculeInput> in(1);
    in[0].Z = Z_;
    in[0].xyz = xyz_;
    in[0].charge = settings_.charge;
    in[0].multiplicity = settings_.multiplicity;
    int rc = batch_->setup(in, error);
    if (rc) return rc;
    const std::string& sp_name = settings_.scf_path;
    rc = batch_->set_scf_path(sp_name == "batched" ? 1 : sp_name == "large" ? 2 : sp_name == "large_mixed" ? 3 : 0,
                              error);
    if (rc) return rc;
    if (uhf && !state_a_.empty()) {
      rc = batch_->set_start_spin_densities(state_a_.data(), state_b_.data(), error);
      if (rc) return rc;
    } else if (!state_.empty()) {
      rc = batch_->set_start_density(state_.data(), error);
      if (rc) return rc;
    }
    const bool grad = (required_ & SG_PROP_GRADIENTS) != 0;
    rc = batch_->run(sp, grad, error);
    if (rc) return rc;
    std::vector<MoleculeOutput> out;
    rc = batch_->fetch(out, grad, error);
    if (rc) return rc;
    result_ = out[0];
    have_result_ = true;
    have_gradient_ = grad;
    batch_->fetch_density(0, density_, error);
    eps_.clear();  // stays empty on the large-molecule path, which has no orbitals
    batch_->fetch_orbital_energies(0, eps_, error);
    charges_.clear();
    if (required_ & SG_PROP_ATOMIC_CHARGES) batch_->fetch_charges(0, charges_, error);
    dipole_.clear();
    if (required_ & SG_PROP_DIPOLE) {
      dipole_.resize(3);
      batch_->dipole(0, dipole_.data(), error);
    }
    eps_b_.clear();
    dens_a_.clear();
    dens_b_.clear();
    if (uhf) {
      batch_->fetch_orbital_energies(0, eps_b_, error, true);
      batch_->fetch_spin_densities(0, dens_a_, dens_b_, error);
    }
    if (result_.status != kDevOk) {
      error = "device SCF failure code " + std::to_string(result_.status);
      return kErrDevice;
    }
    hessian_.clear();
    if (required_ & SG_PROP_HESSIAN) {
      // semi-numerical, as the reference (GenericMethodWrapper.cpp:76-88)
      HessianRequest hr;
      hr.method = method_;
      hr.parameters = settings_.parameters;
      hr.unrestricted = uhf;
      hr.molecule = in[0];
      hr.scf = sp;
      int unconverged = 0;
      rc = numerical_hessian(hr, hessian_, unconverged, error);
      if (rc) return rc;
    }
    if (!result_.converged) {
      error = "SCF did not converge in " + std::to_string(result_.iterations) + " iterations";
      return kErrNotConverged;
    }
    return kOk;
  }
  const std::vector<double>& hessian() const { return hessian_; }
  const std::vector<double>& atomic_charges() const { return charges_; }
  const std::vector<double>& dipole() const { return dipole_; }
  const std::vector<double>& alpha_density() const { return dens_a_; }
  const std::vector<double>& beta_density() const { return dens_b_; }
  int set_spin_densities(const double* Pa, const double* Pb) {
    const int n = n_aos();
    if (n == 0) {
      error = "no structure set";
      return kErrEmptyStructure;
    }
    state_a_.assign(Pa, Pa + (size_t)n * n);
    state_b_.assign(Pb, Pb + (size_t)n * n);
    state_.resize((size_t)n * n);
    for (size_t k = 0; k < state_.size(); ++k) state_[k] = state_a_[k] + state_b_[k];
    return kOk;
  }

  // TD-DFTB on the converged DFTB reference of the last calculate()
  int excitations(int nroots, bool triplet, double* omega, double* dip) {
    if (!have_result_ || !result_.converged) {
      error = "TD-DFTB needs a converged reference calculation";
      return kErrNoResults;
    }
    int rc = batch_->run_tddftb(nroots, triplet, kTddftbResidual, kTddftbMaxIter, error);
    if (rc) return rc;
    std::vector<double> om, dp;
    std::vector<int> info;
    rc = batch_->fetch_tddftb(om, dp, info, error);
    if (rc) return rc;
    std::memcpy(omega, om.data(), sizeof(double) * om.size());
    if (dip) std::memcpy(dip, dp.data(), sizeof(double) * dp.size());
    return td_status(info[1], error);
  }
  static int td_status(int st, std::string& error) {
    if (st == 0) return kOk;
    if (st == 1) {
      error = "TD-DFTB Davidson did not converge";
      return kErrNotConverged;
    }
    error = "TD-DFTB device failure code " + std::to_string(st);
    return kErrDevice;
  }

  bool have_result() const { return have_result_; }
  bool have_gradient() const { return have_gradient_; }
  const MoleculeOutput& result() const { return result_; }
  const std::vector<double>& density() const { return density_; }
  const std::vector<double>& orbital_energies() const { return eps_; }
  const std::vector<double>& beta_orbital_energies() const { return eps_b_; }
  int set_density(const double* P) {
    if (Z_.empty()) {
      error = "no structure set";
      return kErrEmptyStructure;
    }
    int n = 0;
    for (int z : Z_) {
      int k = aos_of(z);
      if (!k) {
        error = "unsupported element";
        return kErrUnsupportedElement;
      }
      n += k;
    }
    state_.assign(P, P + (size_t)n * n);
    return kOk;
  }
  int n_aos() const {
    int n = 0;
    for (int z : Z_) n += aos_of(z);
    return n;
  }
  // AOs of element Z under the current parameter source
  int aos_of(int z) const {
    const std::string& src = settings_.parameters;
    if (is_dftb(method_)) return dftb_n_aos(src.empty() ? dftb_default_set(method_) : src.c_str(), z);
    std::string unused;
    auto set = src.empty() ? nullptr : nddo_parameter_set(method_, src, unused);
    return engine_n_aos(method_, z, set.get());
  }
  std::unique_ptr<Calculator> clone() const {
    std::unique_ptr<Calculator> c(new Calculator(method_));
    c->settings_ = settings_;
    c->Z_ = Z_;
    c->xyz_ = xyz_;
    c->required_ = required_;
    return c;
  }

 private:
  void invalidate(bool new_structure) {
    have_result_ = have_gradient_ = false;
    hessian_.clear();
    if (new_structure) state_a_.clear(), state_b_.clear();
    if (new_structure) state_.clear();
  }
  Method method_;
  Settings settings_;
  std::unique_ptr<Batch> batch_;
  std::vector<int> Z_;
  std::vector<double> xyz_;
  uint32_t required_ = SG_PROP_ENERGY;
  MoleculeOutput result_;
  bool have_result_ = false, have_gradient_ = false;
  std::vector<double> density_, eps_, eps_b_, state_, hessian_, charges_, dipole_;
  std::vector<double> dens_a_, dens_b_, state_a_, state_b_;  // unrestricted: spin densities and their start
};

}  // namespace sgb

using namespace sgb;

struct sg_calculator {
  std::unique_ptr<Calculator> impl;
};

struct sg_batch {
  std::unique_ptr<Batch> impl;
  ScfParams sp;
  uint32_t props = SG_PROP_ENERGY;
  std::string error;
};

namespace {
thread_local std::string g_create_error;

int32_t fail(sg_calculator* h, int32_t code, const std::string& msg) {
  if (h) h->impl->error = msg;
  return code;
}

bool read_molecules(int32_t n_mol, const int32_t* n_atoms, const int32_t* Z, const double* xyz,
                    const int32_t* charges, std::vector<MoleculeInput>& mols, std::string& err) {
  if (n_mol <= 0 || !n_atoms || !Z || !xyz) {
    err = "empty batch";
    return false;
  }
  mols.resize(n_mol);
  size_t a = 0;
  for (int i = 0; i < n_mol; ++i) {
    if (n_atoms[i] <= 0) {
      err = "molecule " + std::to_string(i) + " has no atoms";
      return false;
    }
    mols[i].Z.assign(Z + a, Z + a + n_atoms[i]);
    mols[i].xyz.assign(xyz + 3 * a, xyz + 3 * (a + n_atoms[i]));
    mols[i].charge = charges ? charges[i] : 0;
    a += n_atoms[i];
  }
  return true;
}
}  // namespace

extern "C" {

const char* sg_version(void) { return "sparrow_b200 0.1 (NDDO MNDO/AM1/PM6, s/p elements, sm_100a)"; }

int32_t sg_create(const char* method, sg_calculator** out) {
  if (!out) return SG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  Method m;
  if (!method || !parse_method(method, m)) {
    g_create_error = std::string("unknown method '") + (method ? method : "") + "' (PM6, AM1, MNDO)";
    return SG_ERR_UNKNOWN_METHOD;
  }
  *out = new sg_calculator{std::unique_ptr<Calculator>(new Calculator(m))};
  return SG_OK;
}

void sg_destroy(sg_calculator* h) { delete h; }

int32_t sg_clone(const sg_calculator* h, sg_calculator** out) {
  if (!h || !out) return SG_ERR_INVALID_ARGUMENT;
  *out = new sg_calculator{h->impl->clone()};
  return SG_OK;
}

const char* sg_last_error(const sg_calculator* h) { return h ? h->impl->error.c_str() : g_create_error.c_str(); }

int32_t sg_set_structure(sg_calculator* h, int32_t n, const int32_t* Z, const double* xyz) {
  if (!h) return SG_ERR_INVALID_ARGUMENT;
  return h->impl->set_structure(n, Z, xyz);
}

int32_t sg_modify_positions(sg_calculator* h, const double* xyz) {
  if (!h || !xyz) return SG_ERR_INVALID_ARGUMENT;
  return h->impl->modify_positions(xyz);
}

int32_t sg_get_positions(const sg_calculator* h, double* xyz) {
  if (!h || !xyz) return SG_ERR_INVALID_ARGUMENT;
  const auto& p = h->impl->positions();
  std::memcpy(xyz, p.data(), sizeof(double) * p.size());
  return SG_OK;
}

int32_t sg_get_n_atoms(const sg_calculator* h, int32_t* n) {
  if (!h || !n) return SG_ERR_INVALID_ARGUMENT;
  *n = h->impl->n_atoms();
  return SG_OK;
}

int32_t sg_set_setting_int(sg_calculator* h, const char* key, int64_t v) {
  if (!h || !key) return SG_ERR_INVALID_ARGUMENT;
  Settings& s = h->impl->settings();
  std::string k(key);
  if (k == "molecular_charge") s.charge = (int)v;
  else if (k == "spin_multiplicity") {
    if (v < 1) return fail(h, SG_ERR_INVALID_ARGUMENT, "spin_multiplicity must be >= 1");
    s.multiplicity = (int)v;
  } else if (k == "max_scf_iterations") {
    if (v < 1) return fail(h, SG_ERR_INVALID_ARGUMENT, "max_scf_iterations must be >= 1");
    s.max_iter = (int)v;
  } else
    return fail(h, SG_ERR_UNKNOWN_SETTING, "unknown integer setting '" + k + "'");
  return SG_OK;
}

int32_t sg_set_setting_double(sg_calculator* h, const char* key, double v) {
  if (!h || !key) return SG_ERR_INVALID_ARGUMENT;
  Settings& s = h->impl->settings();
  std::string k(key);
  if (!(v > 0) || !std::isfinite(v)) return fail(h, SG_ERR_INVALID_ARGUMENT, k + " must be a positive number");
  if (k == "self_consistence_criterion") s.scc = v;
  else if (k == "density_rmsd_criterion") s.rmsd = v;
  else
    return fail(h, SG_ERR_UNKNOWN_SETTING, "unknown real setting '" + k + "'");
  return SG_OK;
}

int32_t sg_set_setting_string(sg_calculator* h, const char* key, const char* v) {
  if (!h || !key || !v) return SG_ERR_INVALID_ARGUMENT;
  Settings& s = h->impl->settings();
  std::string k(key), val(v);
  if (k == "spin_mode") {
    if (val != "any" && val != "restricted" && val != "unrestricted" && val != "restricted_open_shell")
      return fail(h, SG_ERR_INVALID_ARGUMENT, "unknown spin_mode '" + val + "'");
    s.spin_mode = val;
  } else if (k == "scf_mixer") {
    if (val != "diis" && val != "no_mixer" && val != "none")
      return fail(h, SG_ERR_INVALID_ARGUMENT, "unsupported scf_mixer '" + val + "' (diis, no_mixer)");
    s.mixer = val == "diis" ? "diis" : "none";
  } else if (k == "method_parameters") {
    s.parameters = val;
  } else if (k == "scf_path") {
    if (val != "auto" && val != "batched" && val != "large" && val != "large_mixed")
      return fail(h, SG_ERR_INVALID_ARGUMENT, "unknown scf_path '" + val + "' (auto, batched, large, large_mixed)");
    s.scf_path = val;
  } else
    return fail(h, SG_ERR_UNKNOWN_SETTING, "unknown string setting '" + k + "'");
  return SG_OK;
}

int32_t sg_get_setting_double(const sg_calculator* h, const char* key, double* v) {
  if (!h || !key || !v) return SG_ERR_INVALID_ARGUMENT;
  const Settings& s = h->impl->settings();
  std::string k(key);
  if (k == "self_consistence_criterion") *v = s.scc;
  else if (k == "density_rmsd_criterion") *v = s.rmsd;
  else
    return SG_ERR_UNKNOWN_SETTING;
  return SG_OK;
}

int32_t sg_get_setting_int(const sg_calculator* h, const char* key, int64_t* v) {
  if (!h || !key || !v) return SG_ERR_INVALID_ARGUMENT;
  const Settings& s = h->impl->settings();
  std::string k(key);
  if (k == "molecular_charge") *v = s.charge;
  else if (k == "spin_multiplicity") *v = s.multiplicity;
  else if (k == "max_scf_iterations") *v = s.max_iter;
  else
    return SG_ERR_UNKNOWN_SETTING;
  return SG_OK;
}

int32_t sg_set_required_properties(sg_calculator* h, uint32_t mask) {
  if (!h) return SG_ERR_INVALID_ARGUMENT;
  if (mask & ~(SG_PROP_ENERGY | SG_PROP_GRADIENTS | SG_PROP_HESSIAN | SG_PROP_ATOMIC_CHARGES | SG_PROP_DIPOLE))
    return fail(h, SG_ERR_INVALID_ARGUMENT, "unknown property bit");
  h->impl->set_required(mask);
  return SG_OK;
}

int32_t sg_calculate(sg_calculator* h) {
  if (!h) return SG_ERR_INVALID_ARGUMENT;
  return h->impl->calculate();
}

int32_t sg_get_energy(const sg_calculator* h, double* e) {
  if (!h || !e) return SG_ERR_INVALID_ARGUMENT;
  if (!h->impl->have_result()) return SG_ERR_NO_RESULTS;
  *e = h->impl->result().energy;
  return SG_OK;
}

int32_t sg_get_gradients(const sg_calculator* h, double* g) {
  if (!h || !g) return SG_ERR_INVALID_ARGUMENT;
  if (!h->impl->have_result() || !h->impl->have_gradient()) return SG_ERR_NO_RESULTS;
  const auto& v = h->impl->result().gradient;
  std::memcpy(g, v.data(), sizeof(double) * v.size());
  return SG_OK;
}

int32_t sg_get_spin_densities(const sg_calculator* h, double* Pa, double* Pb) {
  if (!h || !Pa || !Pb) return SG_ERR_INVALID_ARGUMENT;
  const auto& a = h->impl->alpha_density();
  const auto& b = h->impl->beta_density();
  if (!h->impl->have_result() || a.empty()) return SG_ERR_NO_RESULTS;
  std::memcpy(Pa, a.data(), sizeof(double) * a.size());
  std::memcpy(Pb, b.data(), sizeof(double) * b.size());
  return SG_OK;
}

int32_t sg_set_spin_densities(sg_calculator* h, const double* Pa, const double* Pb) {
  if (!h || !Pa || !Pb) return SG_ERR_INVALID_ARGUMENT;
  return h->impl->set_spin_densities(Pa, Pb);
}

int32_t sg_get_dipole(const sg_calculator* h, double* dipole3) {
  if (!h || !dipole3) return SG_ERR_INVALID_ARGUMENT;
  const auto& v = h->impl->dipole();
  if (!h->impl->have_result() || v.size() != 3) return SG_ERR_NO_RESULTS;
  std::memcpy(dipole3, v.data(), 3 * sizeof(double));
  return SG_OK;
}

int32_t sg_get_atomic_charges(const sg_calculator* h, double* charges) {
  if (!h || !charges) return SG_ERR_INVALID_ARGUMENT;
  const auto& v = h->impl->atomic_charges();
  if (!h->impl->have_result() || v.empty()) return SG_ERR_NO_RESULTS;
  std::memcpy(charges, v.data(), sizeof(double) * v.size());
  return SG_OK;
}

int32_t sg_get_hessian(const sg_calculator* h, double* hessian) {
  if (!h || !hessian) return SG_ERR_INVALID_ARGUMENT;
  const auto& v = h->impl->hessian();
  if (!h->impl->have_result() || v.empty()) return SG_ERR_NO_RESULTS;
  std::memcpy(hessian, v.data(), sizeof(double) * v.size());
  return SG_OK;
}

int32_t sg_get_scf_info(const sg_calculator* h, int32_t* it, int32_t* conv, int32_t* nao, int32_t* nocc) {
  if (!h) return SG_ERR_INVALID_ARGUMENT;
  if (!h->impl->have_result()) return SG_ERR_NO_RESULTS;
  const auto& r = h->impl->result();
  if (it) *it = r.iterations;
  if (conv) *conv = r.converged;
  if (nao) *nao = r.nao;
  if (nocc) *nocc = r.nocc;
  return SG_OK;
}

int32_t sg_get_orbital_energies(const sg_calculator* h, double* eps) {
  if (!h || !eps) return SG_ERR_INVALID_ARGUMENT;
  const auto& v = h->impl->orbital_energies();
  if (!h->impl->have_result() || v.empty()) return SG_ERR_NO_RESULTS;  // none on the large-molecule path
  std::memcpy(eps, v.data(), sizeof(double) * v.size());
  return SG_OK;
}

int32_t sg_get_beta_orbital_energies(const sg_calculator* h, double* eps) {
  if (!h || !eps) return SG_ERR_INVALID_ARGUMENT;
  if (!h->impl->have_result()) return SG_ERR_NO_RESULTS;
  const auto& v = h->impl->beta_orbital_energies();
  if (v.empty()) return SG_ERR_NO_RESULTS;  // restricted calculation
  std::memcpy(eps, v.data(), sizeof(double) * v.size());
  return SG_OK;
}

int32_t sg_calculate_excitations(sg_calculator* h, int32_t nroots, int32_t triplet, double* omega, double* dipoles) {
  if (!h || !omega) return SG_ERR_INVALID_ARGUMENT;
  return h->impl->excitations(nroots, triplet != 0, omega, dipoles);
}

int32_t sg_get_density(const sg_calculator* h, double* P) {
  if (!h || !P) return SG_ERR_INVALID_ARGUMENT;
  if (!h->impl->have_result()) return SG_ERR_NO_RESULTS;
  const auto& v = h->impl->density();
  std::memcpy(P, v.data(), sizeof(double) * v.size());
  return SG_OK;
}

int32_t sg_set_density(sg_calculator* h, const double* P) {
  if (!h || !P) return SG_ERR_INVALID_ARGUMENT;
  return h->impl->set_density(P);
}

namespace {

int32_t batch_create(const char* method, int32_t n_mol, const int32_t* n_atoms, const int32_t* Z, const double* xyz,
                     const int32_t* charges, const int32_t* multiplicities, bool uhf, sg_batch** out) {
  if (!out) return SG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  Method m;
  std::string set;
  if (!method || !parse_method_spec(method, m, set)) {
    g_create_error = "unknown method";
    return SG_ERR_UNKNOWN_METHOD;
  }
  std::vector<MoleculeInput> mols;
  std::string err;
  if (!read_molecules(n_mol, n_atoms, Z, xyz, charges, mols, err)) {
    g_create_error = err;
    return SG_ERR_EMPTY_STRUCTURE;
  }
  if (multiplicities)
    for (int i = 0; i < n_mol; ++i) mols[i].multiplicity = multiplicities[i];
  std::unique_ptr<sg_batch> b(new sg_batch);
  b->impl.reset(new Batch(m));
  b->impl->set_parameters(set);
  b->impl->set_unrestricted(uhf);
  int rc = b->impl->setup(mols, err);
  if (rc) {
    g_create_error = err;
    return rc;
  }
  *out = b.release();
  return SG_OK;
}

}  // namespace

int32_t sg_batch_create(const char* method, int32_t n_mol, const int32_t* n_atoms, const int32_t* Z,
                        const double* xyz, const int32_t* charges, sg_batch** out) {
  return batch_create(method, n_mol, n_atoms, Z, xyz, charges, nullptr, false, out);
}

int32_t sg_batch_create_unrestricted(const char* method, int32_t n_mol, const int32_t* n_atoms, const int32_t* Z,
                                     const double* xyz, const int32_t* charges, const int32_t* multiplicities,
                                     sg_batch** out) {
  return batch_create(method, n_mol, n_atoms, Z, xyz, charges, multiplicities, true, out);
}

void sg_batch_destroy(sg_batch* b) { delete b; }

const char* sg_batch_last_error(const sg_batch* b) { return b ? b->error.c_str() : g_create_error.c_str(); }

int32_t sg_batch_set_scf(sg_batch* b, double scc, double rmsd, int32_t max_iter) {
  if (!b || !(scc > 0) || !(rmsd > 0) || max_iter < 1) return SG_ERR_INVALID_ARGUMENT;
  b->sp.scc = scc;
  b->sp.rmsd = rmsd;
  b->sp.max_iter = max_iter;
  return SG_OK;
}

int32_t sg_batch_set_scf_path(sg_batch* b, int32_t path) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  return b->impl->set_scf_path(path, b->error);
}

int32_t sg_batch_set_mixed_switch(sg_batch* b, double rmsd) {
  if (!b || !(rmsd > 0) || !std::isfinite(rmsd)) return SG_ERR_INVALID_ARGUMENT;
  b->sp.mixed_switch_rmsd = rmsd;
  return SG_OK;
}

int32_t sg_batch_set_tuning(sg_batch* b, int32_t orbital_update, int32_t diis_size) {
  const bool mode_ok = orbital_update == -1 || orbital_update == kEigExact || orbital_update == kEigHybrid ||
                       orbital_update == kEigRotation;
  if (!b || !mode_ok || diis_size == 0 || diis_size < -1 || diis_size > kDiisMax) return SG_ERR_INVALID_ARGUMENT;
  const ScfParams tuned;
  for (int k = 0; k < kTuneBins; ++k) {
    b->sp.eig_mode_bin[k] = (signed char)(orbital_update >= 0 ? orbital_update : tuned.eig_mode_bin[k]);
    b->sp.diis_bin[k] = (signed char)(diis_size > 0 ? diis_size : tuned.diis_bin[k]);
  }
  return SG_OK;
}

int32_t sg_tuning_table(int32_t* orbital_update, int32_t* diis_size, int32_t capacity) {
  if (capacity < 0 || (capacity > 0 && (!orbital_update || !diis_size))) return -SG_ERR_INVALID_ARGUMENT;
  const ScfParams tuned;
  for (int k = 0; k < kTuneBins && k < capacity; ++k) {
    orbital_update[k] = tuned.eig_mode_bin[k];
    diis_size[k] = tuned.diis_bin[k];
  }
  return kTuneBins;
}

int32_t sg_batch_excitations(sg_batch* b, int32_t nroots, int32_t triplet, double* omega, double* dipoles,
                             int32_t* status) {
  if (!b || !omega) return SG_ERR_INVALID_ARGUMENT;
  int rc = b->impl->run_tddftb(nroots, triplet != 0, kTddftbResidual, kTddftbMaxIter, b->error);
  if (rc) return rc;
  std::vector<double> om, dp;
  std::vector<int> info;
  rc = b->impl->fetch_tddftb(om, dp, info, b->error);
  if (rc) return rc;
  std::memcpy(omega, om.data(), sizeof(double) * om.size());
  if (dipoles) std::memcpy(dipoles, dp.data(), sizeof(double) * dp.size());
  // per-molecule outcomes go to status; the return code is the worst of them,
  // a reference that did not converge counting as not converged
  int failed = 0, unconverged = 0;
  for (size_t i = 0; i < info.size() / 2; ++i) {
    const int st = info[2 * i + 1];
    if (status) status[i] = st;
    if (st == 1 || st == 4) ++unconverged;
    else if (st != 0) ++failed;
  }
  if (failed) return Calculator::td_status(2, b->error);
  if (unconverged) {
    b->error = std::to_string(unconverged) + " molecule(s) without converged excitations (see status)";
    return SG_ERR_NOT_CONVERGED;
  }
  return SG_OK;
}

int32_t sg_batch_excitation_cycles(sg_batch* b, int64_t* cycles3) {
  if (!b || !cycles3) return SG_ERR_INVALID_ARGUMENT;
  std::vector<long long> c;
  const int rc = b->impl->fetch_tddftb_cycles(c, b->error);
  if (rc) return rc;
  for (size_t i = 0; i < c.size(); ++i) cycles3[i] = c[i];
  return SG_OK;
}

int32_t sg_batch_set_positions(sg_batch* b, const double* xyz) {
  if (!b || !xyz) return SG_ERR_INVALID_ARGUMENT;
  return b->impl->set_positions(xyz, b->error);
}

int32_t sg_batch_run(sg_batch* b, uint32_t props) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  b->props = props;
  return b->impl->run(b->sp, (props & SG_PROP_GRADIENTS) != 0, b->error);
}

int32_t sg_batch_results(sg_batch* b, double* energies, double* gradients, int32_t* iterations, int32_t* converged) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  const bool grad = gradients && (b->props & SG_PROP_GRADIENTS);
  std::vector<MoleculeOutput> out;
  int rc = b->impl->fetch(out, grad, b->error);
  if (rc) return rc;
  size_t a = 0;
  int status = SG_OK;
  for (size_t i = 0; i < out.size(); ++i) {
    if (energies) energies[i] = out[i].energy;
    if (iterations) iterations[i] = out[i].iterations;
    if (converged) converged[i] = out[i].converged;
    if (grad) {
      std::memcpy(gradients + 3 * a, out[i].gradient.data(), sizeof(double) * out[i].gradient.size());
      a += out[i].gradient.size() / 3;
    }
    if (out[i].status != kDevOk) status = SG_ERR_DEVICE;
    else if (!out[i].converged && status == SG_OK) status = SG_ERR_NOT_CONVERGED;
  }
  return status;
}

int32_t sg_batch_launches(const sg_batch* b) { return b ? b->impl->launches_last_run() : 0; }

void* sg_batch_stream(const sg_batch* b) { return b ? (void*)b->impl->stream() : nullptr; }

int32_t sg_batch_stage_times(sg_batch* b, double* ms4) {
  if (!b || !ms4) return SG_ERR_INVALID_ARGUMENT;
  return b->impl->stage_times(ms4, b->error);
}

int32_t sg_batch_record_event(sg_batch* b, int32_t slot) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  return b->impl->record_event(slot, b->error);
}

int32_t sg_batch_event_elapsed(sg_batch* b, int32_t s0, int32_t s1, double* ms) {
  if (!b || !ms) return SG_ERR_INVALID_ARGUMENT;
  return b->impl->event_elapsed(s0, s1, ms, b->error);
}

int32_t sg_batch_scf_stats(sg_batch* b, int32_t* nfull, int32_t* sweeps, int64_t* cycles5) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  std::vector<MolResult> r;
  int rc = b->impl->fetch_raw_results(r, b->error);
  if (rc) return rc;
  for (size_t i = 0; i < r.size(); ++i) {
    if (nfull) nfull[i] = r[i].full_diag;
    if (sweeps) sweeps[i] = r[i].jacobi_sweeps;
    if (cycles5)
      for (int k = 0; k < 5; ++k) cycles5[5 * i + k] = r[i].cycles[k];
  }
  return SG_OK;
}

int32_t sg_batch_convergence(sg_batch* b, double* last_delta_energy, double* last_rms_density_change) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  std::vector<MolResult> r;
  int rc = b->impl->fetch_raw_results(r, b->error);
  if (rc) return rc;
  for (size_t i = 0; i < r.size(); ++i) {
    if (last_delta_energy) last_delta_energy[i] = r[i].last_dE;
    if (last_rms_density_change) last_rms_density_change[i] = r[i].last_rmsd;
  }
  return SG_OK;
}

int32_t sg_batch_transfer_bytes(const sg_batch* b, int64_t* h2d, int64_t* d2h) {
  if (!b) return SG_ERR_INVALID_ARGUMENT;
  if (h2d) *h2d = b->impl->h2d_bytes();
  if (d2h) *d2h = b->impl->d2h_bytes();
  return SG_OK;
}

void sg_release_cached_memory(void) { release_cached_memory(); }

int32_t sg_batch_calculate(const char* method, int32_t n_mol, const int32_t* n_atoms, const int32_t* Z,
                           const double* xyz, const int32_t* charges, double scc, double rmsd, int32_t max_iter,
                           uint32_t props, double* energies, double* gradients, int32_t* iterations,
                           int32_t* converged, char* errmsg, int32_t errcap) {
  sg_batch* b = nullptr;
  int32_t rc = sg_batch_create(method, n_mol, n_atoms, Z, xyz, charges, &b);
  std::string err;
  if (rc == SG_OK) {
    rc = sg_batch_set_scf(b, scc, rmsd, max_iter);
    if (rc == SG_OK) rc = sg_batch_run(b, props);
    if (rc == SG_OK) rc = sg_batch_results(b, energies, gradients, iterations, converged);
    err = b->error;
    sg_batch_destroy(b);
  } else {
    err = g_create_error;
  }
  if (errmsg && errcap > 0) {
    std::strncpy(errmsg, err.c_str(), (size_t)errcap - 1);
    errmsg[errcap - 1] = 0;
  }
  return rc;
}

struct sg_server {
  std::unique_ptr<sgb::Server> impl;
};

namespace {
thread_local std::string g_server_error;

int32_t server_result(const sgb::ServerResult& r, double* energy, double* gradients, int32_t* iterations,
                      int32_t* status, double* latency_s) {
  if (energy) *energy = r.energy;
  if (gradients && !r.gradient.empty()) std::memcpy(gradients, r.gradient.data(), sizeof(double) * r.gradient.size());
  if (iterations) *iterations = r.iterations;
  if (status) *status = r.status;
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  g_server_error = r.error;
  return SG_OK;
}
}  // namespace

int32_t sg_server_create(uint64_t budget, int32_t slots, int32_t max_batch, double scc, double rmsd, int32_t max_iter,
                         sg_server** out) {
  if (!out) return SG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!(scc > 0) || !(rmsd > 0) || max_iter < 1 || slots < 1 || max_batch < 1) {
    g_server_error = "server settings must be positive";
    return SG_ERR_INVALID_ARGUMENT;
  }
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    g_server_error = "no CUDA device";
    return SG_ERR_CUDA;
  }
  sgb::ScfParams sp;
  sp.scc = scc;
  sp.rmsd = rmsd;
  sp.max_iter = max_iter;
  auto* s = new sg_server;
  s->impl.reset(new sgb::Server((size_t)budget, slots, max_batch, sp));
  *out = s;
  return SG_OK;
}

void sg_server_destroy(sg_server* s) { delete s; }

const char* sg_server_last_error(void) { return g_server_error.c_str(); }

int32_t sg_server_submit(sg_server* s, const char* method, int32_t n, const int32_t* Z, const double* xyz,
                         int32_t charge, uint32_t props, int64_t* id) {
  return sg_server_submit_spin(s, method, n, Z, xyz, charge, 1, props, id);
}

int32_t sg_server_submit_spin(sg_server* s, const char* method, int32_t n, const int32_t* Z, const double* xyz,
                              int32_t charge, int32_t multiplicity, uint32_t props, int64_t* id) {
  if (!s || !id) return SG_ERR_INVALID_ARGUMENT;
  sgb::Method m;
  std::string set;
  if (!method || !sgb::parse_method_spec(method, m, set) || !set.empty()) {
    g_server_error = std::string("unknown method '") + (method ? method : "") + "' (the server uses the default sets)";
    return SG_ERR_UNKNOWN_METHOD;
  }
  if (n <= 0 || !Z || !xyz) {
    g_server_error = "empty molecular structure";
    return SG_ERR_EMPTY_STRUCTURE;
  }
  sgb::MoleculeInput mol;
  mol.Z.assign(Z, Z + n);
  mol.xyz.assign(xyz, xyz + 3 * (size_t)n);
  mol.charge = charge;
  mol.multiplicity = multiplicity;
  std::string err;
  const long long r = s->impl->submit(m, std::move(mol), (props & SG_PROP_GRADIENTS) != 0, err);
  if (r < 0) {
    g_server_error = err;
    return (int32_t)(-r);
  }
  *id = r;
  return SG_OK;
}

int32_t sg_server_wait(sg_server* s, int64_t id, double timeout_s, double* energy, double* gradients,
                       int32_t* iterations, int32_t* status, double* latency_s) {
  if (!s) return SG_ERR_INVALID_ARGUMENT;
  sgb::ServerResult r;
  const int rc = s->impl->wait(id, r, timeout_s);
  if (rc == 1) return SG_ERR_TIMEOUT;
  if (rc != 0) {
    g_server_error = "unknown request id";
    return SG_ERR_INVALID_ARGUMENT;
  }
  return server_result(r, energy, gradients, iterations, status, latency_s);
}

int32_t sg_server_poll(sg_server* s, int64_t id, double* energy, double* gradients, int32_t* iterations,
                       int32_t* status, double* latency_s) {
  if (!s) return SG_ERR_INVALID_ARGUMENT;
  sgb::ServerResult r;
  const int rc = s->impl->poll(id, r);
  if (rc == 1) return SG_PENDING;
  if (rc != 0) {
    g_server_error = "unknown request id";
    return SG_ERR_INVALID_ARGUMENT;
  }
  return server_result(r, energy, gradients, iterations, status, latency_s);
}

int32_t sg_server_drain(sg_server* s) {
  if (!s) return SG_ERR_INVALID_ARGUMENT;
  s->impl->drain();
  return SG_OK;
}

int32_t sg_server_stats(sg_server* s, int64_t* submitted, int64_t* completed, int64_t* batches, int64_t* max_batch) {
  if (!s) return SG_ERR_INVALID_ARGUMENT;
  const sgb::ServerStats st = s->impl->stats();
  if (submitted) *submitted = st.submitted;
  if (completed) *completed = st.completed;
  if (batches) *batches = st.batches;
  if (max_batch) *max_batch = st.max_batch;
  return SG_OK;
}

}  // extern "C"

namespace {

void copy_message(const std::string& s, char* errmsg, int32_t errcap) {
  if (errmsg && errcap > 0) {
    std::strncpy(errmsg, s.c_str(), (size_t)errcap - 1);
    errmsg[errcap - 1] = 0;
  }
}

}  // namespace

int32_t sg_element_parameters(const char* method, int32_t Z, double* out, int32_t n_out, char* errmsg,
                              int32_t errcap) {
  using namespace sgb;
  Method m;
  std::string src;
  if (!method || !parse_method_spec(method, m, src)) {
    copy_message("unknown method", errmsg, errcap);
    return SG_ERR_UNKNOWN_METHOD;
  }
  if (!out || n_out < (is_dftb(m) ? SG_DFTB_ELEMENT_VALUES : SG_NDDO_ELEMENT_VALUES)) {
    copy_message("output buffer too small", errmsg, errcap);
    return SG_ERR_INVALID_ARGUMENT;
  }
  std::string err;
  if (is_dftb(m)) {
    const std::string set = src.empty() ? dftb_default_set(m) : src;
    if (!dftb_parameter_set(set, err)) {
      copy_message(err, errmsg, errcap);
      return SG_ERR_PARAMETERS;
    }
    DftbPrepared p;
    if (!dftb_prepare(set, m == kDFTB3 ? 3 : 2, {Z}, p, err)) {
      copy_message(err, errmsg, errcap);
      return SG_ERR_UNSUPPORTED_ELEMENT;
    }
    const DftbElemDev& e = p.elems[0];
    const double v[SG_DFTB_ELEMENT_VALUES] = {(double)e.nao, e.occ, e.es, e.ep, e.U, e.hd, e.w, (double)e.has_w};
    std::memcpy(out, v, sizeof(v));
    return SG_OK;
  }
  std::shared_ptr<const NddoParamSet> set;
  if (!src.empty()) {
    set = nddo_parameter_set(m, src, err);
    if (!set) {
      copy_message(err, errmsg, errcap);
      return SG_ERR_PARAMETERS;
    }
  }
  ElemDev e;
  if (!make_elem(m, Z, e, err, set.get())) {
    copy_message(err, errmsg, errcap);
    return SG_ERR_UNSUPPORTED_ELEMENT;
  }
  double* o = out;
  const double head[20] = {(double)e.nao, e.core, e.Uss, e.Upp,  e.betaS,  e.betaP,  e.alpha,
                           e.D[1],        e.D[3], e.rho[0], e.rho[1], e.rho[2], e.rho[3], e.pcore,
                           e.gss,         e.gsp,  e.gpp,  e.gp2,    e.hsp,    e.hpp};
  std::memcpy(o, head, sizeof(head));
  o += 20;
  for (const double* a : {e.s_exp, e.s_coef, e.p_exp, e.p_coef}) {
    std::memcpy(o, a, 6 * sizeof(double));
    o += 6;
  }
  *o++ = e.n_gauss;
  for (const double* a : {e.ga, e.gb, e.gc}) {
    std::memcpy(o, a, 4 * sizeof(double));
    o += 4;
  }
  return SG_OK;
}

int32_t sg_diatomic_parameters(const char* method, int32_t Z1, int32_t Z2, double* alpha_x, char* errmsg,
                               int32_t errcap) {
  using namespace sgb;
  Method m;
  std::string src;
  if (!method || !parse_method_spec(method, m, src) || is_dftb(m)) {
    copy_message("unknown NDDO method", errmsg, errcap);
    return SG_ERR_UNKNOWN_METHOD;
  }
  if (!alpha_x) return SG_ERR_INVALID_ARGUMENT;
  std::string err;
  std::shared_ptr<const NddoParamSet> set;
  if (!src.empty() && !(set = nddo_parameter_set(m, src, err))) {
    copy_message(err, errmsg, errcap);
    return SG_ERR_PARAMETERS;
  }
  const DiatomicDev d = make_diatomic(m, Z1, Z2, set.get());
  if (!d.present) {
    copy_message("no diatomic parameters for the pair", errmsg, errcap);
    return SG_ERR_UNSUPPORTED_ELEMENT;
  }
  alpha_x[0] = d.alpha;
  alpha_x[1] = d.x;
  return SG_OK;
}

int32_t sg_calculate_hessian(const char* method, int32_t n_atoms, const int32_t* Z, const double* xyz, int32_t charge,
                             int32_t multiplicity, int32_t unrestricted, double scc, double rmsd, int32_t max_iter,
                             double step, double* hessian, int32_t* not_converged, char* errmsg, int32_t errcap) {
  using namespace sgb;
  HessianRequest hr;
  std::string src;
  if (!method || !parse_method_spec(method, hr.method, src)) {
    copy_message("unknown method", errmsg, errcap);
    return SG_ERR_UNKNOWN_METHOD;
  }
  if (n_atoms <= 0 || !Z || !xyz || !hessian) {
    copy_message("empty molecular structure or no output buffer", errmsg, errcap);
    return n_atoms <= 0 ? SG_ERR_EMPTY_STRUCTURE : SG_ERR_INVALID_ARGUMENT;
  }
  hr.parameters = src;
  hr.unrestricted = unrestricted != 0 || multiplicity != 1;
  hr.molecule.Z.assign(Z, Z + n_atoms);
  hr.molecule.xyz.assign(xyz, xyz + 3 * (size_t)n_atoms);
  hr.molecule.charge = charge;
  hr.molecule.multiplicity = multiplicity;
  hr.scf.scc = scc;
  hr.scf.rmsd = rmsd;
  hr.scf.max_iter = max_iter;
  if (step > 0) hr.step = step;
  std::vector<double> H;
  int unconverged = 0;
  std::string err;
  const int rc = numerical_hessian(hr, H, unconverged, err);
  if (not_converged) *not_converged = unconverged;
  if (rc) {
    copy_message(err, errmsg, errcap);
    return rc;
  }
  std::memcpy(hessian, H.data(), sizeof(double) * H.size());
  return SG_OK;
}

