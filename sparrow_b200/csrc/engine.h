// Host orchestration of batched NDDO single points on one GPU.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "engine_types.h"
#include "kernels.h"
#include "param_files.h"

namespace sgb {

// Residual norm at which the TD-DFTB Davidson iteration stops (on the Casida
// matrix, whose eigenvalues are omega^2 ~ 1e-3..1e-1 Hartree^2).  An
// eigenvector error is about the residual over the gap to the next root; the
// lowest roots of long polyenes lie ~2e-4 Hartree^2 apart, so 1e-10 keeps
// transition dipoles of several e bohr within 1e-5.
constexpr double kTddftbResidual = 1e-10;
constexpr int kTddftbMaxIter = 300;

struct MoleculeInput {
  std::vector<int> Z;
  std::vector<double> xyz;  // bohr, 3 per atom
  int charge = 0;
  int multiplicity = 1;     // 2S + 1 (unrestricted batches)
};

struct MoleculeOutput {
  double energy = 0, e_el = 0, e_rep = 0;
  int iterations = 0, converged = 0, status = 0;
  int nao = 0, nocc = 0, nel = 0;
  int nocc_b = 0;  // unrestricted: beta electrons (nocc: alpha electrons)
  std::vector<double> gradient;  // 3 per atom (Hartree/bohr)
};

// Status codes shared with the C-ABI (include/sparrow_b200.h).
enum Status : int {
  kOk = 0,
  kErrInvalidArgument = 1,
  kErrUnknownMethod = 2,
  kErrUnsupportedElement = 3,
  kErrEmptyStructure = 4,
  kErrOddElectrons = 5,
  kErrNotConverged = 6,
  kErrCuda = 7,
  kErrOutOfMemory = 8,
  kErrNoResults = 9,
  kErrUnknownSetting = 10,
  kErrDevice = 11,
  kErrTimeout = 12,
  kPending = 13,
  kErrParameters = 14,  // a parameter file is missing or malformed
};

// A batch resident on the device: descriptors, integrals, matrices, results.
class Batch {
 public:
  explicit Batch(Method m);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // Host-side setup and upload of a set of molecules.  Returns a Status.
  // check_pairs: wait for the device-built pair table and report coincident
  // atoms as an error (a caller that validated the geometries itself, like
  // the request server, passes false and setup does not block).
  int setup(const std::vector<MoleculeInput>& mols, std::string& err, bool check_pairs = true);
  // Replace positions (same atoms, same order) and upload them.
  int set_positions(const double* xyz_bohr_all, std::string& err);
  // Optional start densities (one N x N matrix per molecule, concatenated).
  int set_start_density(const double* P_all, std::string& err);
  // Run integrals -> SCF -> (gradient) on the device.  Asynchronous on stream().
  int run(const ScfParams& sp, bool gradient, std::string& err);
  // Copy results back (synchronises the stream).
  int fetch(std::vector<MoleculeOutput>& out, bool gradient, std::string& err);
  int fetch_density(int mol, std::vector<double>& P, std::string& err);
  int fetch_raw_results(std::vector<MolResult>& r, std::string& err);
  // Atomic charges of molecule mol after run(): DFTB the Mulliken charges of
  // the SCC (computed on the device with the final density), NDDO core charge
  // minus the atom's diagonal density (Mulliken in the orthogonal NDDO basis).
  int fetch_charges(int mol, std::vector<double>& q, std::string& err);
  // Dipole moment (e bohr) of molecule mol after run(): DFTB sum_a q_a R_a
  // (Dftb/Utils/DipoleUtils/DFTBDipoleMomentCalculator.cpp:23-35); NDDO the
  // NDDO approximation about the centre of mass, sum_a q_a (R_a - R_cm) minus
  // 2 D_sp1 P_{s,p} per s/p atom (Nddo/Utils/DipoleUtils/NDDODipoleMomentCalculator.cpp:76-110).
  int dipole(int mol, double out[3], std::string& err);
  // Unrestricted batches: the spin densities of molecule mol, and start spin
  // densities for the next run() (mat_total doubles each, the molecules' N x N
  // blocks in order; the warm start of an open-shell geometry step).
  int fetch_spin_densities(int mol, std::vector<double>& Pa, std::vector<double>& Pb, std::string& err);
  int set_start_spin_densities(const double* Pa, const double* Pb, std::string& err);
  // alpha orbital energies (restricted: the orbital energies); beta = true: the beta ones
  int fetch_orbital_energies(int mol, std::vector<double>& eps, std::string& err, bool beta = false);
  // Linear-response TD-DFTB (DFTB2 / DFTB3 batches, after run()): the nroots
  // (<= 16) lowest singlet (or triplet) excitations of every molecule.
  // Asynchronous on stream(); overwrites the orbital scratch (the gradient of
  // the preceding run() stays valid).  tol: Davidson residual norm.
  int run_tddftb(int nroots, bool triplet, double tol, int max_iter, std::string& err);
  // omega [nmol * nroots] (Hartree), dipoles [nmol * nroots * 3] (e bohr,
  // zero for triplets), info [nmol * 2] (Davidson iterations, status).
  int fetch_tddftb(std::vector<double>& omega, std::vector<double>& dipoles, std::vector<int>& info, std::string& err);
  // SM cycles per molecule of the last TD-DFTB run: canonical orbitals,
  // transition charges, Davidson (3 per molecule)
  int fetch_tddftb_cycles(std::vector<long long>& cycles, std::string& err);
  int tddftb_roots() const { return td_roots_; }

  cudaStream_t stream() const { return stream_; }
  Method method() const { return method_; }
  // Parameter source, the reference's "method_parameters" setting; empty =
  // the method's embedded default.  DFTB: an embedded set name (mio-1-1,
  // 3ob-3-1, 3ob-2-1) or a directory of Slater-Koster files; NDDO: the path of
  // a parameters.json file.  Takes effect at the next setup().
  void set_parameters(const std::string& source) { param_source_ = source; }
  // Unrestricted (UHF) SCF for every molecule of the batch, each with its
  // MoleculeInput::multiplicity (NDDO, batched SCF path).  Takes effect at
  // the next setup().
  void set_unrestricted(bool u) { uhf_ = u; }
  bool unrestricted() const { return uhf_; }
  const std::string& parameters() const { return param_source_; }
  // SCF path: 0 automatic (one NDDO molecule of more than 1024 AOs runs the
  // large-molecule path, anything else the batched kernel), 1 batched
  // kernel, 2 large-molecule path in FP64, 3 large-molecule path with
  // mixed-precision purification.  Paths 2 and 3 take one NDDO molecule.
  int set_scf_path(int path, std::string& err);
  int scf_path() const { return scf_path_; }
  // Path taken by the last run(): 1 batched kernel, 2 / 3 large-molecule
  bool last_run_large() const { return dev_.large != 0; }
  int n_molecules() const { return (int)mols_.size(); }
  int n_atoms() const { return (int)atoms_.size(); }
  long long device_bytes() const { return arena_bytes_; }
  const DeviceBatch& device() const { return dev_; }
  // Kernel launches of the last run() (for accounting)
  int launches_last_run() const { return launches_; }
  // Device time (ms) of the stages of the last run(): pair integrals,
  // one-electron assembly, SCF, gradient.  Synchronises on the last event.
  int stage_times(double ms[4], std::string& err);
  // Bytes copied host->device and device->host since the batch was set up.
  long long h2d_bytes() const { return h2d_bytes_; }
  long long d2h_bytes() const { return d2h_bytes_; }
  // User timing events on the batch stream (slots 0..7).
  int record_event(int slot, std::string& err);
  int event_elapsed(int s0, int s1, double* ms, std::string& err);

 private:
  int ensure_arena(size_t bytes, std::string& err);
  Method method_;
  cudaStream_t stream_ = nullptr;
  void* arena_ = nullptr;
  size_t arena_bytes_ = 0;
  void* pinned_ = nullptr;
  size_t pinned_bytes_ = 0;
  DeviceBatch dev_;
  std::vector<MolDev> mols_;
  std::vector<AtomDev> atoms_;
  std::vector<ElemDev> elems_;
  std::vector<DiatomicDev> diat_;
  std::vector<int> ao_atom_, order_;
  long long npairs_ = 0, nhh_ = 0;  // pair and heavy-pair tables are built on the device
  std::string param_source_;
  bool uhf_ = false;
  bool spin_given_ = false;
  std::shared_ptr<const NddoParamSet> nddo_set_;  // resolved NDDO source (nullptr: embedded)
  int scf_path_ = 0;
  void* td_scratch_ = nullptr;
  size_t td_scratch_bytes_ = 0;
  int td_roots_ = 0;
  double* td_omega_ = nullptr;
  double* td_dip_ = nullptr;
  int* td_info_ = nullptr;
  long long* td_cycles_ = nullptr;
  void* large_scratch_ = nullptr;
  size_t large_scratch_bytes_ = 0;
  int scf_grid_ = 0;
  int scf_grid_nao_ = 0;
  int launches_ = 0;
  bool density_given_ = false;
  long long h2d_bytes_ = 0, d2h_bytes_ = 0;
  cudaEvent_t stage_ev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t user_ev_[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool stages_recorded_ = false;
};

// Device arenas and pinned staging buffers are cached per device after a
// batch is destroyed, so repeated batches do not pay cudaMalloc/cudaFree.
void release_cached_memory();

// Human-readable message for a CUDA error, also used by the C-ABI.
std::string cuda_message(cudaError_t e);

}  // namespace sgb
