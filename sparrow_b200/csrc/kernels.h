// Kernel launch interface of the batched NDDO engine.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "engine_types.h"

namespace sgb {

struct LocalTermTable;
struct DftbElemDev;
struct DftbPairDev;
struct DftbSplineDev;

// Recorded Jacobi rotations per SCF CTA (device scratch): a cold start of up
// to six sweeps fits without an intermediate replay for N <= 256.
constexpr size_t kScfRotationBytesPerCta = size_t(2) << 20;

// Device pointers of one batch (all inside one arena).
struct DeviceBatch {
  int method = kPM6;
  int nmol = 0, natoms = 0, npairs = 0;
  long long nao_total = 0, mat_total = 0, diis_total = 0, int_total = 0;
  int max_nao = 0;
  MolDev* mols = nullptr;
  AtomDev* atoms = nullptr;
  PairDev* pairs = nullptr;
  ElemDev* elems = nullptr;
  DiatomicDev* diat = nullptr;      // [kMaxElementSlots * kMaxElementSlots]
  int* ao_atom = nullptr;           // [nao_total] global atom of each AO
  int* order = nullptr;             // molecule processing order (largest first)
  int* counter = nullptr;           // work counter of the persistent SCF kernel
  double* ints = nullptr;           // [int_total]
  double* vcore = nullptr;          // [npairs * 20]
  double* jbuf = nullptr;           // [npairs * 20] per-pair Coulomb vectors of the Fock build
  int* hh_pairs = nullptr;          // [n_hh] global pair indices of s/p-s/p pairs
  int nhh_total = 0;
  double* ovl = nullptr;            // [npairs * 16]
  double* erep = nullptr;           // [npairs]
  double* H = nullptr;              // [mat_total]
  double* P = nullptr;
  double* F = nullptr;
  double* C = nullptr;
  double* W1 = nullptr;
  double* W2 = nullptr;
  double* eps = nullptr;            // [nao_total] orbital energies
  double* diis = nullptr;           // [diis_total]
  double* rotbuf = nullptr;         // [scf_grid * rot_budget] recorded Jacobi rotations per SCF CTA
  int scf_grid = 0;
  double* gpair = nullptr;          // [npairs * 3]
  double* grad = nullptr;           // [natoms * 3]
  MolResult* res = nullptr;         // [nmol]
  // unrestricted (UHF) batches: P holds P_alpha + P_beta, F the alpha Fock
  // matrix, C / eps the alpha orbitals; the beta ones and both spin densities here
  int uhf = 0;
  double* Pa = nullptr;             // [mat_total] alpha density
  double* Pb = nullptr;             // [mat_total] beta density
  double* Fb = nullptr;             // [mat_total] beta Fock matrix
  double* Cb = nullptr;             // [mat_total] beta orbitals (orbital-major)
  double* epsb = nullptr;           // [nao_total] beta orbital energies
  double* diisb = nullptr;          // [diis_total] beta DIIS ring
  double* Ppb = nullptr;            // [mat_total] DFTB: beta density in the orthogonal basis
  double* sshift = nullptr;         // [natoms * 2] DFTB: shell spin shifts eps_{a,s}, eps_{a,p}
  int use_guess = 1;                // 0: P already holds a start density
  int spin_given = 0;               // unrestricted: Pa / Pb hold given start spin densities (P = Pa + Pb)
  int large = 0;                    // 1: one molecule over the whole GPU (large-molecule path)
  void* large_scratch = nullptr;    // [large_scf_scratch_bytes(nao)] when large
  // DFTB (H holds H0)
  int dftb_order = 0;               // 2 or 3 for DFTB batches
  long long gam_total = 0;
  double* S = nullptr;              // [mat_total] overlap
  double* X = nullptr;              // [mat_total] S^-1/2
  double* Pp = nullptr;             // [mat_total] density in the orthogonal basis
  double* W3 = nullptr;             // [mat_total] scratch of the canonical-orbital pass (F, W1 stay intact)
  double* gam = nullptr;            // [gam_total] gamma (nat x nat per molecule)
  double* Gam = nullptr;            // [gam_total] Gamma (DFTB3)
  double* qat = nullptr;            // [natoms] Mulliken charges
  double* ashift = nullptr;         // [natoms * 4] atom shift terms
  DftbElemDev* delems = nullptr;    // [kMaxElementSlots]
  DftbPairDev* dpairs = nullptr;    // [kMaxElementSlots^2]
  double* dtable = nullptr;         // completed Slater-Koster tables
  DftbSplineDev* dsplines = nullptr;
};

void upload_local_terms(const LocalTermTable& tab, cudaStream_t stream);
// Per-pair table (atoms, molecule, integral offset) and the heavy-pair list of
// every molecule; flag receives 1 + the index of a pair of coincident atoms.
void launch_build_pairs(const DeviceBatch& b, int max_nat, int* flag, cudaStream_t s);
void launch_pair_values(const DeviceBatch& b, cudaStream_t s);
void launch_one_electron(const DeviceBatch& b, cudaStream_t s);
void launch_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s);
// Unrestricted batches (DeviceBatch::uhf): the same launch shape as launch_scf.
void launch_uhf_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s);
void launch_gradient(const DeviceBatch& b, cudaStream_t s);
void launch_gather_gradient(const DeviceBatch& b, cudaStream_t s);
// Fock matrix F = H + G(P) of the batch's single (large) molecule over the
// whole GPU; *energy (device) receives the electronic energy of P.
void launch_fock_grid(const DeviceBatch& b, const double* P, double* F, double* energy, cudaStream_t s);
// DFTB: pair and on-site terms (+ start density), SCC loop, gradient
void launch_dftb_setup(const DeviceBatch& b, cudaStream_t s);
void launch_dftb_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s);
// Canonical orbitals after convergence (ScfParams::canonical): warm
// diagonalisations of the final Fock matrices left by the SCF kernels.
void launch_canonical(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s);
void launch_dftb_canonical(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s);
void launch_dftb_gradient(const DeviceBatch& b, cudaStream_t s);
// Large-molecule SCF of the batch's single molecule m (host-driven grid
// kernels, SP2 density): precision 0 FP64, 1 mixed (split-BF16 SP2 products
// until rms(dP) < 1e-5, then FP64).  Synchronises the stream a few times per
// iteration; fills res[0] (full_diag: iterations with mixed-precision SP2,
// jacobi_sweeps: SP2 steps in total) and adds its kernel launches to
// *launches.  Returns a Status.
int run_large_scf(const DeviceBatch& b, const MolDev& m, const ScfParams& sp, int precision, cudaStream_t s,
                  int* launches, std::string& err);
size_t large_scf_scratch_bytes(long long nao);
// TD-DFTB per-molecule scratch: subspace size and doubles of the block of a
// molecule with dim occupied-virtual transitions, nat atoms and k roots.
#ifdef __CUDACC__
#define SGB_TD_HD __host__ __device__
#else
#define SGB_TD_HD
#endif
SGB_TD_HD inline int td_subspace(int dim, int k) {
  int m = 6 * k;
  if (m > 64) m = 64;
  if (m < 2 * k) m = 2 * k;
  return m < dim ? m : dim;
}
SGB_TD_HD inline long long td_block_doubles(int dim, int nat, int k) {
  const long long mm = td_subspace(dim, k);
  return (long long)nat * dim + 4LL * dim + 2 * mm * dim + 2LL * k * dim + 2LL * nat * mm + mm * mm;
}
// TD-DFTB of every molecule of a converged DFTB batch: td (device scratch,
// td_off[mol] doubles per molecule), omega [nmol * nroots], dip
// [nmol * nroots * 3], info [nmol * 2] (Davidson iterations, status), cycles
// [nmol * 3] (SM cycles: canonical orbitals, transition charges, Davidson).
void launch_tddftb(const DeviceBatch& b, double* td, const long long* td_off, int nroots, int triplet, double tol,
                   int max_iter, double* omega, double* dip, int* info, long long* cycles, int grid, cudaStream_t s);
int scf_max_grid(int max_nao);
size_t scf_rotation_bytes_per_cta();

}  // namespace sgb
