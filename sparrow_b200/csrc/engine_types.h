// Device-visible data layout of the batched NDDO engine.
//
// A batch is a set of independent molecules.  Everything lives in one device
// arena; the structs below are the descriptors the kernels read.  Layout in
// HBM (all FP64 unless noted):
//   atoms      AtomDev[n_atoms]            element slot, AO start, position (bohr)
//   pairs      PairDev[n_pairs]            i<j atom pairs of every molecule, sorted by
//                                          molecule and by (i, j); int_off indexes the
//                                          integral pool
//   integrals  double[int_total]           per pair: dA x dB global 2c2e block
//                                          (dA, dB in {1, 10}; packed orbital-pair
//                                          index p(mu<=nu) = nu(nu+1)/2 + mu)
//   vcore      double[n_pairs][20]         core-attraction vectors VA[10] | VB[10]
//   overlap    double[n_pairs][16]         STO-6G overlap block S[mu on i][nu on j]
//   erep       double[n_pairs]             core-core repulsion of the pair
//   H, P, F, C double[mat_total]           per molecule N x N, row-major, at mat_off
//   DIIS       double[diis_total]          per molecule 2 * kDiisMax * N * N
#pragma once
#include <cstdint>

namespace sgb {

constexpr int kMaxAtomsPerMolecule = 4096;
constexpr int kDiisMax = 6;          // Pulay subspace size
// Largest stored <E, E> below which every Pulay error vector is rounding
// noise: F and P commute to working precision (a converged system, or one
// pinned by symmetry such as H2, where FP - PF vanishes identically).  The B
// matrix is then noise and its solution arbitrary, so the step keeps F.
constexpr double kDiisNoiseNorm = 1e-24;
constexpr int kMaxElementSlots = 16; // distinct elements in one batch

enum Method : int { kMNDO = 0, kAM1 = 1, kPM6 = 2, kDFTB2 = 3, kDFTB3 = 4 };
inline bool is_dftb(int m) { return m == kDFTB2 || m == kDFTB3; }

struct ElemDev {
  int Z = 0;
  int nao = 0;
  double core = 0;     // core charge
  double cbrtZ = 0;    // Z^(1/3) with Z the atomic number
  double Uss = 0, Upp = 0, betaS = 0, betaP = 0;
  double alpha = 0;    // MNDO/AM1 core-repulsion exponent (1/bohr)
  double rho[4] = {0, 0, 0, 0};  // Klopman radii by multipole class: ss0, sp1, pp0, pp2
  double D[4] = {0, 0, 0, 0};    // charge separations by class: 0, D_sp1, 0, D_pp2
  double pcore = 0;
  double gss = 0, gsp = 0, gpp = 0, gp2 = 0, hsp = 0, hpp = 0;
  int n_gauss = 0;
  double ga[4] = {0, 0, 0, 0}, gb[4] = {0, 0, 0, 0}, gc[4] = {0, 0, 0, 0};
  double s_exp[6], s_coef[6], p_exp[6], p_coef[6];
};

struct DiatomicDev {
  double alpha = 0;  // 1/bohr (1/bohr^2 for X-H with X in C, N, O)
  double x = 0;
  int present = 0;
};

struct AtomDev {
  double x, y, z;
  int slot;   // element slot
  int ao0;    // first AO within the molecule
  int mol;    // molecule index
  int pad;
};

struct PairDev {
  int a, b;      // global atom indices, a < b, same molecule
  int mol;
  int int_off;   // offset into the integral pool
};

struct MolDev {
  int nat, nao, nocc, nel;
  int atom0;      // first atom (global index)
  int pair0;      // first pair (global index)
  int npairs;
  int ao_base;    // first AO (global index) in the ao_atom map
  int hh0;        // first entry of this molecule in the list of s/p-s/p pairs
  int nhh;        // number of pairs where both atoms carry an s/p shell
  int nocc_b;     // unrestricted: beta electrons (nocc holds the alpha count)
  int pad_;
  long long mat_off;   // N*N matrices (H, P, F, C, scratch) at this offset
  long long diis_off;  // DIIS history
  long long int_off;   // first integral of the molecule
  long long gam_off;  // DFTB: offset of the molecule's nat x nat gamma blocks
};

// Per-molecule result record written by the SCF kernel.
struct MolResult {
  double energy;       // E_el + E_rep (Hartree)
  double e_el;
  double e_rep;
  double last_dE;
  double last_rmsd;
  int iterations;
  int converged;       // 1 if both criteria were met
  int status;          // 0 ok, nonzero = device-side failure code
  int full_diag;       // full diagonalisations performed
  int jacobi_sweeps;   // total Jacobi sweeps
  int pad;
  // SM cycles (clock64 on the CTA) spent per phase: Fock build, DIIS,
  // occupied-virtual rotation, full diagonalisation, density
  long long cycles[5];
};

constexpr int kEigExact = 0, kEigHybrid = 1, kEigRotation = 2;
constexpr int kTuneBins = 16;  // molecule-size bins of 32 AOs for the tuned SCF choices
}  // namespace sgb
#include "tuned_table.h"
namespace sgb {

struct ScfParams {
  double scc = 1e-7;   // |Delta E| criterion (Hartree)
  double rmsd = 1e-5;  // rms(Delta P) criterion
  int max_iter = 100;
  int diis_size = kDiisMax;
  int jacobi_max_sweeps = 30;
  // cap on the sweeps of the first (cold) diagonalisation, which only has to
  // separate occupied from virtual orbitals; 0 = the method's default (NDDO
  // 3: the rotations converge the rest cheaper than more sweeps; DFTB 6: the
  // small gaps of conjugated chains need the better start)
  int cold_sweeps = 0;
  // 1: after convergence, diagonalise the final Fock matrix from the current
  // orbitals (a warm Jacobi), so the orbital energies are its eigenvalues.
  // The occupied-virtual rotation leaves the occupied-occupied and
  // virtual-virtual blocks unrotated, which changes no density or energy but
  // leaves the individual orbital energies as diagonal elements.
  int canonical = 0;
  // Orbital update and Pulay subspace size per molecule-size bin (32 AOs per
  // bin, the last one open), defaulting to the autotuner's table
  // (tuned_table.h).  Orbital-update modes (kEig*): exact = a full
  // diagonalisation of the extrapolated Fock matrix every iteration
  // (Householder tridiagonal solver, Jacobi on clustered spectra); hybrid =
  // the tridiagonal solver for the start, then occupied-virtual rotations;
  // rotation = a Jacobi start, then occupied-virtual rotations.  diis_size
  // above caps every bin's subspace.
  signed char eig_mode_bin[kTuneBins] = SGB_TUNED_ORBITAL_UPDATE;
  signed char diis_bin[kTuneBins] = SGB_TUNED_DIIS_SIZE;
  // large-molecule mixed-precision path: purification switches from split-BF16
  // to FP64 once rms(Delta P) falls below this (or stops halving below 1e-4)
  double mixed_switch_rmsd = 1e-5;
};

__host__ __device__ inline int tune_bin(int nao) { return (nao >> 5) < kTuneBins ? (nao >> 5) : kTuneBins - 1; }
__host__ __device__ inline int scf_eig_mode(const ScfParams& sp, int nao) { return sp.eig_mode_bin[tune_bin(nao)]; }
__host__ __device__ inline int scf_diis_size(const ScfParams& sp, int nao) {
  int m = sp.diis_bin[tune_bin(nao)];
  if (sp.diis_size < m) m = sp.diis_size;
  return m < 1 ? 1 : (m > kDiisMax ? kDiisMax : m);
}

// Device failure codes (MolResult::status)
enum DeviceStatus : int {
  kDevOk = 0,
  kDevJacobiNotConverged = 1,
  kDevDiisSingular = 2,
  kDevNonFinite = 3,
  kDevSp2NotConverged = 4,  // large-molecule path: SP2 purification did not settle
};

}  // namespace sgb
