// Raw (as published) NDDO parameter records.
//
// Field meaning follows the reference's parameter pack
// (src/Sparrow/Sparrow/Implementations/Nddo/Parameters.h:20-138): one-centre
// energies U_ss/U_pp and resonance integrals beta_s/beta_p in eV, Slater
// exponents zeta_s/zeta_p, one-centre two-electron integrals g_ss, g_pp, g_sp,
// g_p2, h_sp in eV, the core Klopman radius pcore in bohr, the core-repulsion
// exponent alpha in 1/Angstrom and up to four Gaussian core-repulsion terms
// (a [-], b [1/Angstrom^2], c [Angstrom]).  The STO-6G expansions are the
// (exponent, normalised coefficient) pairs that the reference's overlap code
// multiplies directly (Nddo/Utils/IntegralsEvaluationUtils/GTOOverlapMatrixBlock.cpp:70-134).
//
// The data tables themselves live in nddo_tables.inc, generated by
// sparrow_b200/params/gen_tables.py.  This header is plain C/C++ so both the
// CUDA engine and the CPU oracle can read the same published numbers.
#pragma once

enum NddoRawIndex {
  kRawUss = 0,
  kRawUpp,
  kRawBetaS,
  kRawBetaP,
  kRawZetaS,
  kRawZetaP,
  kRawGss,
  kRawGpp,
  kRawGsp,
  kRawGp2,
  kRawHsp,
  kRawPcore,
  kRawAlpha,
  kRawCount
};

struct NddoRawAtomic {
  int Z;
  int has_d;            // the element carries d-shell parameters in this method
  double v[kRawCount];  // indexed by NddoRawIndex
  int n_gauss;
  double ga[4], gb[4], gc[4];
  double s_exp[6], s_coef[6];
  double p_exp[6], p_coef[6];
};

struct NddoRawDiatomic {
  int z1, z2;       // as stored in the published file (any order)
  double exponent;  // alpha_AB (1/Angstrom, or 1/Angstrom^2 for X-H with X in {C,N,O})
  double factor;    // x_AB
};
