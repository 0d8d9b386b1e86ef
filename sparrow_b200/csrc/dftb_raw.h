// Raw DFTB parameter records as generated into dftb_tables.inc from the
// reference's Slater-Koster parameter sets (see params/gen_dftb_tables.py).
// Atomic units (Hartree, bohr).
#pragma once

namespace sgb {

struct DftbElemRaw {
  int Z;
  double es, ep, ed;     // orbital energies
  double us, up, ud;     // Hubbard parameters (the s value is the atom's U)
  double fs, fp, fd;     // occupations of the neutral atom
  double hubbard_derivative;
  int has_hubbard_derivative;
  double wss, wpp;       // spin constants (spin.dat): triplet excitations, spin-polarised SCC
  int has_spin;
  double wsp, wps;       // the s-p spin constants (spin-polarised SCC)
};

struct DftbPairRaw {
  int z1, z2;            // file Z1-Z2.skf
  double grid;           // grid distance
  int rows, row0;        // table rows and first row in kDftbTable
  int n_spline;          // repulsion spline intervals
  double cutoff, a1, a2, a3, c4, c5;
  int spline0;           // first interval in kDftbSplineRaw
};

struct DftbSplineRaw {
  double start, end, c0, c1, c2, c3;
};

struct DftbSetRaw {
  const char* name;
  int elem0, n_elem, pair0, n_pair;
};

}  // namespace sgb
