// Host-side NDDO parameter processing: published (eV / Angstrom) parameters
// to the atomic-unit runtime values the kernels consume.
//
// Follows the reference's RawParameterProcessor
// (src/Sparrow/Sparrow/Implementations/Nddo/Utils/ParameterUtils/RawParameterProcessor.cpp:67-190),
// KlopmanParameter.cpp:26-92, ChargeSeparationParameter.cpp:24-47 and the
// element rules of PrincipalQuantumNumbers.cpp:20-160.
#pragma once
#include <string>

#include "engine_types.h"
#include "nddo_raw.h"

namespace sgb {

// Unit conversions.  The Bohr radius and the Hartree energy are CODATA 2014,
// the values the reference's test vectors are consistent with
// (PM6 H2 energy of src/Sparrow/Python/Tests/CalculatorTest.py:21-24 agrees
// to 5e-11 Hartree with them).
constexpr double kBohrAngstrom = 0.52917721067;
constexpr double kEvPerHartree = 4.359744650e-18 / 1.6021766208e-19;

bool parse_method(const std::string& name, Method& m);
const char* method_name(Method m);

struct NddoParamSet;

// Number of AOs the method gives element Z (0 if unsupported in this engine:
// elements that carry d orbitals or have no parameters).  set: a parameter
// set read from a file, nullptr for the embedded one.
int engine_n_aos(Method m, int Z, const NddoParamSet* set = nullptr);

// Fill the runtime parameter record for element Z.  Returns false (and sets
// err) when the method has no s/p parameters for Z.
bool make_elem(Method m, int Z, ElemDev& out, std::string& err, const NddoParamSet* set = nullptr);

// PM6 diatomic (alpha_AB, x_AB) for a pair of elements; present=0 if missing.
DiatomicDev make_diatomic(Method m, int Z1, int Z2, const NddoParamSet* set = nullptr);

// The embedded (published) NDDO records of a method.
const NddoRawAtomic* nddo_embedded_atomic(Method m, size_t& count);
const NddoRawDiatomic* nddo_embedded_diatomic(Method m, size_t& count);

// Standard atomic weight of element Z (u), 0 for elements outside the table
// (centre of mass of the NDDO dipole moment).
double standard_atomic_mass(int Z);

// Principal quantum number of the valence s (l = 0) or p (l = 1) shell of
// element Z (PrincipalQuantumNumbers.cpp:20-57).
int nddo_shell_n(int Z, int l);

}  // namespace sgb
