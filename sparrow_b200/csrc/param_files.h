// Parameter sets read at run time, in the reference's own file formats.
//
// NDDO (MNDO / AM1 / PM6): a parameters.json file as written by the
// reference's Parameters::write (src/Sparrow/Sparrow/Implementations/Nddo/Parameters.cpp:20-93):
//   {"atomic":   [{"key": Z, "value": {"pack": {...}, "gaussianRepulsion": [{"a","b","c"}...]}}...],
//    "diatomic": [{"key": {"first": Z1, "second": Z2}, "value": {"exponent", "factor"}}...]}
// The STO-6G expansion of each shell follows from the orbital exponent, as the
// reference's RawParameterProcessor::setGtoExpansion does
// (Nddo/Utils/ParameterUtils/RawParameterProcessor.cpp:175-188).
//
// DFTB: a directory of Slater-Koster files X-Y.skf (or XY.skf, either case),
// with optional hubbard.dat and spin.dat, collected as
// ParameterSet::collect does (Dftb/ParameterSet.cpp:34-133) and parsed with the
// SKF grammar of Dftb/Utils/SkfParser.cpp:62-237 (forwarding files included).
// The embedded sets (mio-1-1, 3ob-3-1, 3ob-2-1) come through the same type.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "dftb_raw.h"
#include "engine_types.h"
#include "nddo_raw.h"

namespace sgb {

struct NddoParamSet {
  std::string source;  // file path, or "" for the embedded set
  std::vector<NddoRawAtomic> atomic;
  std::vector<NddoRawDiatomic> diatomic;
  const NddoRawAtomic* find(int Z) const;
  const NddoRawDiatomic* find_pair(int z1, int z2) const;
};

// The parameter set of method m from a parameters.json file (cached per path
// and file modification time).  Returns nullptr and sets err when the file is
// missing or malformed.  An empty path gives the embedded set.
std::shared_ptr<const NddoParamSet> nddo_parameter_set(Method m, const std::string& path, std::string& err);

// STO-6G expansion (exponents, normalised coefficients) of the shell with
// principal quantum number n and angular momentum l (0 or 1) for Slater
// exponent zeta.  The expansion scales with zeta: exponents as zeta^2 and
// normalised coefficients as zeta^(l + 3/2); the zeta = 1 shapes are those of
// the embedded tables.  Returns false for a shell no embedded element has.
bool sto6g_expansion(int n, int l, double zeta, double* exp6, double* coef6);

struct DftbSetData {
  std::string name;  // embedded set name or directory path
  std::vector<DftbElemRaw> elems;
  std::vector<DftbPairRaw> pairs;  // row0 / spline0 index the vectors below
  std::vector<double> table;       // 8 columns per row (Sss Hss Ssp Hsp Spp0 Hpp0 Spp1 Hpp1)
  std::vector<DftbSplineRaw> splines;
  const DftbElemRaw* find_elem(int Z) const;
  const DftbPairRaw* find_pair(int z1, int z2) const;
};

// An embedded set by name, or the s/p elements (H to Ne) of a directory of
// .skf files (cached per path).  Returns nullptr and sets err otherwise.
std::shared_ptr<const DftbSetData> dftb_parameter_set(const std::string& name_or_directory, std::string& err);

}  // namespace sgb
