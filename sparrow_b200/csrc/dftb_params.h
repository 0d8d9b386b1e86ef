// Host-side DFTB parameter preparation: the embedded Slater-Koster sets
// (mio-1-1, 3ob-3-1, 3ob-2-1; elements H, C, N, O) turned into the device
// records of dftb_math.cuh.
//
// Follows the reference's parameter assembly
// (src/Sparrow/Sparrow/Implementations/Dftb/Utils/DFTBCommon.cpp:76-198,
// SKAtom.cpp:16-70, SKPair.cpp:24-128): orbital counts by row of the periodic
// table, core charge = occupation of the neutral atom, U = the s Hubbard
// parameter, table completion from the reverse pair, tail coefficients and
// gamma terms per ordered pair.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "dftb_math.cuh"
#include "engine_types.h"

namespace sgb {

struct DftbSetData;

// An embedded parameter set (mio-1-1, 3ob-3-1, 3ob-2-1) by name, or nullptr.
std::shared_ptr<const DftbSetData> dftb_embedded_set(const std::string& name);

// Default parameter set of a DFTB method (DFTB2: mio-1-1, DFTB3: 3ob-3-1).
const char* dftb_default_set(Method m);
// Orbitals of element Z in a set (1 or 4), 0 when the set has no s/p record for it.
int dftb_n_aos(const char* set, int Z);
// Occupation (core charge) of the neutral atom, or -1 when unknown.
double dftb_core_charge(const char* set, int Z);

struct DftbPrepared {
  std::vector<DftbElemDev> elems;       // by slot
  std::vector<DftbPairDev> pairs;       // kMaxElementSlots x kMaxElementSlots, by slot pair
  std::vector<double> table;            // completed integral tables
  std::vector<DftbSplineDev> splines;   // repulsion splines
};

// Records for the elements Zs (slot i = Zs[i]).  set is an embedded set name
// or a directory of Slater-Koster files.  order 3 requires Hubbard
// derivatives.  Returns false and sets err when a parameter is missing.
bool dftb_prepare(const std::string& set, int order, const std::vector<int>& Zs, DftbPrepared& out, std::string& err);

}  // namespace sgb
