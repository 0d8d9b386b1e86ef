// Builds the point-charge term table of the local two-centre integrals.
//
// Each s/p orbital pair is a sum of multipoles (Local2c2eIntegralCalculator.cpp:125-292
// with no d functions present), each multipole a set of point charges at
// offsets that are multiples of its charge separation (ChargesInMultipoles.cpp:27-125).
// A local integral is the sum, over multipole pairs of equal magnetic quantum
// number, of q1 q2 / sqrt(|r2 - r1 + R z|^2 + (rho_A + rho_B)^2)
// (MultipoleMultipoleTerm.h:58-98).  Terms with identical geometry and class
// are merged, and terms whose merged charge product vanishes are dropped.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "nddo_math.cuh"

namespace sgb {

namespace {

struct Charge { double x, y, z, q; };
enum MP { M00, Qxx, Qyy, Qzz, M1m1, M10, M11, M2m2, M2m1, M21 };

const std::vector<Charge>& charges(MP m) {
  static const std::vector<Charge> c[10] = {
      {{0, 0, 0, 1}},
      {{-2, 0, 0, .25}, {2, 0, 0, .25}, {0, 0, 0, -.5}},
      {{0, -2, 0, .25}, {0, 2, 0, .25}, {0, 0, 0, -.5}},
      {{0, 0, -2, .25}, {0, 0, 2, .25}, {0, 0, 0, -.5}},
      {{0, -1, 0, -.5}, {0, 1, 0, .5}},
      {{0, 0, -1, -.5}, {0, 0, 1, .5}},
      {{-1, 0, 0, -.5}, {1, 0, 0, .5}},
      {{1, 1, 0, .25}, {-1, -1, 0, .25}, {1, -1, 0, -.25}, {-1, 1, 0, -.25}},
      {{0, 1, 1, .25}, {0, -1, -1, .25}, {0, 1, -1, -.25}, {0, -1, 1, -.25}},
      {{1, 0, 1, .25}, {-1, 0, -1, .25}, {1, 0, -1, -.25}, {-1, 0, 1, -.25}},
  };
  return c[m];
}

int m_number(MP m) {
  switch (m) {
    case M1m1: case M2m1: return -1;
    case M11: case M21: return 1;
    case M2m2: return -2;
    default: return 0;
  }
}

struct Mult { double f; MP m; int cls; };

std::vector<Mult> expansion(int p) {
  switch (p) {
    case 0: return {{1, M00, 0}};
    case 1: return {{1, M11, 1}};
    case 3: return {{1, M1m1, 1}};
    case 6: return {{1, M10, 1}};
    case 7: return {{1, M21, 3}};
    case 8: return {{1, M2m1, 3}};
    case 4: return {{1, M2m2, 3}};
    case 9: return {{1, M00, 2}, {1, Qzz, 3}};
    case 2: return {{1, M00, 2}, {1, Qxx, 3}};
    case 5: return {{1, M00, 2}, {1, Qyy, 3}};
  }
  return {};
}

}  // namespace

void build_local_term_table(LocalTermTable& tab) {
  std::memset(&tab, 0, sizeof(tab));
  // entries the reference evaluates (Local2c2eMatrix.cpp:91-149); the rest are copies
  static const int kEval[kLocalUnique][2] = {{0, 0}, {0, 2}, {0, 6}, {0, 9}, {2, 0}, {6, 0}, {9, 0},
                                             {1, 1}, {1, 7}, {2, 2}, {2, 5}, {2, 6}, {2, 9}, {6, 2},
                                             {6, 6}, {6, 9}, {7, 1}, {7, 7}, {9, 2}, {9, 6}, {9, 9}};
  int nt = 0;
  for (int e = 0; e < kLocalUnique; ++e) {
    tab.row[e] = kEval[e][0];
    tab.col[e] = kEval[e][1];
    tab.start[e] = nt;
    std::vector<LocalTerm> terms;
    for (const Mult& a : expansion(kEval[e][0]))
      for (const Mult& b : expansion(kEval[e][1])) {
        if (m_number(a.m) != m_number(b.m)) continue;
        for (const Charge& c1 : charges(a.m))
          for (const Charge& c2 : charges(b.m)) {
            LocalTerm t;
            t.q = a.f * b.f * c1.q * c2.q;
            t.x1 = (float)c1.x; t.y1 = (float)c1.y; t.z1 = (float)c1.z;
            t.x2 = (float)c2.x; t.y2 = (float)c2.y; t.z2 = (float)c2.z;
            t.c1 = a.cls;
            t.c2 = b.cls;
            bool merged = false;
            for (auto& u : terms) {
              if (u.c1 == t.c1 && u.c2 == t.c2 && u.x1 == t.x1 && u.y1 == t.y1 && u.z1 == t.z1 && u.x2 == t.x2 &&
                  u.y2 == t.y2 && u.z2 == t.z2) {
                u.q += t.q;
                merged = true;
                break;
              }
            }
            if (!merged) terms.push_back(t);
          }
      }
    for (const auto& t : terms) {
      if (std::fabs(t.q) < 1e-12) continue;
      if (nt >= kLocalMaxTerms) throw std::runtime_error("local term table overflow");
      tab.term[nt++] = t;
    }
    tab.count[e] = nt - tab.start[e];
  }
  tab.n_terms = nt;
  // sigma column (p | ss) entries 0, 4, 5, 6 and row (ss | p) entries 0, 1, 2, 3
  // for p = ss, xx, sz, zz
  static const int kCol[4] = {0, 4, 5, 6}, kRow[4] = {0, 1, 2, 3}, kSig[4] = {0, 2, 6, 9};
  for (int k = 0; k < 4; ++k)
    if (tab.row[kCol[k]] != kSig[k] || tab.col[kCol[k]] != 0 || tab.row[kRow[k]] != 0 || tab.col[kRow[k]] != kSig[k])
      throw std::runtime_error("local term table: unexpected sigma entry order");
  // the heavy-pair value kernel stages every two-electron term and both
  // core-attraction sigma columns' terms of one pair in kPairTermSlots slots
  int ncore = 0;
  for (int k = 0; k < 4; ++k) ncore += tab.count[kCol[k]];
  if (nt + 2 * ncore > kPairTermSlots) throw std::runtime_error("local term table: more terms than pair slots");
}

}  // namespace sgb
