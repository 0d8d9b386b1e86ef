#include "params.h"
#include "dftb_params.h"
#include "param_files.h"

#include <algorithm>
#include <cctype>
#include <cmath>

#include "nddo_raw.h"
#include "nddo_tables.inc"

namespace sgb {

namespace {

constexpr double kHartreePerEv = 1.0 / kEvPerHartree;
constexpr double kAngstromPerBohr = kBohrAngstrom;
constexpr double kBohrPerAngstrom = 1.0 / kBohrAngstrom;

template <size_t N>
const NddoRawAtomic* lookup(const NddoRawAtomic (&tab)[N], int Z) {
  for (size_t i = 0; i < N; ++i)
    if (tab[i].Z == Z) return &tab[i];
  return nullptr;
}

const NddoRawAtomic* raw_for(Method m, int Z, const NddoParamSet* set) {
  if (set) return set->find(Z);
  switch (m) {
    case kPM6: return lookup(kPM6Atomic, Z);
    case kAM1: return lookup(kAM1Atomic, Z);
    default: return lookup(kMNDOAtomic, Z);
  }
}

// Valence shell principal quantum numbers (PrincipalQuantumNumbers.cpp:20-57)
int shell_n_s(int Z) {
  static const int edge[] = {2, 9, 17, 35, 53, 83};
  for (int i = 0; i < 6; ++i)
    if (Z <= edge[i]) return i + 1;
  return 7;
}
int shell_n_p(int Z) {
  static const int edge[] = {10, 18, 36, 54, 83};
  for (int i = 0; i < 5; ++i)
    if (Z <= edge[i]) return i + 2;
  return 7;
}

// PM6 basis size (PrincipalQuantumNumbers.cpp:74-121): ranges of Z with 4 or 9 AOs.
int pm6_n_aos(int Z) {
  struct Range { int last, n; };
  static const Range r[] = {{12, 4}, {17, 9}, {20, 4}, {29, 9}, {32, 4}, {33, 9}, {34, 4}, {35, 9}, {38, 4},
                            {47, 9}, {50, 4}, {51, 9}, {52, 4}, {53, 9}, {56, 4}, {79, 9}, {83, 4}};
  for (const auto& x : r)
    if (Z <= x.last) return x.n;
  return 0;
}

// Core charge (PrincipalQuantumNumbers.cpp:135-160)
double core_charge(int Z) {
  if (Z == 10 || Z == 18 || Z == 36 || Z == 54) return 6.0;
  static const int shells[] = {86, 78, 68, 54, 46, 36, 28, 18, 10, 2};
  for (int c : shells)
    if (Z > c) return Z - c;
  return Z;
}

double factorial(int n) {
  double f = 1;
  for (int i = 2; i <= n; ++i) f *= i;
  return f;
}

// Overlap-like factor A(n1, n2, z1, z2, L) of the charge-separation formula
double sep_factor(int n1, int n2, double z1, double z2, int L) {
  return std::pow(2 * z1, n1 + 0.5) * std::pow(2 * z2, n2 + 0.5) * std::pow(z1 + z2, -(double)(n1 + n2 + L + 1)) /
         std::sqrt(factorial(2 * n1) * factorial(2 * n2)) * factorial(n1 + n2 + L);
}

// Newton solve (start 0.001, stop when the step is <= 1e-8) of
//   dipole:      1/r - 1/sqrt(r^2 + D^2)                      = shift
//   quadrupole:  1/r - 2/sqrt(r^2 + D^2) + 1/sqrt(r^2 + 2 D^2) = shift
double klopman_radius(double D, double shift, bool quadrupole) {
  double r = 0.001, prev = 0;
  while (std::fabs(r - prev) > 1e-8) {
    double r2 = r * r, d2 = D * D;
    double f, df;
    if (!quadrupole) {
      double s = std::sqrt(r2 + d2);
      f = 1.0 / r - 1.0 / s - shift;
      df = -1.0 / r2 + r / (s * s * s);
    } else {
      double s1 = std::sqrt(r2 + d2), s2 = std::sqrt(r2 + 2 * d2);
      f = 1.0 / r - 2.0 / s1 + 1.0 / s2 - shift;
      df = -1.0 / r2 + 2 * r / (s1 * s1 * s1) - r / (s2 * s2 * s2);
    }
    prev = r;
    r = r - f / df;
  }
  return r;
}

}  // namespace

bool parse_method(const std::string& name, Method& m) {
  std::string t = name;
  std::transform(t.begin(), t.end(), t.begin(), [](unsigned char c) { return (char)std::toupper(c); });
  if (t == "PM6") m = kPM6;
  else if (t == "AM1") m = kAM1;
  else if (t == "MNDO") m = kMNDO;
  else if (t == "DFTB2") m = kDFTB2;
  else if (t == "DFTB3") m = kDFTB3;
  else return false;
  return true;
}

const char* method_name(Method m) {
  switch (m) {
    case kPM6: return "PM6";
    case kAM1: return "AM1";
    case kDFTB2: return "DFTB2";
    case kDFTB3: return "DFTB3";
    default: return "MNDO";
  }
}

const NddoRawAtomic* nddo_embedded_atomic(Method m, size_t& count) {
  switch (m) {
    case kPM6: count = sizeof(kPM6Atomic) / sizeof(kPM6Atomic[0]); return kPM6Atomic;
    case kAM1: count = sizeof(kAM1Atomic) / sizeof(kAM1Atomic[0]); return kAM1Atomic;
    default: count = sizeof(kMNDOAtomic) / sizeof(kMNDOAtomic[0]); return kMNDOAtomic;
  }
}

const NddoRawDiatomic* nddo_embedded_diatomic(Method m, size_t& count) {
  count = m == kPM6 ? (size_t)kPM6NumDiatomic : 0;
  return kPM6Diatomic;
}

int nddo_shell_n(int Z, int l) { return l == 0 ? shell_n_s(Z) : shell_n_p(Z); }

double standard_atomic_mass(int Z) {
  // IUPAC standard atomic weights (conventional values), Z = 1..56
  static const double m[] = {0.0,       1.00794,    4.002602,  6.941,       9.012182,  10.811,     12.0107,
                             14.0067,   15.9994,    18.9984032, 20.1797,    22.98976928, 24.3050,  26.9815386,
                             28.0855,   30.973762,  32.065,    35.453,      39.948,    39.0983,    40.078,
                             44.955912, 47.867,     50.9415,   51.9961,     54.938045, 55.845,     58.933195,
                             58.6934,   63.546,     65.38,     69.723,      72.64,     74.92160,   78.96,
                             79.904,    83.798,     85.4678,   87.62,       88.90585,  91.224,     92.90638,
                             95.96,     98.0,       101.07,    102.90550,   106.42,    107.8682,   112.411,
                             114.818,   118.710,    121.760,   127.60,      126.90447, 131.293,    132.9054519,
                             137.327};
  return (Z >= 1 && Z < (int)(sizeof(m) / sizeof(m[0]))) ? m[Z] : 0.0;
}

int engine_n_aos(Method m, int Z, const NddoParamSet* set) {
  if (is_dftb(m)) return dftb_n_aos(dftb_default_set(m), Z);
  const NddoRawAtomic* r = raw_for(m, Z, set);
  if (!r) return 0;
  int n = Z == 1 ? 1 : (m == kPM6 ? pm6_n_aos(Z) : 4);
  return (n == 1 || n == 4) ? n : 0;
}

bool make_elem(Method m, int Z, ElemDev& e, std::string& err, const NddoParamSet* set) {
  const NddoRawAtomic* r = raw_for(m, Z, set);
  if (!r) {
    err = std::string("no ") + method_name(m) + " parameters for element Z=" + std::to_string(Z) +
          (set && !set->source.empty() ? " in '" + set->source + "'" : std::string());
    return false;
  }
  int nao = engine_n_aos(m, Z, set);
  if (nao == 0) {
    err = std::string(method_name(m)) + " gives element Z=" + std::to_string(Z) +
          " a d shell; this engine covers s/p elements only";
    return false;
  }
  const double* v = r->v;
  e = ElemDev();
  e.Z = Z;
  e.nao = nao;
  e.core = core_charge(Z);
  e.cbrtZ = std::pow((double)Z, 1.0 / 3.0);
  e.Uss = v[kRawUss] * kHartreePerEv;
  e.Upp = v[kRawUpp] * kHartreePerEv;
  e.betaS = v[kRawBetaS] * kHartreePerEv;
  e.betaP = v[kRawBetaP] * kHartreePerEv;
  e.alpha = v[kRawAlpha] * kAngstromPerBohr;
  const double gss = v[kRawGss] * kHartreePerEv;
  e.rho[0] = 1.0 / (2.0 * gss);
  if (nao == 4) {
    // both separations use min(n_s, n_p) (ChargeSeparationParameter.cpp:24-30)
    int n = std::min(shell_n_s(Z), shell_n_p(Z));
    e.D[1] = sep_factor(n, n, v[kRawZetaS], v[kRawZetaP], 1) / std::sqrt(3.0);
    e.D[3] = std::sqrt(sep_factor(n, n, v[kRawZetaP], v[kRawZetaP], 2)) / std::sqrt(5.0);
    // hpp floor of 0.1 eV: reference built with REPRODUCE_PM6_ERRORS (its default)
    double hpp = std::max(0.1 * kHartreePerEv, 0.5 * (v[kRawGpp] - v[kRawGp2]) * kHartreePerEv);
    e.rho[1] = klopman_radius(e.D[1], 4.0 * v[kRawHsp] * kHartreePerEv, false);
    e.rho[2] = e.rho[0];
    e.rho[3] = klopman_radius(e.D[3], 8.0 * hpp, true);
  }
  e.pcore = v[kRawPcore] != 0 ? v[kRawPcore] : e.rho[0];
  e.gss = gss;
  e.gsp = v[kRawGsp] * kHartreePerEv;
  e.gpp = v[kRawGpp] * kHartreePerEv;
  e.gp2 = v[kRawGp2] * kHartreePerEv;
  e.hsp = v[kRawHsp] * kHartreePerEv;
  e.hpp = 0.5 * (e.gpp - e.gp2);
  e.n_gauss = r->n_gauss;
  for (int k = 0; k < 4; ++k) {
    e.ga[k] = r->ga[k] * kBohrPerAngstrom;
    e.gb[k] = r->gb[k] * kAngstromPerBohr * kAngstromPerBohr;
    e.gc[k] = r->gc[k] * kBohrPerAngstrom;
  }
  for (int k = 0; k < 6; ++k) {
    e.s_exp[k] = r->s_exp[k];
    e.s_coef[k] = r->s_coef[k];
    e.p_exp[k] = r->p_exp[k];
    e.p_coef[k] = r->p_coef[k];
  }
  return true;
}

DiatomicDev make_diatomic(Method m, int Z1, int Z2, const NddoParamSet* set) {
  DiatomicDev d;
  if (m != kPM6) return d;
  size_t count = 0;
  const NddoRawDiatomic* tab = set ? set->diatomic.data() : nddo_embedded_diatomic(m, count);
  if (set) count = set->diatomic.size();
  for (size_t i = 0; i < count; ++i) {
    const NddoRawDiatomic& r = tab[i];
    if ((r.z1 == Z1 && r.z2 == Z2) || (r.z1 == Z2 && r.z2 == Z1)) {
      bool xh = (Z1 == 1 && (Z2 == 6 || Z2 == 7 || Z2 == 8)) || (Z2 == 1 && (Z1 == 6 || Z1 == 7 || Z1 == 8));
      d.alpha = xh ? r.exponent * kAngstromPerBohr * kAngstromPerBohr : r.exponent * kAngstromPerBohr;
      d.x = r.factor;
      d.present = 1;
      break;
    }
  }
  return d;
}

}  // namespace sgb
