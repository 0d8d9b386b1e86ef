// DFTB2 / DFTB3 FP64 CPU oracle.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
// sparrow_b200/: only tests/, __graft_entry__.smoke() and the cpu_baseline leg
// of bench.py load it (as oracle/liboracle_dftb.so through ctypes).  The
// product never links or calls it.
//
// A scalar restatement of the reference's restricted DFTB path for s/p
// elements.  Each routine cites the reference file it follows (paths relative
// to src/Sparrow/Sparrow/Implementations/Dftb/):
//   parameters       Utils/DFTBCommon.cpp:76-198, Utils/SKAtom.cpp:16-70,
//                    Utils/SKPair.cpp:24-128 (table completion, gamma terms)
//   SK integrals     Utils/SKPair.cpp:130-304 (8-point Neville interpolation,
//                    5th-order tail), SKPair.h:80-95 (constants)
//   H0 and S         Utils/ZeroOrderMatricesCalculator.cpp:56-232, 386-412
//   gamma (DFTB2)    Utils/SecondOrderFock.cpp:53-145, 178-195
//   gamma^h (DFTB3)  Utils/ThirdOrderFock.cpp:55-200, 228-255
//   Mulliken, Fock   Utils/ScfFock.cpp:50-103 (charges q = Z - N)
//   repulsion        Utils/PairwiseRepulsion.cpp:27-73, Utils/Repulsion.cpp:33-64
//   density guess    Utils/DensityGuess.cpp:22-40
//   gradient         ZeroOrderMatricesCalculator.cpp:431-460, SecondOrderFock.cpp:148-176,
//                    ThirdOrderFock.cpp:202-226
//   TD-DFTB          Utils/DipoleUtils/TransitionChargesCalculator.h:138-165,
//                    TimeDependent/LinearResponse/TDDFTBSigmaVectorEvaluator.cpp:40-110,
//                    TDDFTBEigenvalueSolver.h:150-197, DipoleUtils/DFTBDipoleMatrixCalculator.cpp:60-84
// The SCF driver, DIIS and the generalised eigensolver live in the
// reference's un-vendored dependency (scine_utilities); they are restated from
// the standard algorithms (Loewdin orthogonalisation, Householder + QL, Pulay
// DIIS on FPS - SPF, lowest-n_occ occupation, W = 2 sum_occ eps C C^T).
// Two behaviours of the reference are kept on purpose:
//   * the tail beyond the last grid point uses the interpolated slope in
//     grid-index units and returns the derivative with respect to the tail
//     coordinate (SKPair.cpp:99-128, 178-190);
//   * the DFTB3 gradient builds d Gamma_ba / dR without the sign flip its
//     gamma term receives (ThirdOrderFock.cpp:73-77, 206-212).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../sparrow_b200/csrc/dftb_raw.h"
#include "oracle_linalg.h"

namespace sgb {
#include "../sparrow_b200/csrc/dftb_tables.inc"
}

namespace dftb_oracle {

using sgb::DftbElemRaw;
using sgb::DftbPairRaw;
using sgb::DftbSetRaw;
using sgb::kDftbElemRaw;
using sgb::kDftbPairRaw;
using sgb::kDftbSetRaw;
using sgb::kDftbSplineRaw;
using sgb::kDftbTable;

thread_local std::string g_error;

// value and derivative with respect to the interatomic distance
struct D1 {
  double v = 0, d = 0;
};
inline D1 operator+(D1 a, D1 b) { return {a.v + b.v, a.d + b.d}; }
inline D1 operator-(D1 a, D1 b) { return {a.v - b.v, a.d - b.d}; }
inline D1 operator*(D1 a, D1 b) { return {a.v * b.v, a.v * b.d + a.d * b.v}; }
inline D1 operator*(double s, D1 b) { return {s * b.v, s * b.d}; }
inline D1 operator+(double s, D1 b) { return {s + b.v, b.d}; }

// value and gradient with respect to the pair vector R = pos_b - pos_a
struct D3 {
  double v = 0, g[3] = {0, 0, 0};
  D3() = default;
  explicit D3(double x) : v(x) {}
};
inline D3 operator+(const D3& a, const D3& b) {
  D3 r(a.v + b.v);
  for (int k = 0; k < 3; ++k) r.g[k] = a.g[k] + b.g[k];
  return r;
}
inline D3 operator-(const D3& a, const D3& b) {
  D3 r(a.v - b.v);
  for (int k = 0; k < 3; ++k) r.g[k] = a.g[k] - b.g[k];
  return r;
}
inline D3 operator*(const D3& a, const D3& b) {
  D3 r(a.v * b.v);
  for (int k = 0; k < 3; ++k) r.g[k] = a.g[k] * b.v + a.v * b.g[k];
  return r;
}

constexpr int kInter = 8, kInterRight = 4, kInterLeft = 4;
constexpr double kDistFudge = 1.0, kDeltaR = 1e-5;

struct Elem {
  int Z = 0, nao = 0;
  double es = 0, ep = 0, U = 0, occ = 0, hd = 0;
  double w = 0;  // atomically resolved spin constant (W_pp for p elements, W_ss for s)
  bool has_hd = false, has_w = false;
  double W[2][2] = {};  // shell spin constants W(l, l'), l = s, p (SKAtom.h:52-66)
};

struct Pair {
  const DftbPairRaw* raw = nullptr;
  const DftbPairRaw* rev = nullptr;
  int nint = 0, n = 0;
  double grid = 0, rmax = 0;
  double c3[10] = {}, c4[10] = {}, c5[10] = {};
  double g1a = 0, g1b = 0, g2a = 0, g2b = 0;
  double dgab1a = 0, dgab1b = 0, dgab2a = 0, dgab2b = 0, dgba1a = 0, dgba1b = 0, dgba2a = 0, dgba2b = 0;
  // integral L at grid row i; L 8 and 9 are the completed p-s columns: the
  // reverse pair's s-p overlap and Hamiltonian integrals, negated (SKPair.cpp:79-89)
  double col(int L, int i) const {
    if (L < 8) return kDftbTable[raw->row0 + i][L];
    return -kDftbTable[rev->row0 + i][L == 8 ? 2 : 3];
  }
};

struct Params {
  const DftbSetRaw* set = nullptr;
  Elem elem[128];
  bool have[128] = {};
  int pair_index[128][128];
};

// Neville interpolation of every integral at grid coordinate x from row
// `start`, carrying the derivative with respect to the distance.
void interpolate(const Pair& p, double x, int start, D1 out[10]) {
  double xa[kInter];
  for (int i = 0; i < kInter; ++i) xa[i] = (double)(start + i);
  double dif = x - start;
  int ns0 = 0;
  for (int i = 0; i < kInter; ++i) {
    const double dift = std::fabs(x - xa[i]);
    if (dift < dif) {
      dif = dift;
      ns0 = i;
    }
  }
  for (int L = 0; L < p.nint; ++L) {
    D1 C[kInter], D[kInter];
    for (int i = 0; i < kInter; ++i) C[i] = D[i] = D1{p.col(L, start + i), 0.0};
    int ns = ns0;
    D1 y{p.col(L, start + ns), 0.0};
    --ns;
    for (int m = 1; m < kInter; ++m) {
      for (int i = 0; i <= kInter - 1 - m; ++i) {
        const double ho = xa[i] - x, hp = xa[i + m] - x;
        const D1 w = C[i + 1] - D[i];
        const D1 den{w.v / (ho - hp), w.d / (ho - hp)};
        D[i] = D1{hp, -1.0 / p.grid} * den;
        C[i] = D1{ho, -1.0 / p.grid} * den;
      }
      if (2 * (ns + 1) < kInter - m) {
        y = y + C[ns + 1];
      } else {
        y = y + D[ns];
        --ns;
      }
    }
    out[L] = y;
  }
}

void precompute_tail(Pair& p) {
  const int start = p.n - kInter;
  D1 t1[10], t2[10];
  interpolate(p, (double)(p.n - 1) - kDeltaR, start, t1);
  interpolate(p, (double)(p.n - 1) + kDeltaR, start, t2);
  for (int L = 0; L < p.nint; ++L) {
    const double yd0 = p.col(L, p.n - 1);
    const double yd1 = t1[L].d;
    const double yd2 = (t2[L].d - t1[L].d) / kDeltaR;
    const double dx1 = -yd1 * (kDistFudge / p.grid);
    const double dx2 = yd2 * (kDistFudge / p.grid) * (kDistFudge / p.grid);
    p.c3[L] = 10 * yd0 - 4 * dx1 + 0.5 * dx2;
    p.c4[L] = -15 * yd0 + 7 * dx1 - dx2;
    p.c5[L] = 6 * yd0 - 3 * dx1 + 0.5 * dx2;
  }
}

// Integrals at distance dist; returns 0 when all of them vanish.
int get_hs(const Pair& p, double dist, D1 I[10]) {
  for (int L = 0; L < 10; ++L) I[L] = D1{};
  if (dist < p.grid || dist > p.rmax) return 0;
  if (dist > p.n * p.grid) {
    const double dr = dist - p.rmax;
    const D1 xr{-dr / kDistFudge, 1.0};
    for (int L = 0; L < p.nint; ++L)
      I[L] = ((p.c5[L] * xr + D1{p.c4[L], 0}) * xr + D1{p.c3[L], 0}) * xr * xr * xr;
    return 1;
  }
  const double position = dist / p.grid - 1.0;
  const int ind = (int)position;
  const int start = ind >= p.n - kInterRight ? p.n - kInter : (ind < kInterLeft ? 0 : ind - kInterLeft + 1);
  interpolate(p, position, start, I);
  return 1;
}

void gamma_terms(const Elem& A, const Elem& B, Pair& p) {
  if (A.Z == B.Z) return;
  const double ta = A.U * 3.2, tb = B.U * 3.2, ta2 = ta * ta, tb2 = tb * tb;
  const double d = ta2 - tb2, e = tb2 - ta2;
  p.g1a = (tb2 * tb2 * ta) / (2.0 * d * d);
  p.g1b = (ta2 * ta2 * tb) / (2.0 * e * e);
  p.g2a = tb2 * tb2 * (tb2 - 3 * ta2) / (d * d * d);
  p.g2b = ta2 * ta2 * (ta2 - 3 * tb2) / (e * e * e);
  p.dgab1a = (tb2 * tb2 * tb2 + 3.0 * ta2 * tb2 * tb2) / (2.0 * d * d * d);
  p.dgab2a = (12.0 * ta2 * ta * tb2 * tb2) / (d * d * d * d);
  p.dgab1b = (2.0 * ta2 * ta * tb2 * tb) / (d * d * d);
  p.dgab2b = (12.0 * ta2 * ta2 * tb2 * tb) / (d * d * d * d);
  p.dgba1a = (ta2 * ta2 * ta2 + 3.0 * tb2 * ta2 * ta2) / (2.0 * e * e * e);
  p.dgba2a = (12.0 * tb2 * tb * ta2 * ta2) / (e * e * e * e);
  p.dgba1b = (2.0 * tb2 * tb * ta2 * ta) / (e * e * e);
  p.dgba2b = (12.0 * tb2 * tb2 * ta2 * ta) / (e * e * e * e);
}

std::vector<Pair> g_pairs_storage;

bool load(const char* set_name, const std::vector<int>& Zs, int order, Params& P, std::vector<Pair>& pairs) {
  for (auto& s : kDftbSetRaw)
    if (!std::strcmp(s.name, set_name)) P.set = &s;
  if (!P.set) {
    g_error = std::string("unknown DFTB parameter set ") + set_name;
    return false;
  }
  for (int i = 0; i < P.set->n_elem; ++i) {
    const DftbElemRaw& r = kDftbElemRaw[P.set->elem0 + i];
    Elem& e = P.elem[r.Z];
    e.Z = r.Z;
    e.nao = r.Z <= 2 ? 1 : (r.Z <= 10 ? 4 : 9);
    e.es = r.es;
    e.ep = r.ep;
    e.U = r.us;
    e.occ = r.fs + r.fp + r.fd;
    e.hd = r.hubbard_derivative;
    e.has_hd = r.has_hubbard_derivative != 0;
    e.w = e.nao == 1 ? r.wss : r.wpp;  // SKAtom.h:94-102
    e.has_w = r.has_spin != 0;
    e.W[0][0] = r.wss;
    e.W[0][1] = r.wsp;
    e.W[1][0] = r.wps;
    e.W[1][1] = r.wpp;
    P.have[r.Z] = true;
  }
  for (int z : Zs) {
    if (z < 0 || z >= 128 || !P.have[z]) {
      g_error = "no parameters for element Z=" + std::to_string(z);
      return false;
    }
    if (order == 3 && !P.elem[z].has_hd) {
      g_error = "no Hubbard derivative for element Z=" + std::to_string(z);
      return false;
    }
  }
  pairs.clear();
  for (auto& row : P.pair_index)
    for (int& v : row) v = -1;
  for (int i = 0; i < P.set->n_pair; ++i) {
    const DftbPairRaw& r = kDftbPairRaw[P.set->pair0 + i];
    P.pair_index[r.z1][r.z2] = (int)pairs.size();
    Pair p;
    p.raw = &r;
    pairs.push_back(p);
  }
  for (auto& p : pairs) {
    const int ri = P.pair_index[p.raw->z2][p.raw->z1];
    p.rev = &kDftbPairRaw[P.set->pair0 + ri];
    p.n = p.raw->rows;
    p.grid = p.raw->grid;
    p.rmax = p.grid * p.n + kDistFudge;
    const int na = P.elem[p.raw->z1].nao, nb = P.elem[p.raw->z2].nao;
    p.nint = na + nb == 2 ? 2 : (na + nb == 5 ? 4 : 10);
    precompute_tail(p);
    gamma_terms(P.elem[p.raw->z1], P.elem[p.raw->z2], p);
  }
  return true;
}

struct Mol {
  int nat = 0, nao = 0, nel = 0, nocc = 0, order = 2;
  int nalpha = 0, nbeta = 0;  // spin-polarised runs
  std::vector<int> Z, ao0, nao_of;
  std::vector<double> pos, core;
  Params P;
  std::vector<Pair> pairs;
  const Pair& pair(int za, int zb) const { return pairs[P.pair_index[za][zb]]; }
};

// S and H0 blocks of atoms a < b (rows on a, columns on b) with gradients
// with respect to R = pos_b - pos_a (ZeroOrderMatricesCalculator.cpp:92-232).
void pair_blocks(const Mol& M, int a, int b, D3 S[4][4], D3 H[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) S[i][j] = H[i][j] = D3(0.0);
  const int za = M.Z[a], zb = M.Z[b];
  const bool flip = za > zb;
  double R[3];
  for (int k = 0; k < 3; ++k) R[k] = flip ? M.pos[3 * a + k] - M.pos[3 * b + k] : M.pos[3 * b + k] - M.pos[3 * a + k];
  const Pair& p = flip ? M.pair(zb, za) : M.pair(za, zb);
  const double dist = std::sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
  D1 I1[10];
  if (get_hs(p, dist, I1) == 0) return;
  D3 I[10];
  for (int L = 0; L < p.nint; ++L) {
    I[L] = D3(I1[L].v);
    for (int k = 0; k < 3; ++k) I[L].g[k] = I1[L].d * R[k] / dist;
  }
  const int nF = M.P.elem[flip ? zb : za].nao, nS = M.P.elem[flip ? za : zb].nao;
  D3 me[2][4][4];
  for (int m = 0; m < 2; ++m) me[m][0][0] = I[m];
  if (nF + nS != 2) {
    D3 v[3], v2[3][3];
    for (int k = 0; k < 3; ++k) {
      // v_k = R_k / |R| with its gradient
      v[k] = D3(R[k] / dist);
      for (int l = 0; l < 3; ++l) v[k].g[l] = ((k == l ? 1.0 : 0.0) - R[k] * R[l] / (dist * dist)) / dist;
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) v2[i][j] = v[i] * v[j];
    for (int m = 0; m < 2; ++m) {
      for (int j = 0; j < 3; ++j) me[m][0][j + 1] = I[2 + m] * v[j];
      if (nF != 1 && nS != 1) {
        for (int j = 0; j < 3; ++j) me[m][j + 1][0] = I[8 + m] * v[j];
        for (int i = 0; i < 3; ++i) {
          me[m][i + 1][i + 1] = I[4 + m] * v2[i][i] + I[6 + m] * (D3(1.0) - v2[i][i]);
          for (int j = i + 1; j < 3; ++j) me[m][j + 1][i + 1] = me[m][i + 1][j + 1] = v2[i][j] * (I[4 + m] - I[6 + m]);
        }
      }
    }
  }
  const int nA = M.nao_of[a], nB = M.nao_of[b];
  for (int i = 0; i < nA; ++i)
    for (int j = 0; j < nB; ++j) {
      if (!flip) {
        S[i][j] = me[0][i][j];
        H[i][j] = me[1][i][j];
      } else {
        // computed for R' = -R: same value, opposite gradient
        S[i][j] = me[0][j][i];
        H[i][j] = me[1][j][i];
        for (int k = 0; k < 3; ++k) {
          S[i][j].g[k] = -S[i][j].g[k];
          H[i][j].g[k] = -H[i][j].g[k];
        }
      }
    }
}

// gamma_ab (DFTB2) as a function of the distance (SecondOrderFock.cpp:82-113)
D1 gamma2(const Mol& M, int a, int b, double R) {
  const Elem& A = M.P.elem[M.Z[a]];
  const Elem& B = M.P.elem[M.Z[b]];
  if (a == b) return D1{A.U, 0};
  const double ta = A.U * 3.2, tb = B.U * 3.2;
  const D1 r{R, 1.0};
  const D1 inv{1.0 / R, -1.0 / (R * R)};
  const D1 expa{std::exp(-ta * R), -ta * std::exp(-ta * R)};
  const D1 expb{std::exp(-tb * R), -tb * std::exp(-tb * R)};
  if (A.Z == B.Z) {
    const double ta2 = ta * ta;
    const D1 expr = inv + D1{0.6875 * ta, 0} + (0.1875 * ta2) * r + (0.02083333333333333 * ta * ta2) * (r * r);
    return inv - expa * expr;
  }
  const Pair& p = M.pair(A.Z, B.Z);
  const D1 terma = -1.0 * (expa * (D1{p.g1a, 0} - p.g2a * inv));
  const D1 termb = -1.0 * (expb * (D1{p.g1b, 0} - p.g2b * inv));
  return inv + terma + termb;
}

// gamma^h_ab, Gamma_ab and Gamma_ba (DFTB3, ThirdOrderFock.cpp:80-155)
void gamma3(const Mol& M, int a, int b, double Rv, D1& gam, D1& Gab, D1& Gba) {
  const Elem& A = M.P.elem[M.Z[a]];
  const Elem& B = M.P.elem[M.Z[b]];
  const double Ua = A.U, Ub = B.U;
  if (a == b) {
    gam = D1{Ua, 0};
    Gab = Gba = D1{0.5 * A.hd, 0};
    return;
  }
  const D1 R{Rv, 1.0};
  const D1 R2 = R * R;
  const D1 inv{1.0 / Rv, -1.0 / (Rv * Rv)};
  D1 h{1.0, 0}, dhdU{0, 0};
  if (A.Z == 1 || B.Z == 1) {
    const double zeta = 4.0;
    const double powerM1 = std::pow((Ua + Ub) / 2.0, zeta - 1.0);
    const double power = powerM1 * (Ua + Ub) / 2.0;
    h = D1{std::exp(-power * R2.v), -power * R2.d * std::exp(-power * R2.v)};
    dhdU = (-zeta / 2.0 * powerM1) * (R2 * h);
  }
  const double ta = Ua * 3.2, tb = Ub * 3.2;
  const D1 expa{std::exp(-ta * Rv), -ta * std::exp(-ta * Rv)};
  const D1 expb{std::exp(-tb * Rv), -tb * std::exp(-tb * Rv)};
  D1 S, dSda, dSdb;
  if (A.Z == B.Z) {
    const double ta2 = ta * ta;
    const D1 g = (1.0 / 48.0) * (48.0 * inv + D1{33.0 * ta, 0} + (9.0 * ta2) * R + (ta * ta2) * R2);
    const D1 dgda = (1.0 / 48.0) * (D1{33.0, 0} + (18.0 * ta) * R + (3.0 * ta2) * R2);
    S = expa * g;
    dSda = dSdb = expa * (dgda - R * g);
  } else {
    const Pair& p = M.pair(A.Z, B.Z);
    const D1 fab = D1{p.g1a, 0} - p.g2a * inv;
    const D1 fba = D1{p.g1b, 0} - p.g2b * inv;
    const D1 dfabda = D1{-p.dgab1a, 0} - p.dgab2a * inv;
    const D1 dfbadb = D1{-p.dgba1a, 0} - p.dgba2a * inv;
    const D1 dfabdb = D1{p.dgab1b, 0} + p.dgab2b * inv;
    const D1 dfbada = D1{p.dgba1b, 0} + p.dgba2b * inv;
    S = expa * fab + expb * fba;
    dSda = expa * (dfabda - R * fab) + expb * dfbada;
    dSdb = expb * (dfbadb - R * fba) + expa * dfabdb;
  }
  const D1 dgdUa = -1.0 * (3.2 * (dSda * h) + S * dhdU);
  const D1 dgdUb = -1.0 * (3.2 * (dSdb * h) + S * dhdU);
  gam = inv - S * h;
  Gab = A.hd * dgdUa;
  Gba = B.hd * dgdUb;
}

// Repulsion energy of the (za, zb) spline at r and dE/dr (PairwiseRepulsion.cpp:40-71)
void repulsion(const Pair& p, double r, double& E, double& dE) {
  const DftbPairRaw& q = *p.raw;
  E = dE = 0;
  if (r > q.cutoff) return;
  const auto* sp = &kDftbSplineRaw[q.spline0];
  if (r < sp[0].start) {
    E = std::exp(-q.a1 * r + q.a2) + q.a3;
    dE = -q.a1 * std::exp(-q.a1 * r + q.a2);
    return;
  }
  int i = (int)((r - sp[0].start) / (q.cutoff - sp[0].start) * q.n_spline);
  if (i >= q.n_spline) i = q.n_spline - 1;
  if (sp[i].start > r) {
    while (sp[--i].start > r) {
    }
  } else if (sp[i].end < r) {
    while (sp[++i].end < r) {
    }
  }
  const double dr = r - sp[i].start;
  double c4 = 0, c5 = 0;
  if (i == q.n_spline - 1) {
    c4 = q.c4;
    c5 = q.c5;
  }
  E = sp[i].c0 + dr * (sp[i].c1 + dr * (sp[i].c2 + dr * (sp[i].c3 + dr * (c4 + dr * c5))));
  dE = sp[i].c1 + dr * (2 * sp[i].c2 + dr * (3 * sp[i].c3 + dr * (4 * c4 + dr * 5 * c5)));
}

struct State {
  std::vector<double> H0, S, P, F, C, eps, q, gam, Gam, shift;
  double e_el = 0, e_rep = 0;
  int iterations = 0;
  bool converged = false;
};

double dist_ab(const Mol& M, int a, int b) {
  double s = 0;
  for (int k = 0; k < 3; ++k) {
    const double d = M.pos[3 * b + k] - M.pos[3 * a + k];
    s += d * d;
  }
  return std::sqrt(s);
}

void build_static(const Mol& M, State& st) {
  const int N = M.nao, n = M.nat;
  st.H0.assign((size_t)N * N, 0);
  st.S.assign((size_t)N * N, 0);
  for (int a = 0; a < n; ++a) {
    const Elem& e = M.P.elem[M.Z[a]];
    for (int i = 0; i < M.nao_of[a]; ++i) {
      st.H0[(size_t)(M.ao0[a] + i) * N + M.ao0[a] + i] = i == 0 ? e.es : e.ep;
      st.S[(size_t)(M.ao0[a] + i) * N + M.ao0[a] + i] = 1.0;
    }
  }
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      D3 S[4][4], H[4][4];
      pair_blocks(M, a, b, S, H);
      for (int i = 0; i < M.nao_of[a]; ++i)
        for (int j = 0; j < M.nao_of[b]; ++j) {
          const size_t u = M.ao0[a] + i, v = M.ao0[b] + j;
          st.S[u * N + v] = st.S[v * N + u] = S[i][j].v;
          st.H0[u * N + v] = st.H0[v * N + u] = H[i][j].v;
        }
    }
  st.gam.assign((size_t)n * n, 0);
  st.Gam.assign((size_t)n * n, 0);
  for (int a = 0; a < n; ++a)
    for (int b = a; b < n; ++b) {
      const double R = a == b ? 0.0 : dist_ab(M, a, b);
      if (M.order == 3) {
        D1 g, Gab, Gba;
        gamma3(M, a, b, R, g, Gab, Gba);
        st.gam[a * n + b] = st.gam[b * n + a] = g.v;
        st.Gam[a * n + b] = Gab.v;
        st.Gam[b * n + a] = Gba.v;
      } else {
        const D1 g = gamma2(M, a, b, R);
        st.gam[a * n + b] = st.gam[b * n + a] = g.v;
      }
    }
}

// Mulliken charges q_a = Z_a - sum_{mu in a} (P S)_mu,mu
void charges(const Mol& M, const State& st, std::vector<double>& q) {
  const int N = M.nao;
  q.assign(M.nat, 0);
  for (int a = 0; a < M.nat; ++a) {
    double pop = 0;
    for (int i = 0; i < M.nao_of[a]; ++i) {
      const size_t u = M.ao0[a] + i;
      for (int v = 0; v < N; ++v) pop += st.P[u * N + v] * st.S[(size_t)v * N + u];
    }
    q[a] = M.core[a] - pop;
  }
}

// Atom shifts: HXoverS(mu in a, nu in b) = shift_ab; DFTB2: -1/2 sum_i (g_ai + g_bi) q_i;
// DFTB3 adds 1/6 sum_i q_i (2 (q_a G_ai + q_b G_bi) + q_i (G_ia + G_ib)).
double shift_ab(const Mol& M, const State& st, int a, int b) {
  const int n = M.nat;
  double h1 = 0, h2 = 0;
  for (int i = 0; i < n; ++i) {
    h1 -= (st.gam[a * n + i] + st.gam[b * n + i]) * st.q[i];
    if (M.order == 3)
      h2 += st.q[i] * (2 * (st.q[a] * st.Gam[a * n + i] + st.q[b] * st.Gam[b * n + i]) +
                       st.q[i] * (st.Gam[i * n + a] + st.Gam[i * n + b]));
  }
  return 0.5 * h1 + h2 / 6.0;
}

void fock(const Mol& M, State& st) {
  const int N = M.nao, n = M.nat;
  charges(M, st, st.q);
  st.F = st.H0;
  st.shift.assign((size_t)N * N, 0);
  for (int a = 0; a < n; ++a)
    for (int b = a; b < n; ++b) {
      const double s = shift_ab(M, st, a, b);
      for (int i = 0; i < M.nao_of[a]; ++i)
        for (int j = 0; j < M.nao_of[b]; ++j) {
          const size_t u = M.ao0[a] + i, v = M.ao0[b] + j;
          st.shift[u * N + v] = st.shift[v * N + u] = s;
          st.F[u * N + v] = st.H0[u * N + v] + st.S[u * N + v] * s;
          st.F[v * N + u] = st.F[u * N + v];
        }
    }
}

double electronic_energy(const Mol& M, const State& st) {
  const int N = M.nao, n = M.nat;
  double e = 0;
  for (size_t k = 0; k < (size_t)N * N; ++k) e += st.H0[k] * st.P[k];
  if (M.order == 3) {
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        e += 0.5 * st.q[a] * st.q[b] * st.gam[a * n + b];
        e -= st.q[a] * st.q[a] * st.q[b] * st.Gam[a * n + b] / 3.0;
      }
  } else {
    for (int a = 0; a < n; ++a) {
      e += 0.5 * st.q[a] * st.q[a] * st.gam[a * n + a];
      for (int b = a + 1; b < n; ++b) e += st.q[a] * st.q[b] * st.gam[a * n + b];
    }
  }
  return e;
}

std::vector<double> matmul(int N, const std::vector<double>& A, const std::vector<double>& B) {
  std::vector<double> C((size_t)N * N, 0);
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < N; ++k) {
      const double a = A[(size_t)i * N + k];
      if (a == 0) continue;
      for (int j = 0; j < N; ++j) C[(size_t)i * N + j] += a * B[(size_t)k * N + j];
    }
  return C;
}

bool scf(const Mol& M, State& st, double scc, double rmsd, int max_iter) {
  const int N = M.nao;
  build_static(M, st);
  // X = S^-1/2 (Loewdin)
  std::vector<double> sw, sv;
  if (!oracle_la::eigh(N, st.S, sw, sv)) {
    g_error = "overlap diagonalisation failed";
    return false;
  }
  std::vector<double> X((size_t)N * N, 0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0;
      for (int k = 0; k < N; ++k) s += sv[(size_t)i * N + k] * sv[(size_t)j * N + k] / std::sqrt(sw[k]);
      X[(size_t)i * N + j] = s;
    }
  // density guess: neutral atoms, core charge spread over the atom's AOs
  st.P.assign((size_t)N * N, 0);
  for (int a = 0; a < M.nat; ++a)
    for (int i = 0; i < M.nao_of[a]; ++i)
      st.P[(size_t)(M.ao0[a] + i) * N + M.ao0[a] + i] = M.core[a] / M.nao_of[a];
  std::vector<std::vector<double>> hF, hE;
  double Eold = 0;
  st.converged = false;
  for (int it = 1; it <= max_iter; ++it) {
    st.iterations = it;
    fock(M, st);
    const double E = electronic_energy(M, st);
    // Pulay DIIS on FPS - SPF
    const auto FP = matmul(N, st.F, st.P);
    const auto FPS = matmul(N, FP, st.S);
    std::vector<double> err((size_t)N * N);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) err[(size_t)i * N + j] = FPS[(size_t)i * N + j] - FPS[(size_t)j * N + i];
    hF.push_back(st.F);
    hE.push_back(err);
    if (hF.size() > 8) {
      hF.erase(hF.begin());
      hE.erase(hE.begin());
    }
    std::vector<double> Fx = st.F;
    const int m = (int)hF.size();
    if (m >= 2) {
      std::vector<double> B((size_t)(m + 1) * (m + 1), 0), rhs(m + 1, 0);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          double s = 0;
          for (size_t k = 0; k < err.size(); ++k) s += hE[i][k] * hE[j][k];
          B[i * (m + 1) + j] = s;
        }
      for (int i = 0; i < m; ++i) B[i * (m + 1) + m] = B[m * (m + 1) + i] = -1;
      rhs[m] = -1;
      if (oracle_la::solve_dense(m + 1, B, rhs)) {
        std::fill(Fx.begin(), Fx.end(), 0.0);
        for (int i = 0; i < m; ++i)
          for (size_t k = 0; k < Fx.size(); ++k) Fx[k] += rhs[i] * hF[i][k];
      }
    }
    // generalised eigenproblem through the orthogonal basis
    const auto Fp = matmul(N, X, matmul(N, Fx, X));
    std::vector<double> w, v;
    if (!oracle_la::eigh(N, Fp, w, v)) {
      g_error = "Fock diagonalisation failed";
      return false;
    }
    st.C = matmul(N, X, v);
    st.eps = w;
    std::vector<double> Pn((size_t)N * N, 0);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double s = 0;
        for (int k = 0; k < M.nocc; ++k) s += st.C[(size_t)i * N + k] * st.C[(size_t)j * N + k];
        Pn[(size_t)i * N + j] = 2 * s;
      }
    double d2 = 0;
    for (size_t k = 0; k < Pn.size(); ++k) d2 += (Pn[k] - st.P[k]) * (Pn[k] - st.P[k]);
    const double rms = std::sqrt(d2 / ((double)N * N));
    const bool dE_ok = it > 1 && std::fabs(E - Eold) < scc;
    Eold = E;
    st.P = Pn;
    if (dE_ok && rms < rmsd) {
      st.converged = true;
      break;
    }
  }
  fock(M, st);
  st.e_el = electronic_energy(M, st);
  st.e_rep = 0;
  for (int a = 0; a < M.nat; ++a)
    for (int b = a + 1; b < M.nat; ++b) {
      double E, dE;
      repulsion(M.pair(M.Z[a], M.Z[b]), dist_ab(M, a, b), E, dE);
      st.e_rep += E;
    }
  return true;
}

// Nuclear gradient with the overlap multiplier Wm (energy-weighted density
// minus the density-dependent parts of the Fock matrix that multiply S).
void gradient_with(const Mol& M, const State& st, const std::vector<double>& Wm, std::vector<double>& g) {
  const int N = M.nao, n = M.nat;
  g.assign(3 * (size_t)n, 0);
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      double d[3] = {0, 0, 0};
      D3 S[4][4], H[4][4];
      pair_blocks(M, a, b, S, H);
      for (int i = 0; i < M.nao_of[a]; ++i)
        for (int j = 0; j < M.nao_of[b]; ++j) {
          const size_t u = M.ao0[a] + i, v = M.ao0[b] + j;
          for (int k = 0; k < 3; ++k)
            d[k] += 2 * (st.P[u * N + v] * H[i][j].g[k] - Wm[u * N + v] * S[i][j].g[k]);
        }
      double R[3], r = 0;
      for (int k = 0; k < 3; ++k) {
        R[k] = M.pos[3 * b + k] - M.pos[3 * a + k];
        r += R[k] * R[k];
      }
      r = std::sqrt(r);
      const double qa = st.q[a], qb = st.q[b];
      double coef;  // multiplies the unit vector R / r
      if (M.order == 3) {
        D1 gam, Gab, Gba;
        gamma3(M, a, b, r, gam, Gab, Gba);
        // dE/dR_b along R/r as the reference assembles it: q_a q_b gamma' +
        // q_a q_b / 3 (q_b Gamma_ba' - q_a Gamma_ab').  (The derivative of the
        // energy term -1/3 q_a q_b^2 Gamma_ba carries the opposite sign on
        // Gamma_ba'; the reference's pair term is kept for parity.)
        coef = qa * qb * gam.d + (qa * qb / 3.0) * (qb * Gba.d - qa * Gab.d);
      } else {
        coef = qa * qb * gamma2(M, a, b, r).d;
      }
      double E, dE;
      repulsion(M.pair(M.Z[a], M.Z[b]), r, E, dE);
      coef += dE;
      for (int k = 0; k < 3; ++k) {
        d[k] += coef * R[k] / r;
        g[3 * b + k] += d[k];
        g[3 * a + k] -= d[k];
      }
    }
}

void gradient(const Mol& M, const State& st, std::vector<double>& g) {
  const int N = M.nao;
  // W = 2 sum_occ eps_i C_i C_i^T and the overlap multiplier W - HXoverS o P
  std::vector<double> Wm((size_t)N * N, 0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0;
      for (int k = 0; k < M.nocc; ++k) s += st.eps[k] * st.C[(size_t)i * N + k] * st.C[(size_t)j * N + k];
      Wm[(size_t)i * N + j] = 2 * s - st.shift[(size_t)i * N + j] * st.P[(size_t)i * N + j];
    }
  gradient_with(M, st, Wm, g);
}

bool setup(const char* set, int order, int nat, const int* Z, const double* xyz, int charge, Mol& M,
           int multiplicity = 0) {
  M = Mol();
  M.order = order;
  M.nat = nat;
  M.Z.assign(Z, Z + nat);
  M.pos.assign(xyz, xyz + 3 * nat);
  if (!load(set, M.Z, order, M.P, M.pairs)) return false;
  double occ = 0;
  for (int a = 0; a < nat; ++a) {
    const Elem& e = M.P.elem[Z[a]];
    if (e.nao > 4) {
      g_error = "elements with d orbitals are outside the s/p DFTB path";
      return false;
    }
    M.ao0.push_back(M.nao);
    M.nao_of.push_back(e.nao);
    M.nao += e.nao;
    M.core.push_back(e.occ);
    occ += e.occ;
  }
  M.nel = (int)std::lround(occ) - charge;
  if (multiplicity > 0) {
    const int na2 = M.nel + multiplicity - 1;
    if (M.nel < 0 || (na2 & 1) || M.nel - (multiplicity - 1) < 0 || na2 / 2 > M.nao) {
      g_error = "electron count and spin multiplicity do not match";
      return false;
    }
    M.nalpha = na2 / 2;
    M.nbeta = M.nel - M.nalpha;
    M.nocc = M.nalpha;
    return true;
  }
  if (M.nel < 0 || (M.nel & 1)) {
    g_error = "restricted DFTB needs an even electron count";
    return false;
  }
  M.nocc = M.nel / 2;
  return true;
}

// ---------------------------------------------------------------------------
// Spin-polarised DFTB (Utils/SDFTB.cpp:64-293, Utils/ScfFock.cpp:50-103)
// ---------------------------------------------------------------------------
// Shell spin populations pdif_{a,l} = sum_{mu in (a, l)} sum_nu (Pa - Pb)_mu,nu S_mu,nu,
// shell shifts eps_{a,l} = sum_l' W_a(l, l') pdif_{a,l'}, the spin contribution
// spinC_mu,nu = 1/2 (eps_{a(mu),l(mu)} + eps_{b(nu),l(nu)}) that enters
// F_alpha = F + spinC o S and F_beta = F - spinC o S, and the energy
// 1/2 sum_a sum_{l,l'} pdif_{a,l} W_a(l, l') pdif_{a,l'}.
double spin_terms(const Mol& M, const std::vector<double>& Pa, const std::vector<double>& Pb,
                  const std::vector<double>& S, std::vector<double>& spinC) {
  const int N = M.nao, n = M.nat;
  std::vector<double> pdif(2 * (size_t)n, 0.0), eps(2 * (size_t)n, 0.0);
  std::vector<int> atom_of(N), shell_of(N);
  for (int a = 0; a < n; ++a)
    for (int i = 0; i < M.nao_of[a]; ++i) {
      atom_of[M.ao0[a] + i] = a;
      shell_of[M.ao0[a] + i] = i == 0 ? 0 : 1;
    }
  for (int u = 0; u < N; ++u) {
    double s = 0;
    for (int v = 0; v < N; ++v) s += (Pa[(size_t)u * N + v] - Pb[(size_t)u * N + v]) * S[(size_t)u * N + v];
    pdif[2 * atom_of[u] + shell_of[u]] += s;
  }
  double e = 0;
  for (int a = 0; a < n; ++a) {
    const Elem& el = M.P.elem[M.Z[a]];
    for (int l = 0; l < 2; ++l)
      for (int k = 0; k < 2; ++k) {
        eps[2 * a + l] += el.W[l][k] * pdif[2 * a + k];
        e += 0.5 * pdif[2 * a + l] * el.W[l][k] * pdif[2 * a + k];
      }
  }
  spinC.assign((size_t)N * N, 0.0);
  for (int u = 0; u < N; ++u)
    for (int v = 0; v < N; ++v)
      spinC[(size_t)u * N + v] = 0.5 * (eps[2 * atom_of[u] + shell_of[u]] + eps[2 * atom_of[v] + shell_of[v]]);
  return e;
}

struct SpinState {
  std::vector<double> Pa, Pb, Ca, Cb, epsa, epsb, spinC;
  double e_spin = 0;
};

// Unrestricted SCC: both spins from the restricted Fock matrix of the total
// density plus / minus the spin term; Pulay DIIS on the stacked commutators
// (F_s P_s S - S P_s F_s) with one set of coefficients; start P_a = P_b = P0 / 2.
bool scf_uhf(const Mol& M, State& st, SpinState& ss, double scc, double rmsd, int max_iter) {
  const int N = M.nao;
  const size_t NN = (size_t)N * N;
  build_static(M, st);
  std::vector<double> sw, sv;
  if (!oracle_la::eigh(N, st.S, sw, sv)) {
    g_error = "overlap diagonalisation failed";
    return false;
  }
  std::vector<double> X(NN, 0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0;
      for (int k = 0; k < N; ++k) s += sv[(size_t)i * N + k] * sv[(size_t)j * N + k] / std::sqrt(sw[k]);
      X[(size_t)i * N + j] = s;
    }
  st.P.assign(NN, 0);
  for (int a = 0; a < M.nat; ++a)
    for (int i = 0; i < M.nao_of[a]; ++i)
      st.P[(size_t)(M.ao0[a] + i) * N + M.ao0[a] + i] = M.core[a] / M.nao_of[a];
  ss.Pa.assign(NN, 0);
  ss.Pb.assign(NN, 0);
  for (size_t k = 0; k < NN; ++k) ss.Pa[k] = ss.Pb[k] = 0.5 * st.P[k];
  std::vector<std::vector<double>> hFa, hFb, hE;
  std::vector<double> Fa(NN), Fb(NN);
  auto commutator = [&](const std::vector<double>& F, const std::vector<double>& P, double* out) {
    const auto FPS = matmul(N, matmul(N, F, P), st.S);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) out[(size_t)i * N + j] = FPS[(size_t)i * N + j] - FPS[(size_t)j * N + i];
  };
  auto solve_spin = [&](const std::vector<double>& Fx, int nocc, std::vector<double>& C, std::vector<double>& eps,
                        std::vector<double>& Pn) -> bool {
    const auto Fp = matmul(N, X, matmul(N, Fx, X));
    std::vector<double> v;
    if (!oracle_la::eigh(N, Fp, eps, v)) return false;
    C = matmul(N, X, v);
    Pn.assign(NN, 0);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) {
        double s = 0;
        for (int k = 0; k < nocc; ++k) s += C[(size_t)i * N + k] * C[(size_t)j * N + k];
        Pn[(size_t)i * N + j] = s;
      }
    return true;
  };
  double Eold = 0;
  st.converged = false;
  for (int it = 1; it <= max_iter; ++it) {
    st.iterations = it;
    fock(M, st);
    const double E = electronic_energy(M, st) + spin_terms(M, ss.Pa, ss.Pb, st.S, ss.spinC);
    for (size_t k = 0; k < NN; ++k) {
      Fa[k] = st.F[k] + ss.spinC[k] * st.S[k];
      Fb[k] = st.F[k] - ss.spinC[k] * st.S[k];
    }
    std::vector<double> err(2 * NN);
    commutator(Fa, ss.Pa, err.data());
    commutator(Fb, ss.Pb, err.data() + NN);
    hFa.push_back(Fa);
    hFb.push_back(Fb);
    hE.push_back(err);
    if (hE.size() > 8) {
      hFa.erase(hFa.begin());
      hFb.erase(hFb.begin());
      hE.erase(hE.begin());
    }
    std::vector<double> Fxa = Fa, Fxb = Fb;
    const int m = (int)hE.size();
    if (m >= 2) {
      std::vector<double> B((size_t)(m + 1) * (m + 1), 0), rhs(m + 1, 0);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          double s = 0;
          for (size_t k = 0; k < err.size(); ++k) s += hE[i][k] * hE[j][k];
          B[i * (m + 1) + j] = s;
        }
      for (int i = 0; i < m; ++i) B[i * (m + 1) + m] = B[m * (m + 1) + i] = -1;
      rhs[m] = -1;
      if (oracle_la::solve_dense(m + 1, B, rhs)) {
        std::fill(Fxa.begin(), Fxa.end(), 0.0);
        std::fill(Fxb.begin(), Fxb.end(), 0.0);
        for (int i = 0; i < m; ++i)
          for (size_t k = 0; k < NN; ++k) {
            Fxa[k] += rhs[i] * hFa[i][k];
            Fxb[k] += rhs[i] * hFb[i][k];
          }
      }
    }
    std::vector<double> Pna, Pnb;
    if (!solve_spin(Fxa, M.nalpha, ss.Ca, ss.epsa, Pna) || !solve_spin(Fxb, M.nbeta, ss.Cb, ss.epsb, Pnb)) {
      g_error = "Fock diagonalisation failed";
      return false;
    }
    double da = 0, db = 0;
    for (size_t k = 0; k < NN; ++k) {
      da += (Pna[k] - ss.Pa[k]) * (Pna[k] - ss.Pa[k]);
      db += (Pnb[k] - ss.Pb[k]) * (Pnb[k] - ss.Pb[k]);
    }
    const double rms = std::sqrt(std::max(da, db) / (double)NN);
    ss.Pa.swap(Pna);
    ss.Pb.swap(Pnb);
    for (size_t k = 0; k < NN; ++k) st.P[k] = ss.Pa[k] + ss.Pb[k];
    const bool dE_ok = it > 1 && std::fabs(E - Eold) < scc;
    Eold = E;
    if (dE_ok && rms < rmsd) {
      st.converged = true;
      break;
    }
  }
  fock(M, st);
  ss.e_spin = spin_terms(M, ss.Pa, ss.Pb, st.S, ss.spinC);
  st.e_el = electronic_energy(M, st) + ss.e_spin;
  // orbital energies of the final spin Fock matrices
  for (size_t k = 0; k < NN; ++k) {
    Fa[k] = st.F[k] + ss.spinC[k] * st.S[k];
    Fb[k] = st.F[k] - ss.spinC[k] * st.S[k];
  }
  std::vector<double> tmp;
  solve_spin(Fa, M.nalpha, ss.Ca, ss.epsa, tmp);
  solve_spin(Fb, M.nbeta, ss.Cb, ss.epsb, tmp);
  st.e_rep = 0;
  for (int a = 0; a < M.nat; ++a)
    for (int b = a + 1; b < M.nat; ++b) {
      double E, dE;
      repulsion(M.pair(M.Z[a], M.Z[b]), dist_ab(M, a, b), E, dE);
      st.e_rep += E;
    }
  return true;
}

// Unrestricted gradient: W = sum_s sum_{occ s} eps C C^T, and the overlap
// multiplier W - HXoverS o P - spinC o (Pa - Pb) (SDFTB.cpp:60-83 adds
// 2 (Pa - Pb) spinC dS per atom pair).
void gradient_uhf(const Mol& M, const State& st, const SpinState& ss, std::vector<double>& g) {
  const int N = M.nao;
  std::vector<double> Wm((size_t)N * N, 0);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double s = 0;
      for (int k = 0; k < M.nalpha; ++k) s += ss.epsa[k] * ss.Ca[(size_t)i * N + k] * ss.Ca[(size_t)j * N + k];
      for (int k = 0; k < M.nbeta; ++k) s += ss.epsb[k] * ss.Cb[(size_t)i * N + k] * ss.Cb[(size_t)j * N + k];
      const size_t ij = (size_t)i * N + j;
      Wm[ij] = s - st.shift[ij] * st.P[ij] - ss.spinC[ij] * (ss.Pa[ij] - ss.Pb[ij]);
    }
  gradient_with(M, st, Wm, g);
}

// Linear-response TD-DFTB (restricted reference, singlets or triplets, the
// full Casida form, not TDA) for the nroots lowest excitations.
//   transition charges (TransitionChargesCalculator.h:138-165):
//     q_A^{ia} = 1/2 sum_{mu on A} (C_mu,i (SC)_mu,a + C_mu,a (SC)_mu,i)
//   Casida matrix (TDDFTBSigmaVectorEvaluator.cpp:40-110, factor 4 for a
//   restricted reference, TDDFTBSigmaVectorEvaluator.h:118-120):
//     Omega_{ia,jb} = delta Delta_ia^2 + 4 sqrt(Delta_ia) K_{ia,jb} sqrt(Delta_jb)
//     K = q^T gamma q (singlets), q^T diag(W_A) q (triplets)
//   omega_I = sqrt(eigenvalue), c_ia = sqrt(Delta_ia / omega_I) F_ia
//   (TDDFTBEigenvalueSolver.h:150-197)
//   transition dipole (DFTBDipoleMatrixCalculator.cpp:60-84 for the MO dipole
//   matrix D_ia = sum_A q_A^{ia} R_A; the restricted singlet factor sqrt(2)
//   of the spin-adapted transition density, restated for the un-vendored
//   Utils::TransitionDipoleCalculator): mu_I = sqrt(2) sum_ia c_ia D_ia.
// The eigenproblem is solved densely up to 2000 transitions; above that by a
// matrix-free Davidson iteration on Omega (the reference's Davidson lives in
// the un-vendored scine_utilities; converged eigenpairs do not depend on it).
//
// Lowest nroots eigenpairs of Omega = diag(delta^2) + 4 sqrt(delta) qG q^T
// sqrt(delta) without forming it: products through the atoms (dim * nat),
// unit start vectors of the smallest diagonal entries, diagonal
// preconditioner, Gram-Schmidt twice, restart to the Ritz vectors when the
// subspace is full, residual norm 1e-10 (Davidson, J. Comput. Phys. 17, 1975).
static int g_dense_casida_limit = 2000;  // transitions up to which Omega is diagonalised densely

static bool davidson_lowest(int dim, int nat, int nroots, const std::vector<double>& delta,
                            const std::vector<double>& q, const std::vector<double>& qG, std::vector<double>& w_out,
                            std::vector<double>& X_out) {
  auto apply = [&](const double* x, double* y) {
    std::vector<double> t(nat, 0.0);
    for (int k = 0; k < dim; ++k) {
      const double sk = std::sqrt(delta[k]) * x[k];
      for (int B = 0; B < nat; ++B) t[B] += qG[(size_t)k * nat + B] * sk;
    }
    for (int k = 0; k < dim; ++k) {
      double s = 0;
      for (int B = 0; B < nat; ++B) s += q[(size_t)k * nat + B] * t[B];
      y[k] = delta[k] * delta[k] * x[k] + 4.0 * std::sqrt(delta[k]) * s;
    }
  };
  const int maxsub = std::min(dim, std::max(8 * nroots, 32));
  std::vector<std::vector<double>> V, AV;
  std::vector<int> idx(dim);
  for (int k = 0; k < dim; ++k) idx[k] = k;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return delta[a] < delta[b] || (delta[a] == delta[b] && a < b); });
  auto add_vector = [&](std::vector<double> x) -> bool {
    double n0 = 0;
    for (double xk : x) n0 += xk * xk;
    n0 = std::sqrt(n0);
    if (!(n0 > 0)) return false;
    for (double& xk : x) xk /= n0;  // unit length first: the test below is relative
    for (int pass = 0; pass < 2; ++pass)
      for (const auto& v : V) {
        double d = 0;
        for (int k = 0; k < dim; ++k) d += v[k] * x[k];
        for (int k = 0; k < dim; ++k) x[k] -= d * v[k];
      }
    double nrm = 0;
    for (double xk : x) nrm += xk * xk;
    nrm = std::sqrt(nrm);
    if (nrm < 1e-6) return false;  // (almost) inside the subspace already
    for (double& xk : x) xk /= nrm;
    std::vector<double> ax(dim);
    apply(x.data(), ax.data());
    V.push_back(std::move(x));
    AV.push_back(std::move(ax));
    return true;
  };
  for (int j = 0; j < std::min(dim, 2 * nroots); ++j) {
    std::vector<double> e(dim, 0.0);
    e[idx[j]] = 1.0;
    add_vector(e);
  }
  for (int iter = 0; iter < 500; ++iter) {
    const int m = (int)V.size();
    std::vector<double> Hs((size_t)m * m);
    for (int a = 0; a < m; ++a)
      for (int b = 0; b <= a; ++b) {
        double s = 0;
        for (int k = 0; k < dim; ++k) s += V[a][k] * AV[b][k];
        Hs[(size_t)a * m + b] = Hs[(size_t)b * m + a] = s;
      }
    std::vector<double> th, U;
    if (!oracle_la::eigh(m, Hs, th, U)) return false;
    // Ritz vectors and residuals of the lowest nroots
    std::vector<std::vector<double>> X(nroots, std::vector<double>(dim, 0.0)), R(nroots, std::vector<double>(dim, 0.0));
    double rmax = 0;
    for (int I = 0; I < nroots; ++I) {
      for (int a = 0; a < m; ++a) {
        const double u = U[(size_t)a * m + I];
        for (int k = 0; k < dim; ++k) {
          X[I][k] += u * V[a][k];
          R[I][k] += u * AV[a][k];
        }
      }
      double rn = 0;
      for (int k = 0; k < dim; ++k) {
        R[I][k] -= th[I] * X[I][k];
        rn += R[I][k] * R[I][k];
      }
      rmax = std::max(rmax, std::sqrt(rn));
    }
    if (rmax < 1e-10) {
      w_out.assign(th.begin(), th.begin() + nroots);
      X_out.assign((size_t)dim * nroots, 0.0);
      for (int I = 0; I < nroots; ++I)
        for (int k = 0; k < dim; ++k) X_out[(size_t)k * nroots + I] = X[I][k];
      return true;
    }
    if (m + nroots > maxsub) {  // restart from the Ritz vectors
      V.clear();
      AV.clear();
      for (int I = 0; I < nroots; ++I) add_vector(X[I]);
    }
    int added = 0;
    for (int I = 0; I < nroots; ++I) {
      double rn = 0;
      for (double r : R[I]) rn += r * r;
      if (std::sqrt(rn) < 1e-10) continue;
      std::vector<double> t(dim);
      for (int k = 0; k < dim; ++k) {
        double den = th[I] - delta[k] * delta[k];
        if (std::fabs(den) < 1e-8) den = den < 0 ? -1e-8 : 1e-8;
        t[k] = R[I][k] / den;
      }
      if (add_vector(t)) ++added;
    }
    if (!added) return false;
  }
  return false;
}

bool tddftb(const Mol& M, const State& st, int triplet, int nroots, std::vector<double>& omega,
            std::vector<double>& dip) {
  const int N = M.nao, no = M.nocc, nv = N - no, nat = M.nat;
  const int dim = no * nv;
  if (dim == 0) {
    g_error = "no occupied-virtual transitions";
    return false;
  }
  if (nroots > dim) nroots = dim;
  const auto SC = matmul(N, st.S, st.C);
  std::vector<int> atom_of(N);
  for (int a = 0; a < nat; ++a)
    for (int i = 0; i < M.nao_of[a]; ++i) atom_of[M.ao0[a] + i] = a;
  // q[k][A] with k = i * nv + a
  std::vector<double> q((size_t)dim * nat, 0.0), delta(dim);
  for (int i = 0; i < no; ++i)
    for (int a = 0; a < nv; ++a) {
      const int k = i * nv + a, av = no + a;
      delta[k] = st.eps[av] - st.eps[i];
      for (int mu = 0; mu < N; ++mu) {
        const double v = 0.5 * (st.C[(size_t)mu * N + i] * SC[(size_t)mu * N + av] +
                                st.C[(size_t)mu * N + av] * SC[(size_t)mu * N + i]);
        q[(size_t)k * nat + atom_of[mu]] += v;
      }
    }
  // coupling matrix of the atoms
  std::vector<double> G((size_t)nat * nat, 0.0);
  for (int A = 0; A < nat; ++A)
    for (int B = 0; B < nat; ++B) {
      if (triplet) {
        if (A == B) {
          const Elem& e = M.P.elem[M.Z[A]];
          if (!e.has_w) {
            g_error = "no spin constant for element Z=" + std::to_string(M.Z[A]);
            return false;
          }
          G[(size_t)A * nat + A] = e.w;
        }
      } else {
        G[(size_t)A * nat + B] = st.gam[(size_t)A * nat + B];
      }
    }
  std::vector<double> qG((size_t)dim * nat, 0.0);
  for (int k = 0; k < dim; ++k)
    for (int B = 0; B < nat; ++B) {
      double s = 0;
      for (int A = 0; A < nat; ++A) s += q[(size_t)k * nat + A] * G[(size_t)A * nat + B];
      qG[(size_t)k * nat + B] = s;
    }
  std::vector<double> w, V;
  int ldv = dim;  // V[k * ldv + I]: component k of eigenvector I
  if (dim <= g_dense_casida_limit) {
    std::vector<double> Om((size_t)dim * dim);
    for (int k = 0; k < dim; ++k)
      for (int l = 0; l <= k; ++l) {
        double s = 0;
        for (int B = 0; B < nat; ++B) s += qG[(size_t)k * nat + B] * q[(size_t)l * nat + B];
        double v = 4.0 * std::sqrt(delta[k]) * s * std::sqrt(delta[l]);
        if (k == l) v += delta[k] * delta[k];
        Om[(size_t)k * dim + l] = Om[(size_t)l * dim + k] = v;
      }
    if (!oracle_la::eigh(dim, Om, w, V)) {
      g_error = "Casida diagonalisation failed";
      return false;
    }
  } else {
    if (!davidson_lowest(dim, nat, nroots, delta, q, qG, w, V)) {
      g_error = "Casida Davidson iteration failed";
      return false;
    }
    ldv = nroots;
  }
  omega.assign(nroots, 0.0);
  dip.assign(3 * (size_t)nroots, 0.0);
  for (int I = 0; I < nroots; ++I) {
    if (!(w[I] > 0)) {
      g_error = "non-positive Casida eigenvalue";
      return false;
    }
    const double om = std::sqrt(w[I]);
    omega[I] = om;
    if (triplet) continue;
    for (int k = 0; k < dim; ++k) {
      const double c = std::sqrt(delta[k] / om) * V[(size_t)k * ldv + I];
      for (int A = 0; A < nat; ++A)
        for (int x = 0; x < 3; ++x) dip[3 * I + x] += std::sqrt(2.0) * c * q[(size_t)k * nat + A] * M.pos[3 * A + x];
    }
  }
  return true;
}

}  // namespace dftb_oracle

extern "C" {

const char* dftb_oracle_last_error() { return dftb_oracle::g_error.c_str(); }

// Transitions up to which the TD-DFTB eigenproblem is solved densely (the
// Davidson path above); tests set 0 to check the two paths against each other.
void dftb_oracle_set_dense_casida_limit(int limit) { dftb_oracle::g_dense_casida_limit = limit; }

// H0 and S (N x N, both triangles), gamma (nat x nat) and, for DFTB3, Gamma
// (Gamma[a][b] = Gamma_ab).  nao_out receives N.
int dftb_oracle_matrices(const char* set, int order, int nat, const int* Z, const double* xyz, double* H0, double* S,
                         double* gam, double* Gam, int* nao_out) {
  using namespace dftb_oracle;
  Mol M;
  if (!setup(set, order, nat, Z, xyz, 0, M) && M.nao == 0) return 1;
  State st;
  build_static(M, st);
  if (nao_out) *nao_out = M.nao;
  if (H0) std::memcpy(H0, st.H0.data(), sizeof(double) * st.H0.size());
  if (S) std::memcpy(S, st.S.data(), sizeof(double) * st.S.size());
  if (gam) std::memcpy(gam, st.gam.data(), sizeof(double) * st.gam.size());
  if (Gam && order == 3) std::memcpy(Gam, st.Gam.data(), sizeof(double) * st.Gam.size());
  return 0;
}

// Converged restricted DFTB (order 2 or 3).  info[8] = e_el, e_rep,
// iterations, converged, nao, nocc, nel, 0.  q_out (nat), eps_out (nao) and
// P_out (nao x nao) may be NULL.
int dftb_oracle_scf(const char* set, int order, int nat, const int* Z, const double* xyz, int charge, double scc,
                    double rmsd, int max_iter, int want_grad, double* energy, double* grad, double* info, double* q_out,
                    double* eps_out, double* P_out) {
  using namespace dftb_oracle;
  Mol M;
  if (!setup(set, order, nat, Z, xyz, charge, M)) return 1;
  State st;
  if (!scf(M, st, scc, rmsd, max_iter)) return 2;
  if (energy) *energy = st.e_el + st.e_rep;
  if (info) {
    info[0] = st.e_el;
    info[1] = st.e_rep;
    info[2] = st.iterations;
    info[3] = st.converged ? 1 : 0;
    info[4] = M.nao;
    info[5] = M.nocc;
    info[6] = M.nel;
    info[7] = 0;
  }
  if (q_out) std::memcpy(q_out, st.q.data(), sizeof(double) * M.nat);
  if (eps_out) std::memcpy(eps_out, st.eps.data(), sizeof(double) * M.nao);
  if (P_out) std::memcpy(P_out, st.P.data(), sizeof(double) * st.P.size());
  if (want_grad && grad) {
    std::vector<double> g;
    gradient(M, st, g);
    std::memcpy(grad, g.data(), sizeof(double) * g.size());
  }
  return st.converged ? 0 : 3;
}

// Spin-polarised (unrestricted) DFTB2/3 single point with spin multiplicity
// mult.  info[8] = {E_el, E_rep, iterations, converged, nao, n_alpha, n_beta,
// E_spin}; q_out (Mulliken charges), eps_a / eps_b (nao) optional.
int dftb_oracle_scf_uhf(const char* set, int order, int nat, const int* Z, const double* xyz, int charge, int mult,
                        double scc, double rmsd, int max_iter, int want_grad, double* energy, double* grad,
                        double* info, double* q_out, double* eps_a, double* eps_b) {
  using namespace dftb_oracle;
  Mol M;
  if (mult < 1 || !setup(set, order, nat, Z, xyz, charge, M, mult)) {
    if (mult < 1) g_error = "spin multiplicity must be positive";
    return 1;
  }
  State st;
  SpinState ss;
  if (!scf_uhf(M, st, ss, scc, rmsd, max_iter)) return 2;
  if (energy) *energy = st.e_el + st.e_rep;
  if (info) {
    double v[8] = {st.e_el, st.e_rep, (double)st.iterations, st.converged ? 1.0 : 0.0, (double)M.nao,
                   (double)M.nalpha, (double)M.nbeta, ss.e_spin};
    std::memcpy(info, v, sizeof(v));
  }
  if (q_out) std::memcpy(q_out, st.q.data(), sizeof(double) * M.nat);
  if (eps_a) std::memcpy(eps_a, ss.epsa.data(), sizeof(double) * M.nao);
  if (eps_b) std::memcpy(eps_b, ss.epsb.data(), sizeof(double) * M.nao);
  if (want_grad && grad) {
    std::vector<double> g;
    gradient_uhf(M, st, ss, g);
    std::memcpy(grad, g.data(), sizeof(double) * g.size());
  }
  return st.converged ? 0 : 3;
}

// TD-DFTB excitations of a converged restricted DFTB reference: omega
// (nroots, Hartree) and, for singlets, the transition dipoles (3 * nroots,
// e bohr).  info[4] = ground-state energy, nao, nocc, transitions.
int dftb_oracle_tddftb(const char* set, int order, int nat, const int* Z, const double* xyz, int charge, double scc,
                       double rmsd, int max_iter, int triplet, int nroots, double* omega, double* dip, double* info) {
  using namespace dftb_oracle;
  Mol M;
  if (!setup(set, order, nat, Z, xyz, charge, M)) return 1;
  State st;
  if (!scf(M, st, scc, rmsd, max_iter)) return 2;
  if (!st.converged) {
    g_error = "reference SCF did not converge";
    return 3;
  }
  std::vector<double> om, dp;
  if (!tddftb(M, st, triplet, nroots, om, dp)) return 4;
  std::memcpy(omega, om.data(), sizeof(double) * om.size());
  if (dip) std::memcpy(dip, dp.data(), sizeof(double) * dp.size());
  if (info) {
    info[0] = st.e_el + st.e_rep;
    info[1] = M.nao;
    info[2] = M.nocc;
    info[3] = (double)M.nocc * (M.nao - M.nocc);
  }
  return 0;
}

}  // extern "C"
