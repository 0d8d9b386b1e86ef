// DFTB pair math shared by the DFTB kernels and the host-side parameter
// preparation (all functions __host__ __device__).
//
// Reference behaviour followed (paths relative to
// src/Sparrow/Sparrow/Implementations/Dftb/):
//   Slater-Koster integrals  Utils/SKPair.cpp:130-304: 8-point Neville
//                            interpolation in grid units (row i at distance
//                            (i + 1) * grid), 5th-order tail up to
//                            rows * grid + 1 bohr, zero outside
//   table completion         Utils/SKPair.cpp:79-89: the p-s columns are the
//                            reverse pair's s-p columns, negated
//   H0 / S blocks            Utils/ZeroOrderMatricesCalculator.cpp:92-232
//                            (direction cosines; the atom of lower Z first)
//   gamma (DFTB2)            Utils/SecondOrderFock.cpp:82-113
//   gamma^h, Gamma (DFTB3)   Utils/ThirdOrderFock.cpp:80-155
//   repulsion                Utils/PairwiseRepulsion.cpp:40-71
#pragma once
#include <cmath>

#include "nddo_math.cuh"

namespace sgb {

constexpr int kDftbInter = 8, kDftbInterRight = 4, kDftbInterLeft = 4;
constexpr double kDftbDistFudge = 1.0, kDftbDeltaR = 1e-5;
constexpr int kDftbCols = 10;  // completed integral columns per table row

struct DftbElemDev {
  int Z, nao;
  double es, ep, U, occ, hd;
  double w;    // atomically resolved spin constant (W_pp, or W_ss for s-only atoms)
  int has_w;   // spin constants available (triplet excitations, spin-polarised SCC)
  int pad;
  double wss, wsp, wps, wpp;  // shell-resolved spin constants W(l, l') (SDFTB.cpp, SKAtom.h:52-66)
};

// Parameters of an ordered element pair (file Z1-Z2): its completed integral
// table (rows x kDftbCols doubles at table_off), the tail polynomial, the
// gamma terms of SKPair::precalculateGammaTerms and the repulsion spline.
struct DftbPairDev {
  int present, nint, rows, n_spline;
  double grid, rmax;
  long long table_off;
  int spline_off, pad;
  double cutoff, a1, a2, a3, c4, c5;
  double t3[kDftbCols], t4[kDftbCols], t5[kDftbCols];
  double g1a, g1b, g2a, g2b;
  double dgab1a, dgab1b, dgab2a, dgab2b, dgba1a, dgba1b, dgba2a, dgba2b;
};

struct DftbSplineDev {
  double start, end, c0, c1, c2, c3;
};

// Neville interpolation of the first nint integrals at grid coordinate x
// from row `start`: values and derivatives with respect to the distance.
SGB_HD void dftb_interpolate(const double* tab, int nint, double grid, double x, int start, double* val,
                             double* der) {
  double xa[kDftbInter];
  for (int i = 0; i < kDftbInter; ++i) xa[i] = (double)(start + i);
  double dif = x - start;
  int ns0 = 0;
  for (int i = 0; i < kDftbInter; ++i) {
    const double dift = fabs(x - xa[i]);
    if (dift < dif) {
      dif = dift;
      ns0 = i;
    }
  }
  const double dh = -1.0 / grid;
  for (int L = 0; L < nint; ++L) {
    double Cv[kDftbInter], Cd[kDftbInter], Dv[kDftbInter], Dd[kDftbInter];
    for (int i = 0; i < kDftbInter; ++i) {
      Cv[i] = Dv[i] = tab[(size_t)(start + i) * kDftbCols + L];
      Cd[i] = Dd[i] = 0.0;
    }
    int ns = ns0;
    double yv = Cv[ns], yd = 0.0;
    --ns;
    for (int m = 1; m < kDftbInter; ++m) {
      for (int i = 0; i <= kDftbInter - 1 - m; ++i) {
        const double ho = xa[i] - x, hp = xa[i + m] - x;
        const double wv = Cv[i + 1] - Dv[i], wd = Cd[i + 1] - Dd[i];
        const double denv = wv / (ho - hp), dend = wd / (ho - hp);
        Dv[i] = hp * denv;
        Dd[i] = hp * dend + dh * denv;
        Cv[i] = ho * denv;
        Cd[i] = ho * dend + dh * denv;
      }
      if (2 * (ns + 1) < kDftbInter - m) {
        yv += Cv[ns + 1];
        yd += Cd[ns + 1];
      } else {
        yv += Dv[ns];
        yd += Dd[ns];
        --ns;
      }
    }
    val[L] = yv;
    der[L] = yd;
  }
}

// |R| as a function of the pair vector (a plain value for T = double).
template <class T>
SGB_HD T dual_r(const double* R, double dist);
template <>
SGB_HD double dual_r<double>(const double*, double dist) { return dist; }
template <>
SGB_HD Dual3 dual_r<Dual3>(const double* R, double dist) { return Dual3(dist, R[0] / dist, R[1] / dist, R[2] / dist); }

// Direction cosine R_k / |R| (with its gradient for T = Dual3).
template <class T>
SGB_HD T direction_cosine(const double* R, double dist, int k);
template <>
SGB_HD double direction_cosine<double>(const double* R, double dist, int k) { return R[k] / dist; }
template <>
SGB_HD Dual3 direction_cosine<Dual3>(const double* R, double dist, int k) {
  const double v = R[k] / dist, inv = 1.0 / dist;
  return Dual3(v, ((k == 0) - v * R[0] * inv) * inv, ((k == 1) - v * R[1] * inv) * inv,
               ((k == 2) - v * R[2] * inv) * inv);
}

// Integrals of pair p at distance dist (values, d/d distance); 0 when they vanish.
SGB_HD int dftb_integrals(const DftbPairDev& p, const double* table, double dist, double* val, double* der) {
  for (int L = 0; L < kDftbCols; ++L) val[L] = der[L] = 0.0;
  if (dist < p.grid || dist > p.rmax) return 0;
  const double* tab = table + p.table_off;
  if (dist > p.rows * p.grid) {
    // tail: derivative taken with respect to the tail coordinate (as the reference does)
    const double xr = -(dist - p.rmax) / kDftbDistFudge;
    for (int L = 0; L < p.nint; ++L) {
      const double q = (p.t5[L] * xr + p.t4[L]) * xr + p.t3[L];
      const double dq = 2.0 * p.t5[L] * xr + p.t4[L];
      val[L] = q * xr * xr * xr;
      der[L] = dq * xr * xr * xr + 3.0 * q * xr * xr;
    }
    return 1;
  }
  const double position = dist / p.grid - 1.0;
  const int ind = (int)position;
  const int start = ind >= p.rows - kDftbInterRight ? p.rows - kDftbInter
                                                     : (ind < kDftbInterLeft ? 0 : ind - kDftbInterLeft + 1);
  dftb_interpolate(tab, p.nint, p.grid, position, start, val, der);
  return 1;
}

// S (m = 0) and H0 (m = 1) blocks me[m][i][j] of the first (lower-Z) atom
// with nF orbitals against the second with nS, for the vector R from the
// first to the second; T = double (values) or Dual3 (values and gradients).
template <class T>
SGB_HD int dftb_blocks(const DftbPairDev& p, const double* table, int nF, int nS, const double* R, T me[2][4][4]) {
  for (int m = 0; m < 2; ++m)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) me[m][i][j] = T(0.0);
  const double dist = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
  double iv[kDftbCols], id[kDftbCols];
  if (dftb_integrals(p, table, dist, iv, id) == 0) return 0;
  T I[kDftbCols];
  const T rr = dual_r<T>(R, dist);
  for (int L = 0; L < p.nint; ++L) I[L] = lift(iv[L], id[L], rr);
  for (int m = 0; m < 2; ++m) me[m][0][0] = I[m];
  if (nF + nS == 2) return 1;
  T v[3];
  for (int k = 0; k < 3; ++k) v[k] = direction_cosine<T>(R, dist, k);
  for (int m = 0; m < 2; ++m) {
    for (int j = 0; j < 3; ++j) me[m][0][j + 1] = I[2 + m] * v[j];
    if (nF != 1 && nS != 1) {
      for (int j = 0; j < 3; ++j) me[m][j + 1][0] = I[8 + m] * v[j];
      for (int i = 0; i < 3; ++i) {
        const T vii = v[i] * v[i];
        me[m][i + 1][i + 1] = I[4 + m] * vii + I[6 + m] * (T(1.0) - vii);
        for (int j = i + 1; j < 3; ++j)
          me[m][j + 1][i + 1] = me[m][i + 1][j + 1] = (v[i] * v[j]) * (I[4 + m] - I[6 + m]);
      }
    }
  }
  return 1;
}

// gamma_ab of DFTB2 (a != b) at distance R and its derivative.
SGB_HD void dftb_gamma2(const DftbElemDev& A, const DftbElemDev& B, const DftbPairDev& pab, double R, double& g,
                        double& dg) {
  const double ta = A.U * 3.2, tb = B.U * 3.2;
  const double inv = 1.0 / R, dinv = -1.0 / (R * R);
  const double ea = exp(-ta * R), eb = exp(-tb * R);
  if (A.Z == B.Z) {
    const double ta2 = ta * ta;
    const double ex = inv + 0.6875 * ta + 0.1875 * R * ta2 + 0.02083333333333333 * R * R * ta * ta2;
    const double dex = dinv + 0.1875 * ta2 + 2.0 * 0.02083333333333333 * R * ta * ta2;
    g = inv - ea * ex;
    dg = dinv + ta * ea * ex - ea * dex;
    return;
  }
  const double fa = pab.g1a - pab.g2a * inv, dfa = -pab.g2a * dinv;
  const double fb = pab.g1b - pab.g2b * inv, dfb = -pab.g2b * dinv;
  g = inv - ea * fa - eb * fb;
  dg = dinv + ta * ea * fa - ea * dfa + tb * eb * fb - eb * dfb;
}

// First-order dual in the distance (value, derivative) for the DFTB3 terms.
struct DftbD1 {
  double v, d;
};
SGB_HD DftbD1 d1_mul(DftbD1 a, DftbD1 b) { return DftbD1{a.v * b.v, a.v * b.d + a.d * b.v}; }
SGB_HD DftbD1 d1_add(DftbD1 a, DftbD1 b) { return DftbD1{a.v + b.v, a.d + b.d}; }
SGB_HD DftbD1 d1_sub(DftbD1 a, DftbD1 b) { return DftbD1{a.v - b.v, a.d - b.d}; }
SGB_HD DftbD1 d1_scl(double s, DftbD1 a) { return DftbD1{s * a.v, s * a.d}; }

// gamma^h_ab, Gamma_ab, Gamma_ba of DFTB3 (a != b) and their derivatives:
// out = {gamma, dgamma, Gab, dGab, Gba, dGba}.
SGB_HD void dftb_gamma3(const DftbElemDev& A, const DftbElemDev& B, const DftbPairDev& pab, double Rv, double out[6]) {
  const double Ua = A.U, Ub = B.U;
  const DftbD1 R{Rv, 1.0};
  const DftbD1 R2 = d1_mul(R, R);
  const DftbD1 inv{1.0 / Rv, -1.0 / (Rv * Rv)};
  DftbD1 h{1.0, 0.0}, dhdU{0.0, 0.0};
  if (A.Z == 1 || B.Z == 1) {
    const double zeta = 4.0;
    const double powerM1 = pow((Ua + Ub) / 2.0, zeta - 1.0);
    const double power = powerM1 * (Ua + Ub) / 2.0;
    const double e = exp(-power * R2.v);
    h = DftbD1{e, -power * R2.d * e};
    dhdU = d1_scl(-zeta / 2.0 * powerM1, d1_mul(R2, h));
  }
  const double ta = Ua * 3.2, tb = Ub * 3.2;
  const DftbD1 ea{exp(-ta * Rv), -ta * exp(-ta * Rv)};
  const DftbD1 eb{exp(-tb * Rv), -tb * exp(-tb * Rv)};
  DftbD1 S, dSda, dSdb;
  if (A.Z == B.Z) {
    const double ta2 = ta * ta;
    const DftbD1 g = d1_scl(1.0 / 48.0, d1_add(d1_add(d1_add(d1_scl(48.0, inv), DftbD1{33.0 * ta, 0.0}),
                                                      d1_scl(9.0 * ta2, R)),
                                               d1_scl(ta * ta2, R2)));
    const DftbD1 dgda = d1_scl(1.0 / 48.0, d1_add(d1_add(DftbD1{33.0, 0.0}, d1_scl(18.0 * ta, R)), d1_scl(3.0 * ta2, R2)));
    S = d1_mul(ea, g);
    dSda = dSdb = d1_mul(ea, d1_sub(dgda, d1_mul(R, g)));
  } else {
    const DftbD1 fab = d1_sub(DftbD1{pab.g1a, 0.0}, d1_scl(pab.g2a, inv));
    const DftbD1 fba = d1_sub(DftbD1{pab.g1b, 0.0}, d1_scl(pab.g2b, inv));
    const DftbD1 dfabda = d1_sub(DftbD1{-pab.dgab1a, 0.0}, d1_scl(pab.dgab2a, inv));
    const DftbD1 dfbadb = d1_sub(DftbD1{-pab.dgba1a, 0.0}, d1_scl(pab.dgba2a, inv));
    const DftbD1 dfabdb = d1_add(DftbD1{pab.dgab1b, 0.0}, d1_scl(pab.dgab2b, inv));
    const DftbD1 dfbada = d1_add(DftbD1{pab.dgba1b, 0.0}, d1_scl(pab.dgba2b, inv));
    S = d1_add(d1_mul(ea, fab), d1_mul(eb, fba));
    dSda = d1_add(d1_mul(ea, d1_sub(dfabda, d1_mul(R, fab))), d1_mul(eb, dfbada));
    dSdb = d1_add(d1_mul(eb, d1_sub(dfbadb, d1_mul(R, fba))), d1_mul(ea, dfabdb));
  }
  const DftbD1 dgdUa = d1_scl(-1.0, d1_add(d1_scl(3.2, d1_mul(dSda, h)), d1_mul(S, dhdU)));
  const DftbD1 dgdUb = d1_scl(-1.0, d1_add(d1_scl(3.2, d1_mul(dSdb, h)), d1_mul(S, dhdU)));
  const DftbD1 gam = d1_sub(inv, d1_mul(S, h));
  out[0] = gam.v;
  out[1] = gam.d;
  out[2] = A.hd * dgdUa.v;
  out[3] = A.hd * dgdUa.d;
  out[4] = B.hd * dgdUb.v;
  out[5] = B.hd * dgdUb.d;
}

// Repulsion of pair p at r and dE/dr.
SGB_HD void dftb_repulsion(const DftbPairDev& p, const DftbSplineDev* splines, double r, double& E, double& dE) {
  E = dE = 0.0;
  if (r > p.cutoff || p.n_spline < 1) return;
  const DftbSplineDev* sp = splines + p.spline_off;
  if (r < sp[0].start) {
    const double e = exp(-p.a1 * r + p.a2);
    E = e + p.a3;
    dE = -p.a1 * e;
    return;
  }
  int i = (int)((r - sp[0].start) / (p.cutoff - sp[0].start) * p.n_spline);
  if (i > p.n_spline - 1) i = p.n_spline - 1;
  if (i < 0) i = 0;
  if (sp[i].start > r) {
    while (i > 0 && sp[--i].start > r) {
    }
  } else if (sp[i].end < r) {
    while (i < p.n_spline - 1 && sp[++i].end < r) {
    }
  }
  const double dr = r - sp[i].start;
  double c4 = 0.0, c5 = 0.0;
  if (i == p.n_spline - 1) {
    c4 = p.c4;
    c5 = p.c5;
  }
  E = sp[i].c0 + dr * (sp[i].c1 + dr * (sp[i].c2 + dr * (sp[i].c3 + dr * (c4 + dr * c5))));
  dE = sp[i].c1 + dr * (2.0 * sp[i].c2 + dr * (3.0 * sp[i].c3 + dr * (4.0 * c4 + dr * 5.0 * c5)));
}

}  // namespace sgb
