// NDDO pair math shared by the integral and gradient kernels.
//
// All functions are __host__ __device__ and templated on the scalar type T:
// double for values, Dual3 (value + d/dX, d/dY, d/dZ of the pair vector) for
// the nuclear gradient.  Reference behaviour followed (paths relative to
// src/Sparrow/Sparrow/Implementations/Nddo/):
//   multipole local integrals  Utils/IntegralsEvaluationUtils/Local2c2eIntegralCalculator.cpp:39-292,
//                              MultipoleMultipoleTerm.h:58-98, ChargesInMultipoles.cpp:27-125
//   local 10x10 block          Local2c2eMatrix.cpp:39-149 (which entries are evaluated,
//                              which are copies, <xy|xy> = (<xx|xx> - <xx|yy>)/2)
//   frame rotation             OrbitalRotation.cpp:78-154, Global2c2eMatrix.cpp:46-151
//   overlap                    GTOOverlapMatrixBlock.cpp:70-165
//   core repulsion             Pm6/PM6PairwiseRepulsion.h:76-192, Am1/AM1PairwiseRepulsion.h:64-151
#pragma once
#include <cmath>

#include "engine_types.h"

#ifdef __CUDACC__
#define SGB_HD __host__ __device__ __forceinline__
#else
#define SGB_HD inline
#endif

namespace sgb {

// ---------------------------------------------------------------------------
// Dual number for first derivatives with respect to the pair vector (X, Y, Z)
// ---------------------------------------------------------------------------
struct Dual3 {
  double v, dx, dy, dz;
  SGB_HD Dual3() : v(0), dx(0), dy(0), dz(0) {}
  SGB_HD Dual3(double a) : v(a), dx(0), dy(0), dz(0) {}
  SGB_HD Dual3(double a, double b, double c, double d) : v(a), dx(b), dy(c), dz(d) {}
};
SGB_HD Dual3 operator+(const Dual3& a, const Dual3& b) { return Dual3(a.v + b.v, a.dx + b.dx, a.dy + b.dy, a.dz + b.dz); }
SGB_HD Dual3 operator-(const Dual3& a, const Dual3& b) { return Dual3(a.v - b.v, a.dx - b.dx, a.dy - b.dy, a.dz - b.dz); }
SGB_HD Dual3 operator-(const Dual3& a) { return Dual3(-a.v, -a.dx, -a.dy, -a.dz); }
SGB_HD Dual3 operator*(const Dual3& a, const Dual3& b) {
  return Dual3(a.v * b.v, a.dx * b.v + a.v * b.dx, a.dy * b.v + a.v * b.dy, a.dz * b.v + a.v * b.dz);
}
SGB_HD Dual3 operator*(double s, const Dual3& b) { return Dual3(s * b.v, s * b.dx, s * b.dy, s * b.dz); }
SGB_HD Dual3 operator/(const Dual3& a, const Dual3& b) {
  double inv = 1.0 / b.v, q = a.v * inv;
  return Dual3(q, (a.dx - q * b.dx) * inv, (a.dy - q * b.dy) * inv, (a.dz - q * b.dz) * inv);
}
SGB_HD Dual3& operator+=(Dual3& a, const Dual3& b) {
  a.v += b.v; a.dx += b.dx; a.dy += b.dy; a.dz += b.dz;
  return a;
}
SGB_HD Dual3 dsqrt(const Dual3& a) {
  double s = sqrt(a.v), h = 0.5 / s;
  return Dual3(s, a.dx * h, a.dy * h, a.dz * h);
}
SGB_HD Dual3 dexp(const Dual3& a) {
  double e = exp(a.v);
  return Dual3(e, a.dx * e, a.dy * e, a.dz * e);
}
SGB_HD double dsqrt(double a) { return sqrt(a); }
SGB_HD double dexp(double a) { return exp(a); }
SGB_HD double value_of(double a) { return a; }
SGB_HD double value_of(const Dual3& a) { return a.v; }
// f(R) with df/dR, lifted to a function of the pair vector whose |R| is r
SGB_HD double lift(double f, double, const double&) { return f; }
SGB_HD Dual3 lift(double f, double df, const Dual3& r) { return Dual3(f, df * r.dx, df * r.dy, df * r.dz); }

// ---------------------------------------------------------------------------
// Local integral term table (built once on the host, see local_terms.cpp)
// ---------------------------------------------------------------------------
// A term is one point-charge pair of the multipole expansion: charge product
// q, charge offsets (in units of the charge separation of its multipole class)
// on centre A (x1,y1,z1) and on centre B (x2,y2,z2), and the multipole classes
// c1, c2 (0 ss0, 1 sp1, 2 pp0, 3 pp2) selecting D and the Klopman radius.
struct LocalTerm {
  double q;
  float x1, y1, z1, x2, y2, z2;
  int c1, c2;
};

constexpr int kLocalUnique = 21;
constexpr int kLocalMaxTerms = 512;
// Term slots of one pair in the heavy-pair value kernel: every two-electron
// term plus the terms of both core-attraction sigma columns (checked when the
// table is built).
constexpr int kPairTermSlots = 256;

struct LocalTermTable {
  int row[kLocalUnique], col[kLocalUnique];  // orbital-pair indices of the evaluated entries
  int start[kLocalUnique], count[kLocalUnique];
  int n_terms;
  LocalTerm term[kLocalMaxTerms];
};

// Orbital-pair index of (mu, nu), s=0, x=1, y=2, z=3
SGB_HD int pair_index(int a, int b) { return a <= b ? b * (b + 1) / 2 + a : a * (a + 1) / 2 + b; }

// One evaluated local entry (value and d/dR).  coreB: the second centre is a
// bare core with Klopman radius rhoCoreB and no multipoles (VuvB).
SGB_HD void local_entry(const LocalTermTable& tab, int e, double R, const ElemDev& A, const ElemDev& B, bool coreB,
                        double rhoCoreB, double& val, double& dval) {
  val = 0;
  dval = 0;
  const int s = tab.start[e], n = tab.count[e];
  for (int t = s; t < s + n; ++t) {
    const LocalTerm& T = tab.term[t];
    double rA = A.rho[T.c1];
    double rB = coreB ? rhoCoreB : B.rho[T.c2];
    double D1 = A.D[T.c1];
    double d2 = coreB ? 0.0 : B.D[T.c2];
    double dx = d2 * T.x2 - D1 * T.x1;
    double dy = d2 * T.y2 - D1 * T.y1;
    double dz = R + d2 * T.z2 - D1 * T.z1;
    double rr = rA + rB;
    double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + rr * rr);
    val += T.q * inv;
    dval -= dz * T.q * inv * inv * inv;
  }
}

// Entries of the local dA x dB block that the reference copies by symmetry
// about the bond axis (Local2c2eMatrix.cpp:91-149).
SGB_HD void local_copies(int dA, int dB, double L[10][10], double dL[10][10]) {
  if (dB == 10) { L[0][5] = L[0][2]; dL[0][5] = dL[0][2]; }
  if (dA == 10) { L[5][0] = L[2][0]; dL[5][0] = dL[2][0]; }
  if (dA == 10 && dB == 10) {
    const int cp[10][4] = {{3, 3, 1, 1}, {3, 8, 1, 7}, {5, 2, 2, 5}, {5, 5, 2, 2}, {5, 6, 2, 6},
                           {5, 9, 2, 9}, {6, 5, 6, 2}, {8, 3, 7, 1}, {8, 8, 7, 7}, {9, 5, 9, 2}};
    for (int k = 0; k < 10; ++k) {
      L[cp[k][0]][cp[k][1]] = L[cp[k][2]][cp[k][3]];
      dL[cp[k][0]][cp[k][1]] = dL[cp[k][2]][cp[k][3]];
    }
    L[4][4] = 0.5 * (L[2][2] - L[2][5]);
    dL[4][4] = 0.5 * (dL[2][2] - dL[2][5]);
  }
}

// Fill the local dA x dB block (dA, dB in {1, 10}) the way the reference does.
SGB_HD void local_block(const LocalTermTable& tab, int dA, int dB, double R, const ElemDev& A, const ElemDev& B,
                        bool coreB, double rhoCoreB, double L[10][10], double dL[10][10]) {
  for (int i = 0; i < dA; ++i)
    for (int j = 0; j < dB; ++j) L[i][j] = dL[i][j] = 0;
  for (int e = 0; e < kLocalUnique; ++e) {
    int i = tab.row[e], j = tab.col[e];
    if (i >= dA || j >= dB) continue;
    local_entry(tab, e, R, A, B, coreB, rhoCoreB, L[i][j], dL[i][j]);
  }
  local_copies(dA, dB, L, dL);
}

// Rotation coefficients rot[global][local] for s, x, y, z given the pair
// vector; |R| returned in R.  When the vector lies on the z axis the
// reference sets cos(alpha)=1, sin(alpha)=0 with zero derivatives.
template <class T>
SGB_HD void frame_rotation(const T& X, const T& Y, const T& Z, T rot[4][4], T& R) {
  R = dsqrt(X * X + Y * Y + Z * Z);
  double xv = value_of(X), yv = value_of(Y);
  T proj = T(0.0);
  if (sqrt(xv * xv + yv * yv) != 0) proj = dsqrt(X * X + Y * Y);
  T ca = T(1.0), sa = T(0.0);
  if (value_of(proj) != 0) {
    ca = X / proj;
    sa = Y / proj;
  }
  T cb = Z / R, sb = proj / R;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) rot[i][j] = T(0.0);
  rot[0][0] = T(1.0);
  rot[1][1] = ca * cb;
  rot[2][1] = sa * cb;
  rot[3][1] = -sb;
  rot[1][2] = -sa;
  rot[2][2] = ca;
  rot[1][3] = ca * sb;
  rot[2][3] = sa * sb;
  rot[3][3] = cb;
}

// Pair-rotation matrix W[p(mu,nu)][p(mu',nu')] = sum over orderings of
// rot[mu][mu'] rot[nu][nu'] for an atom with n (1 or 4) orbitals.
template <class T>
SGB_HD void pair_rotation(int n, const T rot[4][4], T W[10][10]) {
  int d = n == 1 ? 1 : 10;
  for (int a = 0; a < d; ++a)
    for (int b = 0; b < d; ++b) W[a][b] = T(0.0);
  for (int mu = 0; mu < n; ++mu)
    for (int nu = mu; nu < n; ++nu) {
      int p = pair_index(mu, nu);
      // s and p never mix under rotation: skip the structurally zero s/p couplings
      for (int m2 = (mu == 0 ? 0 : 1); m2 < (mu == 0 ? 1 : n); ++m2)
        for (int n2 = (nu == 0 ? 0 : 1); n2 < (nu == 0 ? 1 : n); ++n2)
          W[p][pair_index(m2, n2)] += rot[mu][m2] * rot[nu][n2];
    }
}

// Global two-centre block G[p on A][p' on B] for Rab = pos_B - pos_A.
template <class T>
SGB_HD void global_block(const LocalTermTable& tab, const ElemDev& A, const ElemDev& B, const T& X, const T& Y,
                         const T& Z, T G[10][10]) {
  T rot[4][4], R;
  frame_rotation(X, Y, Z, rot, R);
  const int dA = A.nao == 1 ? 1 : 10, dB = B.nao == 1 ? 1 : 10;
  double L[10][10], dL[10][10];
  local_block(tab, dA, dB, value_of(R), A, B, false, 0.0, L, dL);
  T WA[10][10], WB[10][10];
  pair_rotation(A.nao, rot, WA);
  pair_rotation(B.nao, rot, WB);
  T tmp[10][10];
  for (int a = 0; a < dA; ++a)
    for (int l = 0; l < dB; ++l) {
      T s = T(0.0);
      for (int k = 0; k < dB; ++k)
        if (L[a][k] != 0 || dL[a][k] != 0) s += lift(L[a][k], dL[a][k], R) * WB[l][k];
      tmp[a][l] = s;
    }
  for (int g = 0; g < dA; ++g)
    for (int l = 0; l < dB; ++l) {
      T s = T(0.0);
      for (int a = 0; a < dA; ++a) s += WA[g][a] * tmp[a][l];
      G[g][l] = s;
    }
}

// Core-attraction vector V[p on A] = -Z_B (mu nu | s_B s_B) with B's Klopman
// radius replaced by its core radius pcore (VuvB.cpp:17-31, VuvB.h:39-49).
template <class T>
SGB_HD void core_vector(const LocalTermTable& tab, const ElemDev& A, const ElemDev& B, const T& X, const T& Y,
                        const T& Z, T V[10]) {
  T rot[4][4], R;
  frame_rotation(X, Y, Z, rot, R);
  const int dA = A.nao == 1 ? 1 : 10;
  double L[10][10], dL[10][10];
  local_block(tab, dA, 1, value_of(R), A, B, true, B.pcore, L, dL);
  T WA[10][10];
  pair_rotation(A.nao, rot, WA);
  for (int g = 0; g < dA; ++g) {
    T s = T(0.0);
    for (int a = 0; a < dA; ++a)
      if (L[a][0] != 0) s += WA[g][a] * lift(L[a][0], dL[a][0], R);
    V[g] = (-B.core) * s;
  }
}

// STO-6G overlap block S[mu on A][nu on B], B displaced by R from A.
template <class T>
SGB_HD void overlap_block(const ElemDev& A, const ElemDev& B, const T R[3], T S[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) S[i][j] = T(0.0);
  const double pi = 3.14159265358979323846;
  T R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
  const int nla = A.nao == 4 ? 2 : 1, nlb = B.nao == 4 ? 2 : 1;
  for (int la = 0; la < nla; ++la)
    for (int lb = 0; lb < nlb; ++lb)
      for (int i = 0; i < 6; ++i) {
        double a = la ? A.p_exp[i] : A.s_exp[i], ca = la ? A.p_coef[i] : A.s_coef[i];
        for (int j = 0; j < 6; ++j) {
          double b = lb ? B.p_exp[j] : B.s_exp[j], cb = lb ? B.p_coef[j] : B.s_coef[j];
          double p = a + b;
          double s00 = sqrt(pi / p);
          T K = (ca * cb) * dexp((-a * b / p) * R2);
          T PA[3], PB[3];
          for (int d = 0; d < 3; ++d) {
            PA[d] = (b / p) * R[d];
            PB[d] = PA[d] - R[d];
          }
          if (!la && !lb) {
            S[0][0] += (s00 * s00 * s00) * K;
          } else if (la && !lb) {
            for (int u = 0; u < 3; ++u) S[1 + u][0] += (s00 * s00 * s00) * (PA[u] * K);
          } else if (!la && lb) {
            for (int v = 0; v < 3; ++v) S[0][1 + v] += (s00 * s00 * s00) * (PB[v] * K);
          } else {
            for (int u = 0; u < 3; ++u)
              for (int v = 0; v < 3; ++v) {
                T f = u == v ? PA[u] * PB[u] + T(1.0 / (2 * p)) : PA[u] * PB[v];
                S[1 + u][1 + v] += (s00 * s00 * s00) * (f * K);
              }
          }
        }
      }
}

// Core-core repulsion energy of a pair at distance R and dE/dR.
SGB_HD void core_repulsion(int method, const ElemDev& A, const ElemDev& B, const DiatomicDev& AB, double R,
                           double& E, double& dE) {
  const double ev = 4.359744650e-18 / 1.6021766208e-19;
  const double angPerBohr = 0.52917721067;
  double ps = A.pcore + B.pcore;
  double g = 1.0 / sqrt(R * R + ps * ps);
  double dg = -g * g * g * R;
  double ZZ = A.core * B.core;
  double f, df;
  E = dE = 0;
  if (method == kPM6) {
    const double cAdd = 0.0000207389327971913490822259;  // 1e-8 Angstrom^12 in bohr^12
    const double expC = 0.00001244878365801758178693335; // 3e-4 Angstrom^-5 in bohr^-5
    const double ccExp = 3.1644797213016;                // 5.98 / Angstrom
    const double sioDist = 5.480205761238679760340424;   // 2.9 Angstrom
    bool xh = (A.Z == 1 && (B.Z == 8 || B.Z == 7 || B.Z == 6)) || (B.Z == 1 && (A.Z == 8 || A.Z == 7 || A.Z == 6));
    if (xh) {
      double e = exp(-AB.alpha * R * R);
      f = 1 + 2 * AB.x * e;
      df = 2 * AB.x * e * (-2 * AB.alpha * R);
    } else {
      double R2 = R * R, R6 = R2 * R2 * R2;
      double e = exp(-AB.alpha * (R + expC * R6));
      f = 1 + 2 * AB.x * e;
      df = 2 * AB.x * e * (-AB.alpha * (1 + 6 * expC * R2 * R2 * R));
      if (A.Z == 6 && B.Z == 6) {
        double c = 9.28 * exp(-ccExp * R);
        f += c;
        df -= ccExp * c;
      }
      if ((A.Z == 14 && B.Z == 8) || (A.Z == 8 && B.Z == 14)) {
        double r1 = R - sioDist;
        double c = -0.0007 * exp(-r1 * r1);
        f += c;
        df += -2 * r1 * c;
      }
    }
    E = ZZ * g * f;
    dE = ZZ * (dg * f + g * df);
    double v = (A.cbrtZ + B.cbrtZ) / R;
    double v2 = v * v, v6 = v2 * v2 * v2, v12 = v6 * v6;
    E += cAdd * v12 / ev;
    dE += cAdd * (-12.0 * v12 / R) / ev;
    // only the first Gaussian of each atom enters (early return in the reference's loop)
    double gs = 0, dgs = 0;
    if (A.n_gauss > 0) {
      double rc = R - A.gc[0], e = A.ga[0] * exp(-A.gb[0] * rc * rc);
      gs += e;
      dgs += -2 * A.gb[0] * rc * e;
    }
    if (B.n_gauss > 0) {
      double rc = R - B.gc[0], e = B.ga[0] * exp(-B.gb[0] * rc * rc);
      gs += e;
      dgs += -2 * B.gb[0] * rc * e;
    }
    E += gs / R * ZZ / ev;
    dE += (dgs / R - gs / (R * R)) * ZZ / ev;
    return;
  }
  double eA = exp(-A.alpha * R), eB = exp(-B.alpha * R);
  if (A.Z == 1 && (B.Z == 7 || B.Z == 8)) {
    f = 1 + eA + R * angPerBohr * eB;
    df = -A.alpha * eA + angPerBohr * eB * (1 - B.alpha * R);
  } else if (B.Z == 1 && (A.Z == 7 || A.Z == 8)) {
    f = 1 + R * angPerBohr * eA + eB;
    df = angPerBohr * eA * (1 - A.alpha * R) - B.alpha * eB;
  } else {
    f = 1 + eA + eB;
    df = -A.alpha * eA - B.alpha * eB;
  }
  E = ZZ * g * f;
  dE = ZZ * (dg * f + g * df);
  if (method == kAM1) {
    double gs = 0, dgs = 0;
    for (int k = 0; k < A.n_gauss; ++k) {
      double rc = R - A.gc[k], e = A.ga[k] * exp(-A.gb[k] * rc * rc);
      gs += e;
      dgs += -2 * A.gb[k] * rc * e;
    }
    for (int k = 0; k < B.n_gauss; ++k) {
      double rc = R - B.gc[k], e = B.ga[k] * exp(-B.gb[k] * rc * rc);
      gs += e;
      dgs += -2 * B.gb[k] * rc * e;
    }
    E += gs / R * ZZ / ev;
    dE += (dgs / R - gs / (R * R)) * ZZ / ev;
  }
}

}  // namespace sgb
