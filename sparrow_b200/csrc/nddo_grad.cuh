// Reverse-mode pieces of the NDDO pair gradient.
//
// The pair energy (TwoElectronMatrix.cpp:182-241, OneElectronMatrix.cpp:156-229)
//   E = sum_pq F_pq G_pq + sum_p fA_p VA_p + sum_p fB_p VB_p + sum (bA + bB) P S + E_rep
// depends on the pair vector through |R| (local integrals, repulsion) and
// through the rotation rot(R) of the local frame.  With G = W L W'^T, the
// pair-rotation matrix W[p(mu,nu)][q(a,b)] = rot[mu][a] rot[nu][b] +
// (a != b) rot[mu][b] rot[nu][a] and the local block L(|R|):
//   dE/d|R|  = sum dL o (W^T F W')                           (radial part)
//   dE/dW    = F W' L^T,  dE/dW' = F^T W L                    (rotation part)
// and dE/drot follows from W's bilinear form; the gradient is
//   dE/dR = (dE/d|R|) R/|R| + sum_ij (dE/drot_ij) drot_ij/dR.
// The reversed frame of the core attraction on the second atom (VuvB with
// the vector B -> A) gets its own rotation and adjoint.
#pragma once
#include "nddo_math.cuh"

namespace sgb {

// (mu, nu), mu <= nu, of orbital-pair index p = nu (nu + 1) / 2 + mu
SGB_HD void pair_orbitals(int p, int& mu, int& nu) {
  nu = p >= 6 ? 3 : (p >= 3 ? 2 : (p >= 1 ? 1 : 0));
  mu = p - nu * (nu + 1) / 2;
}

SGB_HD double w_entry(const double r[4][4], int p, int q) {
  int mu, nu, a, b;
  pair_orbitals(p, mu, nu);
  pair_orbitals(q, a, b);
  double w = r[mu][a] * r[nu][b];
  if (a != b) w += r[mu][b] * r[nu][a];
  return w;
}

// adj += c * dW[p][q] / drot
SGB_HD void w_adjoint(const double r[4][4], int p, int q, double c, double adj[4][4]) {
  int mu, nu, a, b;
  pair_orbitals(p, mu, nu);
  pair_orbitals(q, a, b);
  adj[mu][a] += c * r[nu][b];
  adj[nu][b] += c * r[mu][a];
  if (a != b) {
    adj[mu][b] += c * r[nu][a];
    adj[nu][a] += c * r[mu][b];
  }
}

// Rotation of the local frame for the vector (X, Y, Z) given as duals (so the
// reversed frame differentiates with respect to the original vector), with
// the value and gradient of every entry.
struct RotGrad {
  double r[4][4];
  double d[4][4][3];
};
SGB_HD void rotation_grad(const Dual3& X, const Dual3& Y, const Dual3& Z, RotGrad& out) {
  Dual3 rot[4][4], R;
  frame_rotation(X, Y, Z, rot, R);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      out.r[i][j] = rot[i][j].v;
      out.d[i][j][0] = rot[i][j].dx;
      out.d[i][j][1] = rot[i][j].dy;
      out.d[i][j][2] = rot[i][j].dz;
    }
}

SGB_HD void add_rotation_gradient(const RotGrad& rg, const double adj[4][4], double g[3]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 3; ++k) g[k] += adj[i][j] * rg.d[i][j][k];
}

// Density factor of the two-centre energy in orbital-pair form:
//   F[p][q] = sum over the orderings (mu,nu) of p and (la,si) of q of
//             P_mu,nu P_la,si - 1/2 P_mu,la P_nu,si
// with PA, PB the one-atom blocks and PAB the A-rows / B-columns block.
SGB_HD double density_factor(const double PA[4][4], const double PB[4][4], const double PAB[4][4], int p, int q) {
  int mu, nu, la, si;
  pair_orbitals(p, mu, nu);
  pair_orbitals(q, la, si);
  double s = 0;
  for (int o1 = 0; o1 < (mu == nu ? 1 : 2); ++o1) {
    const int m1 = o1 ? nu : mu, n1 = o1 ? mu : nu;
    for (int o2 = 0; o2 < (la == si ? 1 : 2); ++o2) {
      const int l1 = o2 ? si : la, s1 = o2 ? la : si;
      s += PA[m1][n1] * PB[l1][s1] - 0.5 * PAB[m1][l1] * PAB[n1][s1];
    }
  }
  return s;
}

// Unrestricted: the exchange products of the two spins,
// P_a P_a + P_b P_b = 1/2 (P P + S S) with S = P_a - P_b the spin density
// (TwoElectronMatrix.cpp:182-241 with the spin densities).
SGB_HD double density_factor_uhf(const double PA[4][4], const double PB[4][4], const double PAB[4][4],
                                 const double SAB[4][4], int p, int q) {
  int mu, nu, la, si;
  pair_orbitals(p, mu, nu);
  pair_orbitals(q, la, si);
  double s = 0;
  for (int o1 = 0; o1 < (mu == nu ? 1 : 2); ++o1) {
    const int m1 = o1 ? nu : mu, n1 = o1 ? mu : nu;
    for (int o2 = 0; o2 < (la == si ? 1 : 2); ++o2) {
      const int l1 = o2 ? si : la, s1 = o2 ? la : si;
      s += PA[m1][n1] * PB[l1][s1] - 0.5 * (PAB[m1][l1] * PAB[n1][s1] + SAB[m1][l1] * SAB[n1][s1]);
    }
  }
  return s;
}

// fA[p] = sum over the orderings of p of P_mu,nu (one-atom block)
SGB_HD double atom_factor(const double PA[4][4], int p) {
  int mu, nu;
  pair_orbitals(p, mu, nu);
  return mu == nu ? PA[mu][nu] : 2.0 * PA[mu][nu];
}

// Local entries of the column s_B s_B (or of the row s_A s_A when row_zero):
// the ones that do not vanish by the bond-axis symmetry are ss, xx, yy (= xx),
// sz, zz -- orbital-pair indices 0, 2, 5, 6, 9.
SGB_HD int axis_index(int k) { return k == 0 ? 0 : (k == 1 ? 2 : (k == 2 ? 5 : (k == 3 ? 6 : 9))); }

// Column 0 of the local block of A (dA = 10) against the s function of B,
// values and d/dR, indexed by orbital-pair index (10 entries).  coreB selects
// the core-attraction variant (B's Klopman radius replaced by rhoCoreB).
SGB_HD void local_column(const LocalTermTable& tab, double R, const ElemDev& A, const ElemDev& B, bool coreB,
                         double rhoCoreB, double L[10], double dL[10]) {
  for (int i = 0; i < 10; ++i) L[i] = dL[i] = 0.0;
  for (int e = 0; e < kLocalUnique; ++e) {
    if (tab.col[e] != 0) continue;
    local_entry(tab, e, R, A, B, coreB, rhoCoreB, L[tab.row[e]], dL[tab.row[e]]);
  }
  L[5] = L[2];
  dL[5] = dL[2];
}

// The (s_A s_A | s_B s_B) local entry alone (two s-only atoms), or its
// core-attraction variant.
SGB_HD void local_ss(const LocalTermTable& tab, double R, const ElemDev& A, const ElemDev& B, bool coreB,
                     double rhoCoreB, double& L, double& dL) {
  L = dL = 0.0;
  for (int e = 0; e < kLocalUnique; ++e)
    if (tab.row[e] == 0 && tab.col[e] == 0) local_entry(tab, e, R, A, B, coreB, rhoCoreB, L, dL);
}

// Row 0 (s_A s_A against B's 10 orbital pairs) of the two-centre local block.
SGB_HD void local_row(const LocalTermTable& tab, double R, const ElemDev& A, const ElemDev& B, double L[10],
                      double dL[10]) {
  for (int i = 0; i < 10; ++i) L[i] = dL[i] = 0.0;
  for (int e = 0; e < kLocalUnique; ++e) {
    if (tab.row[e] != 0) continue;
    local_entry(tab, e, R, A, B, false, 0.0, L[tab.col[e]], dL[tab.col[e]]);
  }
  L[5] = L[2];
  dL[5] = dL[2];
}

// Overlap contribution of one primitive pair (shells la, lb; primitives i, j)
// to sum_{u,v} f[u][v] dS[u][v]/dR (GTOOverlapMatrixBlock.cpp:70-165).
SGB_HD void overlap_primitive_grad(const ElemDev& A, const ElemDev& B, const double Rv[3], int la, int lb, int i, int j,
                                   const double f[4][4], double g[3]) {
  const double pi = 3.14159265358979323846;
  const Dual3 R[3] = {Dual3(Rv[0], 1, 0, 0), Dual3(Rv[1], 0, 1, 0), Dual3(Rv[2], 0, 0, 1)};
  const Dual3 R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
  const double a = la ? A.p_exp[i] : A.s_exp[i], ca = la ? A.p_coef[i] : A.s_coef[i];
  const double b = lb ? B.p_exp[j] : B.s_exp[j], cb = lb ? B.p_coef[j] : B.s_coef[j];
  const double p = a + b;
  const double s00 = sqrt(pi / p);
  const double s3 = s00 * s00 * s00;
  const Dual3 K = (ca * cb) * dexp((-a * b / p) * R2);
  Dual3 PA[3], PB[3];
  for (int d = 0; d < 3; ++d) {
    PA[d] = (b / p) * R[d];
    PB[d] = PA[d] - R[d];
  }
  Dual3 acc(0.0);
  if (!la && !lb) {
    acc = (s3 * f[0][0]) * K;
  } else if (la && !lb) {
    for (int u = 0; u < 3; ++u) acc += (s3 * f[1 + u][0]) * (PA[u] * K);
  } else if (!la && lb) {
    for (int v = 0; v < 3; ++v) acc += (s3 * f[0][1 + v]) * (PB[v] * K);
  } else {
    for (int u = 0; u < 3; ++u)
      for (int v = 0; v < 3; ++v) {
        const Dual3 fuv = u == v ? PA[u] * PB[u] + Dual3(1.0 / (2 * p)) : PA[u] * PB[v];
        acc += (s3 * f[1 + u][1 + v]) * (fuv * K);
      }
  }
  g[0] += acc.dx;
  g[1] += acc.dy;
  g[2] += acc.dz;
}

}  // namespace sgb
