// Pair kernels: two-centre integrals (values) and the nuclear gradient.
//
// One thread per atom pair.  The value kernel writes, per pair, the global
// two-electron block, both core-attraction vectors, the overlap block and
// the core-core repulsion (the density-independent part that the reference
// builds in TwoCenterIntegralContainer::update, OneElectronMatrix::calculate
// and PM6RepulsionEnergy::calculateRepulsion).  The gradient kernel repeats
// the pair math in dual numbers and contracts it with the converged density
// (OneElectronMatrix.cpp:136-229, TwoElectronMatrix.cpp:168-241).
#include <cuda_runtime.h>

#include "kernels.h"
#include "nddo_grad.cuh"
#include "nddo_math.cuh"

namespace sgb {

__constant__ LocalTermTable c_local_terms;

void upload_local_terms(const LocalTermTable& tab, cudaStream_t stream) {
  cudaMemcpyToSymbolAsync(c_local_terms, &tab, sizeof(LocalTermTable), 0, cudaMemcpyHostToDevice, stream);
}

// Values of pair p (see the file comment).
__device__ __forceinline__ void pair_values_one(int p, const PairDev& pr, const AtomDev& a, const AtomDev& b,
                                                const ElemDev& A, const ElemDev& B,
                                                const DiatomicDev* __restrict__ diat, int method,
                                                double* __restrict__ ints, double* __restrict__ vcore,
                                                double* __restrict__ ovl, double* __restrict__ erep) {
  const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
  const int dA = A.nao == 1 ? 1 : 10, dB = B.nao == 1 ? 1 : 10;

  double G[10][10];
  global_block<double>(c_local_terms, A, B, X, Y, Z, G);
  double* out = ints + pr.int_off;
  for (int i = 0; i < dA; ++i)
    for (int j = 0; j < dB; ++j) out[i * dB + j] = G[i][j];

  double V[10];
  core_vector<double>(c_local_terms, A, B, X, Y, Z, V);
  double* vc = vcore + (size_t)p * 20;
  for (int i = 0; i < 10; ++i) vc[i] = i < dA ? V[i] : 0.0;
  core_vector<double>(c_local_terms, B, A, -X, -Y, -Z, V);
  for (int i = 0; i < 10; ++i) vc[10 + i] = i < dB ? V[i] : 0.0;

  double R[3] = {X, Y, Z};
  double S[4][4];
  overlap_block<double>(A, B, R, S);
  double* so = ovl + (size_t)p * 16;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) so[i * 4 + j] = S[i][j];

  double E, dE;
  core_repulsion(method, A, B, diat[a.slot * kMaxElementSlots + b.slot], sqrt(X * X + Y * Y + Z * Z), E, dE);
  erep[p] = E;
}

// Pairs with at least one s-only atom, one thread each.  s/p-s/p pairs cost
// two orders of magnitude more and sit in the same rows of the pair table
// (heavy atoms first): they go to k_pair_values_heavy, so that no warp waits
// on one of them while its other lanes idle.
__global__ void __launch_bounds__(128) k_pair_values(const PairDev* __restrict__ pairs, int npairs,
                                                      const AtomDev* __restrict__ atoms,
                                                      const ElemDev* __restrict__ elems,
                                                      const DiatomicDev* __restrict__ diat, int method,
                                                      double* __restrict__ ints, double* __restrict__ vcore,
                                                      double* __restrict__ ovl, double* __restrict__ erep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev pr = pairs[p];
  const AtomDev a = atoms[pr.a], b = atoms[pr.b];
  const ElemDev& A = elems[a.slot];
  const ElemDev& B = elems[b.slot];
  if (A.nao == 4 && B.nao == 4) return;
  pair_values_one(p, pr, a, b, A, B, diat, method, ints, vcore, ovl, erep);
}

// The s/p-s/p pairs (the heavy-pair list), one thread each.
__global__ void __launch_bounds__(128) k_pair_values_heavy(const int* __restrict__ hh, int nhh,
                                                            const PairDev* __restrict__ pairs,
                                                            const AtomDev* __restrict__ atoms,
                                                            const ElemDev* __restrict__ elems,
                                                            const DiatomicDev* __restrict__ diat, int method,
                                                            double* __restrict__ ints, double* __restrict__ vcore,
                                                            double* __restrict__ ovl, double* __restrict__ erep) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nhh) return;
  const int p = hh[h];
  const PairDev pr = pairs[p];
  const AtomDev a = atoms[pr.a], b = atoms[pr.b];
  pair_values_one(p, pr, a, b, elems[a.slot], elems[b.slot], diat, method, ints, vcore, ovl, erep);
}

// Pair gradient, reverse mode (see nddo_grad.cuh), for pairs with at least
// one s-only atom: one thread per pair, 10-vectors only.  Heavy pairs (both
// atoms s/p) return at once; k_pair_gradient_heavy handles them.
__global__ void __launch_bounds__(128) k_pair_gradient_light(const PairDev* __restrict__ pairs, int npairs,
                                                             const AtomDev* __restrict__ atoms,
                                                             const ElemDev* __restrict__ elems,
                                                             const DiatomicDev* __restrict__ diat,
                                                             const MolDev* __restrict__ mols, int method,
                                                             const double* __restrict__ Pall,
                                                             const double* __restrict__ Paall,
                                                             const double* __restrict__ Pball,
                                                             double* __restrict__ gpair) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev pr = pairs[p];
  const AtomDev a = atoms[pr.a], b = atoms[pr.b];
  const ElemDev& A = elems[a.slot];
  const ElemDev& B = elems[b.slot];
  const int nA = A.nao, nB = B.nao;
  if (nA == 4 && nB == 4) return;
  const MolDev m = mols[pr.mol];
  const int N = m.nao;
  const double* P = Pall + m.mat_off;
  const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
  const double R = sqrt(X * X + Y * Y + Z * Z);
  double PA[4][4] = {}, PB[4][4] = {}, PAB[4][4] = {};
  for (int i = 0; i < nA; ++i)
    for (int j = 0; j < nA; ++j) PA[i][j] = P[(size_t)(a.ao0 + i) * N + a.ao0 + j];
  for (int i = 0; i < nB; ++i)
    for (int j = 0; j < nB; ++j) PB[i][j] = P[(size_t)(b.ao0 + i) * N + b.ao0 + j];
  for (int i = 0; i < nA; ++i)
    for (int j = 0; j < nB; ++j) PAB[i][j] = P[(size_t)(a.ao0 + i) * N + b.ao0 + j];
  // unrestricted: spin density of the off-diagonal block
  const bool uhf = Paall != nullptr;
  double SAB[4][4] = {};
  if (uhf)
    for (int i = 0; i < nA; ++i)
      for (int j = 0; j < nB; ++j) {
        const size_t ij = m.mat_off + (size_t)(a.ao0 + i) * N + b.ao0 + j;
        SAB[i][j] = Paall[ij] - Pball[ij];
      }
  double g[3] = {0, 0, 0};
  double adjA[4][4] = {}, adjB[4][4] = {};
  double dR = 0;
  RotGrad ra, rb;
  const bool rotate = nA == 4 || nB == 4;
  if (rotate) {
    rotation_grad(Dual3(X, 1, 0, 0), Dual3(Y, 0, 1, 0), Dual3(Z, 0, 0, 1), ra);
    rotation_grad(Dual3(-X, -1, 0, 0), Dual3(-Y, 0, -1, 0), Dual3(-Z, 0, 0, -1), rb);
  }
  // two-centre term
  if (!rotate) {
    double L, dL;
    local_ss(c_local_terms, R, A, B, false, 0.0, L, dL);
    dR += (uhf ? density_factor_uhf(PA, PB, PAB, SAB, 0, 0) : density_factor(PA, PB, PAB, 0, 0)) * dL;
  } else {
    double L[10], dL[10];
    if (nB == 1) local_column(c_local_terms, R, A, B, false, 0.0, L, dL);
    else local_row(c_local_terms, R, A, B, L, dL);
    for (int g2 = 0; g2 < 10; ++g2) {
      const int fp = nB == 1 ? g2 : 0, fq = nB == 1 ? 0 : g2;
      const double Fg = uhf ? density_factor_uhf(PA, PB, PAB, SAB, fp, fq) : density_factor(PA, PB, PAB, fp, fq);
      if (Fg == 0.0) continue;
      for (int k = 0; k < 5; ++k) {
        const int q = axis_index(k);
        if (L[q] == 0.0 && dL[q] == 0.0) continue;
        w_adjoint(ra.r, g2, q, Fg * L[q], adjA);
        dR += Fg * w_entry(ra.r, g2, q) * dL[q];
      }
    }
  }
  // core attraction: A's orbitals against B's core (frame A->B), B's against A's (frame B->A)
  for (int side = 0; side < 2; ++side) {
    const ElemDev& O = side ? B : A;    // orbitals
    const ElemDev& C = side ? A : B;    // core
    const double (*PO)[4] = side ? PB : PA;
    const RotGrad& rg = side ? rb : ra;
    double(*adj)[4] = side ? adjB : adjA;
    if (O.nao == 1) {
      double L, dL;
      local_ss(c_local_terms, R, O, C, true, C.pcore, L, dL);
      dR += -C.core * PO[0][0] * dL;
    } else {
      double L[10], dL[10];
      local_column(c_local_terms, R, O, C, true, C.pcore, L, dL);
      for (int g2 = 0; g2 < 10; ++g2) {
        const double f = -C.core * atom_factor(PO, g2);
        if (f == 0.0) continue;
        for (int k = 0; k < 5; ++k) {
          const int q = axis_index(k);
          if (L[q] == 0.0 && dL[q] == 0.0) continue;
          w_adjoint(rg.r, g2, q, f * L[q], adj);
          dR += f * w_entry(rg.r, g2, q) * dL[q];
        }
      }
    }
  }
  // overlap (resonance integrals)
  {
    double f[4][4] = {};
    for (int i = 0; i < nA; ++i)
      for (int j = 0; j < nB; ++j)
        f[i][j] = ((i == 0 ? A.betaS : A.betaP) + (j == 0 ? B.betaS : B.betaP)) * PAB[i][j];
    const double Rv[3] = {X, Y, Z};
    for (int la = 0; la < (nA == 4 ? 2 : 1); ++la)
      for (int lb = 0; lb < (nB == 4 ? 2 : 1); ++lb)
        for (int i = 0; i < 6; ++i)
          for (int j = 0; j < 6; ++j) overlap_primitive_grad(A, B, Rv, la, lb, i, j, f, g);
  }
  // core repulsion
  {
    double E, dE;
    core_repulsion(method, A, B, diat[a.slot * kMaxElementSlots + b.slot], R, E, dE);
    dR += dE;
  }
  g[0] += dR * X / R;
  g[1] += dR * Y / R;
  g[2] += dR * Z / R;
  if (rotate) {
    add_rotation_gradient(ra, adjA, g);
    add_rotation_gradient(rb, adjB, g);
  }
  gpair[(size_t)p * 3 + 0] = g[0];
  gpair[(size_t)p * 3 + 1] = g[1];
  gpair[(size_t)p * 3 + 2] = g[2];
}

// Pair gradient, reverse mode, for pairs of two s/p atoms: one warp per pair
// with the 10 x 10 blocks in shared memory.  Lanes split the 21 unique local
// integrals, the 100-entry matrices and products, the rotation adjoints and
// the 144 primitive pairs of the overlap; each lane's partial gradient is
// summed across the warp at the end.
constexpr int kGradWarps = 4;
struct HeavyGradShared {
  double L[100], dL[100], W[100], F[100], T1[100], T2[100];
  double Lc[10], dLc[10], Lcb[10], dLcb[10];
  double PA[4][4], PB[4][4], PAB[4][4], SAB[4][4];
  RotGrad ra, rb;
};

__global__ void __launch_bounds__(kGradWarps * 32) k_pair_gradient_heavy(
    const int* __restrict__ hh, int nhh, const PairDev* __restrict__ pairs, const AtomDev* __restrict__ atoms,
    const ElemDev* __restrict__ elems, const DiatomicDev* __restrict__ diat, const MolDev* __restrict__ mols, int method,
    const double* __restrict__ Pall, const double* __restrict__ Paall, const double* __restrict__ Pball,
    double* __restrict__ gpair) {
  __shared__ HeavyGradShared shm[kGradWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.x * kGradWarps + warp;
  if (w >= nhh) return;  // uniform per warp
  HeavyGradShared& s = shm[warp];
  const int p = hh[w];
  const PairDev pr = pairs[p];
  const AtomDev a = atoms[pr.a], b = atoms[pr.b];
  const ElemDev& A = elems[a.slot];
  const ElemDev& B = elems[b.slot];
  const MolDev m = mols[pr.mol];
  const int N = m.nao;
  const double* P = Pall + m.mat_off;
  const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
  const double R = sqrt(X * X + Y * Y + Z * Z);
  const LocalTermTable& tab = c_local_terms;
  if (lane < 16) {
    const int i = lane >> 2, j = lane & 3;
    s.PA[i][j] = P[(size_t)(a.ao0 + i) * N + a.ao0 + j];
    s.PB[i][j] = P[(size_t)(b.ao0 + i) * N + b.ao0 + j];
    s.PAB[i][j] = P[(size_t)(a.ao0 + i) * N + b.ao0 + j];
    const size_t ij = m.mat_off + (size_t)(a.ao0 + i) * N + b.ao0 + j;
    s.SAB[i][j] = Paall ? Paall[ij] - Pball[ij] : 0.0;
  }
  if (lane == 30) rotation_grad(Dual3(X, 1, 0, 0), Dual3(Y, 0, 1, 0), Dual3(Z, 0, 0, 1), s.ra);
  if (lane == 31) rotation_grad(Dual3(-X, -1, 0, 0), Dual3(-Y, 0, -1, 0), Dual3(-Z, 0, 0, -1), s.rb);
  for (int k = lane; k < 100; k += 32) s.L[k] = s.dL[k] = 0.0;
  if (lane < 10) s.Lc[lane] = s.dLc[lane] = s.Lcb[lane] = s.dLcb[lane] = 0.0;
  __syncwarp();
  if (lane < kLocalUnique) {
    const int r = tab.row[lane], c = tab.col[lane];
    double v, d;
    local_entry(tab, lane, R, A, B, false, 0.0, v, d);
    s.L[r * 10 + c] = v;
    s.dL[r * 10 + c] = d;
    if (c == 0) {
      local_entry(tab, lane, R, A, B, true, B.pcore, v, d);
      s.Lc[r] = v;
      s.dLc[r] = d;
      local_entry(tab, lane, R, B, A, true, A.pcore, v, d);
      s.Lcb[r] = v;
      s.dLcb[r] = d;
    }
  }
  __syncwarp();
  if (lane == 0) {
    local_copies(10, 10, reinterpret_cast<double(*)[10]>(s.L), reinterpret_cast<double(*)[10]>(s.dL));
    s.Lc[5] = s.Lc[2];
    s.dLc[5] = s.dLc[2];
    s.Lcb[5] = s.Lcb[2];
    s.dLcb[5] = s.dLcb[2];
  }
  for (int k = lane; k < 100; k += 32) {
    s.W[k] = w_entry(s.ra.r, k / 10, k % 10);
    s.F[k] = Paall ? density_factor_uhf(s.PA, s.PB, s.PAB, s.SAB, k / 10, k % 10)
                   : density_factor(s.PA, s.PB, s.PAB, k / 10, k % 10);
  }
  __syncwarp();
  // T1 = F W, T2 = F^T W
  for (int k = lane; k < 100; k += 32) {
    const int r = k / 10, c = k % 10;
    double t1 = 0, t2 = 0;
    for (int l = 0; l < 10; ++l) {
      t1 += s.F[r * 10 + l] * s.W[l * 10 + c];
      t2 += s.F[l * 10 + r] * s.W[l * 10 + c];
    }
    s.T1[k] = t1;
    s.T2[k] = t2;
  }
  __syncwarp();
  double adjA[4][4] = {}, adjB[4][4] = {};
  double dR = 0, g[3] = {0, 0, 0};
  // two-centre: dE/dW[p][q] = sum_j T1[p][j] L[q][j] + sum_a T2[p][a] L[a][q];
  // dE/dL[x][y] = sum_g W[g][x] T1[g][y]
  for (int k = lane; k < 100; k += 32) {
    const int pp = k / 10, qq = k % 10;
    double adw = 0;
    for (int j = 0; j < 10; ++j) adw += s.T1[pp * 10 + j] * s.L[qq * 10 + j] + s.T2[pp * 10 + j] * s.L[j * 10 + qq];
    if (adw != 0.0) w_adjoint(s.ra.r, pp, qq, adw, adjA);
    if (s.dL[k] != 0.0) {
      double mm = 0;
      for (int g2 = 0; g2 < 10; ++g2) mm += s.W[g2 * 10 + pp] * s.T1[g2 * 10 + qq];
      dR += s.dL[k] * mm;
    }
  }
  // core attraction (both sides), 10 orbital pairs x 5 axis entries each
  for (int k = lane; k < 100; k += 32) {
    const int side = k / 50, g2 = (k % 50) / 5, q = axis_index(k % 5);
    const double* Lv = side ? s.Lcb : s.Lc;
    const double* dLv = side ? s.dLcb : s.dLc;
    if (Lv[q] == 0.0 && dLv[q] == 0.0) continue;
    const double f = -(side ? A.core : B.core) * atom_factor(side ? s.PB : s.PA, g2);
    if (f == 0.0) continue;
    const RotGrad& rg = side ? s.rb : s.ra;
    w_adjoint(rg.r, g2, q, f * Lv[q], side ? adjB : adjA);
    dR += f * w_entry(rg.r, g2, q) * dLv[q];
  }
  // overlap: 2 x 2 shells x 6 x 6 primitives
  {
    double f[4][4];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        f[i][j] = ((i == 0 ? A.betaS : A.betaP) + (j == 0 ? B.betaS : B.betaP)) * s.PAB[i][j];
    const double Rv[3] = {X, Y, Z};
    for (int k = lane; k < 144; k += 32)
      overlap_primitive_grad(A, B, Rv, k / 72, (k / 36) % 2, (k / 6) % 6, k % 6, f, g);
  }
  if (lane == 0) {
    double E, dE;
    core_repulsion(method, A, B, diat[a.slot * kMaxElementSlots + b.slot], R, E, dE);
    dR += dE;
  }
  g[0] += dR * X / R;
  g[1] += dR * Y / R;
  g[2] += dR * Z / R;
  add_rotation_gradient(s.ra, adjA, g);
  add_rotation_gradient(s.rb, adjB, g);
  for (int k = 0; k < 3; ++k)
    for (int o = 16; o > 0; o >>= 1) g[k] += __shfl_xor_sync(0xffffffffu, g[k], o);
  if (lane == 0) {
    gpair[(size_t)p * 3 + 0] = g[0];
    gpair[(size_t)p * 3 + 1] = g[1];
    gpair[(size_t)p * 3 + 2] = g[2];
  }
}

// Atom gradient: sum of the pair gradients (+ for the second atom of a pair,
// - for the first).  Pairs of a molecule are stored for i<j in row order, so
// the index of pair (i, j) is i*n - i(i+1)/2 + (j - i - 1).
__global__ void k_gather_gradient(const MolDev* __restrict__ mols, const AtomDev* __restrict__ atoms, int natoms,
                                  const double* __restrict__ gpair, double* __restrict__ grad) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natoms) return;
  const MolDev m = mols[atoms[a].mol];
  const int n = m.nat, i = a - m.atom0;
  double g[3] = {0, 0, 0};
  for (int j = 0; j < n; ++j) {
    if (j == i) continue;
    int lo = i < j ? i : j, hi = i < j ? j : i;
    long long pidx = (long long)m.pair0 + (long long)lo * n - (long long)lo * (lo + 1) / 2 + (hi - lo - 1);
    double s = (i == hi) ? 1.0 : -1.0;
    for (int d = 0; d < 3; ++d) g[d] += s * gpair[pidx * 3 + d];
  }
  for (int d = 0; d < 3; ++d) grad[(size_t)a * 3 + d] = g[d];
}

// One CTA per molecule.  Pair p of a molecule with n atoms is (lo, hi), lo <
// hi, in row-major order: rowstart(l) = l n - l (l + 1) / 2 pairs precede row
// l.  With block sizes c(a) = 1 (s atom) or 10 (sp atom), suffix sums
// S(a) = sum_{h >= a} c(h) and R(l) = sum_{l' < l} c(l') S(l' + 1), the
// integral block of (lo, hi) starts at R(lo) + c(lo) (S(lo + 1) - S(hi))
// past the molecule's first block, the same order the integral kernel and
// the oracle use.  Heavy pairs (both atoms sp) are listed in the same order.
__global__ void __launch_bounds__(256) k_build_pairs(const MolDev* __restrict__ mols,
                                                     const AtomDev* __restrict__ atoms,
                                                     const ElemDev* __restrict__ elems, PairDev* __restrict__ pairs,
                                                     int* __restrict__ hh_pairs, int* __restrict__ flag) {
  extern __shared__ long long sm_pairs[];
  const MolDev m = mols[blockIdx.x];
  const int n = m.nat;
  long long* R = sm_pairs;                              // [n]
  int* S = reinterpret_cast<int*>(R + n);              // [n + 1]
  int* heavy = S + n + 1;                              // [n]
  __shared__ int nheavy;
  if (threadIdx.x == 0) {
    S[n] = 0;
    for (int a = n - 1; a >= 0; --a) S[a] = S[a + 1] + (elems[atoms[m.atom0 + a].slot].nao == 1 ? 1 : 10);
    long long r = 0;
    int h = 0;
    for (int a = 0; a < n; ++a) {
      R[a] = r;
      const int c = S[a] - S[a + 1];
      r += (long long)c * S[a + 1];
      if (c == 10) heavy[h++] = a;
    }
    nheavy = h;
  }
  __syncthreads();
  const int np = m.npairs;
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    // largest lo with rowstart(lo) <= p
    const double nn = n - 0.5;
    int lo = (int)(nn - sqrt(fmax(nn * nn - 2.0 * p, 0.0)));
    if (lo < 0) lo = 0;
    while (lo > 0 && (long long)lo * n - (long long)lo * (lo + 1) / 2 > p) --lo;
    while ((long long)(lo + 1) * n - (long long)(lo + 1) * (lo + 2) / 2 <= p) ++lo;
    const int hi = p - (lo * n - lo * (lo + 1) / 2) + lo + 1;
    const int c = S[lo] - S[lo + 1];
    PairDev pd;
    pd.a = m.atom0 + lo;
    pd.b = m.atom0 + hi;
    pd.mol = blockIdx.x;
    pd.int_off = (int)(m.int_off + R[lo] + (long long)c * (S[lo + 1] - S[hi]));
    pairs[m.pair0 + p] = pd;
    const AtomDev A = atoms[pd.a], B = atoms[pd.b];
    const double dx = B.x - A.x, dy = B.y - A.y, dz = B.z - A.z;
    if (dx * dx + dy * dy + dz * dz < 1e-12) atomicCAS(flag, 0, m.pair0 + p + 1);
  }
  const int H = nheavy;
  const int nhh = H * (H - 1) / 2;
  for (int q = threadIdx.x; q < nhh; q += blockDim.x) {
    const double hh = H - 0.5;
    int i = (int)(hh - sqrt(fmax(hh * hh - 2.0 * q, 0.0)));
    if (i < 0) i = 0;
    while (i > 0 && i * H - i * (i + 1) / 2 > q) --i;
    while ((i + 1) * H - (i + 1) * (i + 2) / 2 <= q) ++i;
    const int j = q - (i * H - i * (i + 1) / 2) + i + 1;
    const int lo = heavy[i], hi = heavy[j];
    hh_pairs[m.hh0 + q] = m.pair0 + lo * n - lo * (lo + 1) / 2 + (hi - lo - 1);
  }
}

void launch_build_pairs(const DeviceBatch& b, int max_nat, int* flag, cudaStream_t s) {
  if (b.nmol == 0) return;
  const size_t smem = sizeof(long long) * max_nat + sizeof(int) * (2 * (size_t)max_nat + 1);
  cudaFuncSetAttribute(k_build_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_build_pairs<<<b.nmol, 256, smem, s>>>(b.mols, b.atoms, b.elems, b.pairs, b.hh_pairs, flag);
}

void launch_pair_values(const DeviceBatch& b, cudaStream_t s) {
  if (b.npairs == 0) return;
  int th = 128;
  k_pair_values<<<(b.npairs + th - 1) / th, th, 0, s>>>(b.pairs, b.npairs, b.atoms, b.elems, b.diat, b.method,
                                                         b.ints, b.vcore, b.ovl, b.erep);
  if (b.nhh_total > 0)
    k_pair_values_heavy<<<(b.nhh_total + th - 1) / th, th, 0, s>>>(b.hh_pairs, b.nhh_total, b.pairs, b.atoms,
                                                                   b.elems, b.diat, b.method, b.ints, b.vcore,
                                                                   b.ovl, b.erep);
}

void launch_gradient(const DeviceBatch& b, cudaStream_t s) {
  if (b.npairs > 0) {
    const int th = 128;
    k_pair_gradient_light<<<(b.npairs + th - 1) / th, th, 0, s>>>(b.pairs, b.npairs, b.atoms, b.elems, b.diat, b.mols,
                                                                   b.method, b.P, b.uhf ? b.Pa : nullptr,
                                                                   b.uhf ? b.Pb : nullptr, b.gpair);
  }
  if (b.nhh_total > 0) {
    k_pair_gradient_heavy<<<(b.nhh_total + kGradWarps - 1) / kGradWarps, kGradWarps * 32, 0, s>>>(
        b.hh_pairs, b.nhh_total, b.pairs, b.atoms, b.elems, b.diat, b.mols, b.method, b.P, b.uhf ? b.Pa : nullptr,
        b.uhf ? b.Pb : nullptr, b.gpair);
  }
  launch_gather_gradient(b, s);
}

void launch_gather_gradient(const DeviceBatch& b, cudaStream_t s) {
  const int th = 128;
  k_gather_gradient<<<(b.natoms + th - 1) / th, th, 0, s>>>(b.mols, b.atoms, b.natoms, b.gpair, b.grad);
}

}  // namespace sgb
