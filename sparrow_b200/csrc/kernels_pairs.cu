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
#include "nddo_math.cuh"

namespace sgb {

__constant__ LocalTermTable c_local_terms;

void upload_local_terms(const LocalTermTable& tab, cudaStream_t stream) {
  cudaMemcpyToSymbolAsync(c_local_terms, &tab, sizeof(LocalTermTable), 0, cudaMemcpyHostToDevice, stream);
}

__global__ void __launch_bounds__(128) k_pair_values(const PairDev* __restrict__ pairs, int npairs,
                                                      const AtomDev* __restrict__ atoms,
                                                      const ElemDev* __restrict__ elems,
                                                      const DiatomicDev* __restrict__ diat, int method,
                                                      double* __restrict__ ints, double* __restrict__ vcore,
                                                      double* __restrict__ ovl, double* __restrict__ erep) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev pr = pairs[p];
  const AtomDev a = atoms[pr.a], b = atoms[pr.b];
  const ElemDev& A = elems[a.slot];
  const ElemDev& B = elems[b.slot];
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

// Per pair: dE/dR_AB (R_AB = pos_B - pos_A) at density P.
__global__ void __launch_bounds__(64) k_pair_gradient(const PairDev* __restrict__ pairs, int npairs,
                                                       const AtomDev* __restrict__ atoms,
                                                       const ElemDev* __restrict__ elems,
                                                       const DiatomicDev* __restrict__ diat,
                                                       const MolDev* __restrict__ mols, int method,
                                                       const double* __restrict__ Pall, double* __restrict__ gpair) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev pr = pairs[p];
  const AtomDev a = atoms[pr.a], b = atoms[pr.b];
  const MolDev m = mols[pr.mol];
  double g[3];
  pair_gradient(c_local_terms, method, elems[a.slot], elems[b.slot], diat[a.slot * kMaxElementSlots + b.slot],
                b.x - a.x, b.y - a.y, b.z - a.z, Pall + m.mat_off, m.nao, a.ao0, b.ao0, g);
  gpair[(size_t)p * 3 + 0] = g[0];
  gpair[(size_t)p * 3 + 1] = g[1];
  gpair[(size_t)p * 3 + 2] = g[2];
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
}

void launch_gradient(const DeviceBatch& b, cudaStream_t s) {
  if (b.npairs > 0) {
    int th = 64;
    k_pair_gradient<<<(b.npairs + th - 1) / th, th, 0, s>>>(b.pairs, b.npairs, b.atoms, b.elems, b.diat, b.mols,
                                                             b.method, b.P, b.gpair);
  }
  launch_gather_gradient(b, s);
}

void launch_gather_gradient(const DeviceBatch& b, cudaStream_t s) {
  const int th = 128;
  k_gather_gradient<<<(b.natoms + th - 1) / th, th, 0, s>>>(b.mols, b.atoms, b.natoms, b.gpair, b.grad);
}

}  // namespace sgb
