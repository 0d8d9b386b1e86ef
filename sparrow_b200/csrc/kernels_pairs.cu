// Pair kernels: two-centre integrals (values) and the nuclear gradient.
//
// The value kernels (a thread per pair with hydrogen, a warp per s/p-s/p
// pair) write, per pair, the global two-electron block, both core-attraction
// vectors, the overlap block and the core-core repulsion (the
// density-independent part that the reference builds in
// TwoCenterIntegralContainer::update, OneElectronMatrix::calculate and
// PM6RepulsionEnergy::calculateRepulsion).  The gradient kernels contract the
// pair math's derivatives with the converged density in reverse mode
// (OneElectronMatrix.cpp:136-229, TwoElectronMatrix.cpp:168-241).
#include <cuda_runtime.h>

#include "kernels.h"
#include "nddo_grad.cuh"
#include "nddo_math.cuh"

namespace sgb {

__constant__ LocalTermTable c_local_terms;
// Global-memory copy of the term table, for reads at lane-dependent indices
// (the constant bank serialises a warp's distinct addresses).
__device__ LocalTermTable g_local_terms;

void upload_local_terms(const LocalTermTable& tab, cudaStream_t stream) {
  cudaMemcpyToSymbolAsync(c_local_terms, &tab, sizeof(LocalTermTable), 0, cudaMemcpyHostToDevice, stream);
  cudaMemcpyToSymbolAsync(g_local_terms, &tab, sizeof(LocalTermTable), 0, cudaMemcpyHostToDevice, stream);
}

// Evaluated local entries (table entries of local_terms.cpp, whose order
// follows Local2c2eMatrix.cpp:91-149) of the sigma column (p | ss) and row
// (ss | p) for the local orbital pairs ss, xx (= yy), sz and zz: the only
// local entries that are nonzero when one side is an s function or a bare
// core.
constexpr int kColSS = 0, kColXX = 4, kColSZ = 5, kColZZ = 6;
constexpr int kRowSS = 0, kRowXX = 1, kRowSZ = 2, kRowZZ = 3;

// Value of evaluated local entry e (no derivative; rsqrt of the squared
// charge distance, within an ulp of 1/sqrt).
__device__ __forceinline__ double local_value(const LocalTermTable& tab, int e, double R, const ElemDev& A,
                                              const ElemDev& B, bool coreB, double rhoCoreB) {
  double val = 0.0;
  const int s = tab.start[e], n = tab.count[e];
  for (int t = s; t < s + n; ++t) {
    const LocalTerm& T = tab.term[t];
    const double rA = A.rho[T.c1];
    const double rB = coreB ? rhoCoreB : B.rho[T.c2];
    const double D1 = A.D[T.c1];
    const double d2 = coreB ? 0.0 : B.D[T.c2];
    const double dx = d2 * T.x2 - D1 * T.x1;
    const double dy = d2 * T.y2 - D1 * T.y1;
    const double dz = R + d2 * T.z2 - D1 * T.z1;
    const double rr = rA + rB;
    val = fma(T.q, rsqrt(dx * dx + dy * dy + dz * dz + rr * rr), val);
  }
  return val;
}

// Orbital pair (mu, nu), mu <= nu, of packed index p = nu (nu + 1) / 2 + mu.
__device__ __forceinline__ void pair_of(int p, int& mu, int& nu) {
  nu = p < 1 ? 0 : (p < 3 ? 1 : (p < 6 ? 2 : 3));
  mu = p - nu * (nu + 1) / 2;
}

// Global value of orbital pair g of an s/p atom from a local block whose
// other side is an s function or a bare core.  Only the sigma entries ss,
// sz, xx = yy and zz are nonzero in the local frame, and global_block's
// pair rotation reduces to G[ss] = L_ss, G[s nu] = rot[nu][z] L_sz,
// G[mu nu] = sum_m rot[mu][m] rot[nu][m] L_mm for p orbitals mu, nu.
__device__ __forceinline__ double sigma_entry(const double rot[4][4], int g, double Lss, double Lsz, double Lxx,
                                              double Lzz) {
  int mu, nu;
  pair_of(g, mu, nu);
  if (nu == 0) return Lss;
  if (mu == 0) return rot[nu][3] * Lsz;
  return rot[mu][1] * rot[nu][1] * Lxx + rot[mu][2] * rot[nu][2] * Lxx + rot[mu][3] * rot[nu][3] * Lzz;
}

// Entry (p, q) of global_block's pair rotation W (both atoms s/p, same frame).
__device__ __forceinline__ double pair_rotation_entry(const double rot[4][4], int p, int q) {
  int mu, nu, m, n;
  pair_of(p, mu, nu);
  pair_of(q, m, n);
  double w = rot[mu][m] * rot[nu][n];
  if (m != n) w += rot[mu][n] * rot[nu][m];
  return w;
}

// Overlap block of an atom pair from five primitive sums.  With p = a + b and
// K = c_a c_b (pi/p)^(3/2) exp(-a b R^2 / p) over the 6 x 6 STO-6G primitive
// products of a shell pair (R = B - A; Gaussian product centre A + (b/p) R),
// the entries of overlap_block (orbital i of A, j of B; 0 = s, 1..3 = x, y, z)
// are
//   S[s][s] = sum_ss K                S[u][s] = R_u sum_ps K b/p
//   S[s][w] = -R_w sum_sp K a/p       S[u][w] = -R_u R_w sum_pp K a b/p^2 + [u = w] sum_pp K / (2p)
// so that every primitive product costs one exponential, shared by the
// entries of its shell pair.
struct OverlapSums {
  double ss, sp, ps, pp, pp0;
};

// Adds primitive product (ii, jj) of shell pair `shell` (0 ss, 1 s on A / p on
// B, 2 p on A / s on B, 3 pp) to o; R2 = |R|^2.  kMu: also to m, weighted by
// mu = a b / p (for the gradient, see overlap_gradient).
template <bool kMu>
__device__ __forceinline__ void overlap_accumulate(const ElemDev& A, const ElemDev& B, int shell, int ii, int jj,
                                                   double R2, OverlapSums& o, OverlapSums* m = nullptr) {
  const double pi = 3.14159265358979323846;
  const bool la = shell >= 2, lb = (shell & 1) != 0;
  const double a = la ? A.p_exp[ii] : A.s_exp[ii], ca = la ? A.p_coef[ii] : A.s_coef[ii];
  const double b = lb ? B.p_exp[jj] : B.s_exp[jj], cb = lb ? B.p_coef[jj] : B.s_coef[jj];
  const double ip = 1.0 / (a + b);
  const double mu = a * b * ip;
  const double s00 = sqrt(pi * ip);
  const double K = (s00 * s00 * s00) * ((ca * cb) * exp(-mu * R2));
  switch (shell) {
    case 0:
      o.ss += K;
      if (kMu) m->ss += mu * K;
      break;
    case 1: {
      const double w = K * (a * ip);
      o.sp += w;
      if (kMu) m->sp += mu * w;
      break;
    }
    case 2: {
      const double w = K * (b * ip);
      o.ps += w;
      if (kMu) m->ps += mu * w;
      break;
    }
    default: {
      const double w = K * (mu * ip), w0 = K * (0.5 * ip);
      o.pp += w;
      o.pp0 += w0;
      if (kMu) {
        m->pp += mu * w;
        m->pp0 += mu * w0;
      }
      break;
    }
  }
}

// Gradient with respect to R = B - A of the overlap energy sum_ij f[i][j]
// S[i][j] (f zero outside the atoms' orbitals) from the sums o and their
// mu-weighted copies m: every sum X = sum K w has dX/dR = -2 R sum mu K w.
__device__ __forceinline__ void overlap_gradient(const OverlapSums& o, const OverlapSums& m, const double f[4][4],
                                                 const double R[3], double g[3]) {
  double a = 0.0, b = 0.0, c = 0.0, t = 0.0, fR[3], Rf[3];
  for (int u = 0; u < 3; ++u) {
    a += f[1 + u][0] * R[u];
    b += f[0][1 + u] * R[u];
    t += f[1 + u][1 + u];
    fR[u] = f[1 + u][1] * R[0] + f[1 + u][2] * R[1] + f[1 + u][3] * R[2];
    Rf[u] = f[1][1 + u] * R[0] + f[2][1 + u] * R[1] + f[3][1 + u] * R[2];
  }
  for (int u = 0; u < 3; ++u) c += R[u] * fR[u];
  const double radial = -2.0 * (f[0][0] * m.ss + a * m.ps - b * m.sp - c * m.pp + t * m.pp0);
  for (int d = 0; d < 3; ++d)
    g[d] += radial * R[d] + f[1 + d][0] * o.ps - f[0][1 + d] * o.sp - (fR[d] + Rf[d]) * o.pp;
}

__device__ __forceinline__ double overlap_from_sums(const OverlapSums& o, const double R[3], int i, int j) {
  if (i == 0 && j == 0) return o.ss;
  if (j == 0) return R[i - 1] * o.ps;
  if (i == 0) return -R[j - 1] * o.sp;
  return -R[i - 1] * R[j - 1] * o.pp + (i == j ? o.pp0 : 0.0);
}

// Pairs with at least one s-only atom, one thread each.  Their local blocks
// are sigma columns or rows (or the single (ss|ss)), so the global values
// follow from a few local entries and the frame rotation in closed form
// (sigma_entry), with no 10 x 10 intermediates.  s/p-s/p pairs cost two
// orders of magnitude more and sit in the same rows of the pair table (heavy
// atoms first): they go to k_pair_values_heavy, so that no warp waits on one
// of them while its other lanes idle.
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
  const LocalTermTable& tab = c_local_terms;
  const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
  double rot[4][4], R;
  frame_rotation<double>(X, Y, Z, rot, R);
  // two-centre block (dA x dB with dA, dB in {1, 10})
  double* out = ints + pr.int_off;
  if (A.nao == 1 && B.nao == 1) {
    out[0] = local_value(tab, kColSS, R, A, B, false, 0.0);
  } else if (A.nao == 4) {
    const double ss = local_value(tab, kColSS, R, A, B, false, 0.0), sz = local_value(tab, kColSZ, R, A, B, false, 0.0);
    const double xx = local_value(tab, kColXX, R, A, B, false, 0.0), zz = local_value(tab, kColZZ, R, A, B, false, 0.0);
    for (int g = 0; g < 10; ++g) out[g] = sigma_entry(rot, g, ss, sz, xx, zz);
  } else {
    const double ss = local_value(tab, kRowSS, R, A, B, false, 0.0), sz = local_value(tab, kRowSZ, R, A, B, false, 0.0);
    const double xx = local_value(tab, kRowXX, R, A, B, false, 0.0), zz = local_value(tab, kRowZZ, R, A, B, false, 0.0);
    for (int g = 0; g < 10; ++g) out[g] = sigma_entry(rot, g, ss, sz, xx, zz);
  }
  // core attraction: A's orbitals against B's core, B's against A's, both in
  // the frame of A -> B (reversing the axis negates the frame's z column,
  // which enters the sigma entries through L_sz alone)
  double* vc = vcore + (size_t)p * 20;
  if (A.nao == 4) {
    const double ss = local_value(tab, kColSS, R, A, B, true, B.pcore), sz = local_value(tab, kColSZ, R, A, B, true, B.pcore);
    const double xx = local_value(tab, kColXX, R, A, B, true, B.pcore), zz = local_value(tab, kColZZ, R, A, B, true, B.pcore);
    for (int g = 0; g < 10; ++g) vc[g] = (-B.core) * sigma_entry(rot, g, ss, sz, xx, zz);
  } else {
    vc[0] = (-B.core) * local_value(tab, kColSS, R, A, B, true, B.pcore);
    for (int g = 1; g < 10; ++g) vc[g] = 0.0;
  }
  if (B.nao == 4) {
    const double ss = local_value(tab, kColSS, R, B, A, true, A.pcore), sz = local_value(tab, kColSZ, R, B, A, true, A.pcore);
    const double xx = local_value(tab, kColXX, R, B, A, true, A.pcore), zz = local_value(tab, kColZZ, R, B, A, true, A.pcore);
    for (int g = 0; g < 10; ++g) vc[10 + g] = (-A.core) * sigma_entry(rot, g, ss, -sz, xx, zz);
  } else {
    vc[10] = (-A.core) * local_value(tab, kColSS, R, B, A, true, A.pcore);
    for (int g = 1; g < 10; ++g) vc[10 + g] = 0.0;
  }
  // overlap block (the entries outside the atoms' orbitals are zero); the
  // shell pairs present: ss, and sp or ps when one atom has p functions
  const double Rv[3] = {X, Y, Z};
  OverlapSums o = {0.0, 0.0, 0.0, 0.0, 0.0};
  const double R2v = X * X + Y * Y + Z * Z;
  const int shell2 = B.nao == 4 ? 1 : (A.nao == 4 ? 2 : -1);
  for (int k = 0; k < 36; ++k) overlap_accumulate<false>(A, B, 0, k / 6, k % 6, R2v, o);
  if (shell2 > 0)
    for (int k = 0; k < 36; ++k) overlap_accumulate<false>(A, B, shell2, k / 6, k % 6, R2v, o);
  double* so = ovl + (size_t)p * 16;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) so[i * 4 + j] = (i < A.nao && j < B.nao) ? overlap_from_sums(o, Rv, i, j) : 0.0;
  double E, dE;
  core_repulsion(method, A, B, diat[a.slot * kMaxElementSlots + b.slot], R, E, dE);
  erep[p] = E;
}

// One point-charge term of a local entry (local_value's summand).
__device__ __forceinline__ double term_value(const LocalTerm& T, double R, const ElemDev& A, const ElemDev& B,
                                             bool coreB, double rhoCoreB) {
  const double rA = A.rho[T.c1];
  const double rB = coreB ? rhoCoreB : B.rho[T.c2];
  const double D1 = A.D[T.c1];
  const double d2 = coreB ? 0.0 : B.D[T.c2];
  const double dx = d2 * T.x2 - D1 * T.x1;
  const double dy = d2 * T.y2 - D1 * T.y1;
  const double dz = R + d2 * T.z2 - D1 * T.z1;
  const double rr = rA + rB;
  return T.q * rsqrt(dx * dx + dy * dy + dz * dz + rr * rr);
}

__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Symmetry copies of the local 10 x 10 block (Local2c2eMatrix.cpp:91-149) as
// flat (destination, source) indices; every source is an evaluated entry.
__device__ const unsigned char kLocalCopies[12][2] = {{5, 2},  {50, 20}, {33, 11}, {38, 17}, {52, 25}, {55, 22},
                                                      {56, 26}, {59, 29}, {65, 62}, {83, 71}, {88, 77}, {95, 92}};

// The s/p-s/p pairs (the heavy-pair list), a warp per group of 32 pairs.
// First thread per pair: the frame rotation, distance and core repulsion of
// the lane's pair, staged in shared memory.  Then pair by pair the warp
// shares the work:
//   - the point-charge terms of the 21 evaluated local integrals and of the
//     two core-attraction sigma columns, one term per lane (coalesced reads
//     of g_local_terms), summed per entry from shared memory;
//   - the 4 x 36 primitive products of the overlap block, one exponential
//     each, reduced over the warp into the five OverlapSums;
//   - the symmetry copies of the local block and its rotation G = W L W^T
//     with the pair rotation W of the common frame (global_block), one
//     output entry per lane step.
// The core attraction of B's orbitals is taken in A's frame: reversing the
// pair axis negates only the frame's z column, which enters the sigma
// entries through L_sz alone.
constexpr int kValWarps = 4;
constexpr int kValGroup = 32;
struct HeavyValShared {
  double frame[kValGroup][13];  // 3 x 3 p block of the frame rotation (row-major), R, and B - A
  int pair[kValGroup], sa[kValGroup], sb[kValGroup], ioff[kValGroup];
  double v[kPairTermSlots];  // term values, then the product L W^T
  double L[100], W[100];
};

__global__ void __launch_bounds__(kValWarps * 32) k_pair_values_heavy(
    const int* __restrict__ hh, int nhh, const PairDev* __restrict__ pairs, const AtomDev* __restrict__ atoms,
    const ElemDev* __restrict__ elems, const DiatomicDev* __restrict__ diat, int method, double* __restrict__ ints,
    double* __restrict__ vcore, double* __restrict__ ovl, double* __restrict__ erep) {
  __shared__ HeavyValShared shm[kValWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g0 = (blockIdx.x * kValWarps + warp) * kValGroup;
  if (g0 >= nhh) return;  // uniform per warp
  HeavyValShared& s = shm[warp];
  const int ng = min(kValGroup, nhh - g0);
  if (lane < ng) {
    const int p = hh[g0 + lane];
    const PairDev pr = pairs[p];
    const AtomDev a = atoms[pr.a], b = atoms[pr.b];
    const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
    double rot[4][4], R;
    frame_rotation<double>(X, Y, Z, rot, R);
    double* f = s.frame[lane];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) f[i * 3 + j] = rot[1 + i][1 + j];
    f[9] = R;
    f[10] = X;
    f[11] = Y;
    f[12] = Z;
    s.pair[lane] = p;
    s.sa[lane] = a.slot;
    s.sb[lane] = b.slot;
    s.ioff[lane] = pr.int_off;
    double E, dE;
    core_repulsion(method, elems[a.slot], elems[b.slot], diat[a.slot * kMaxElementSlots + b.slot], R, E, dE);
    erep[p] = E;
  }
  __syncwarp();
  const LocalTermTable& tab = g_local_terms;
  const int nT = tab.n_terms;
  // core-attraction terms per side: the sigma column's ss, sz, xx, zz entries in turn
  const int c0 = tab.count[kColSS], c1 = c0 + tab.count[kColSZ], c2 = c1 + tab.count[kColXX];
  const int nc = c2 + tab.count[kColZZ];
  const int njobs = nT + 2 * nc;
  for (int i = 0; i < ng; ++i) {
    const ElemDev& A = elems[s.sa[i]];
    const ElemDev& B = elems[s.sb[i]];
    const double* f = s.frame[i];
    double rot[4][4];
    rot[0][0] = 1.0;
    for (int k = 1; k < 4; ++k) rot[0][k] = rot[k][0] = 0.0;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) rot[1 + r][1 + c] = f[r * 3 + c];
    const double R = f[9];
    const double Rv[3] = {f[10], f[11], f[12]};
    for (int k = lane; k < 100; k += 32) {
      s.L[k] = 0.0;
      s.W[k] = pair_rotation_entry(rot, k / 10, k % 10);
    }
    for (int j = lane; j < njobs; j += 32) {
      double v;
      if (j < nT) {
        v = term_value(tab.term[j], R, A, B, false, 0.0);
      } else {
        const int side = j - nT >= nc, k = j - nT - side * nc;
        const int t = k < c0   ? tab.start[kColSS] + k
                      : k < c1 ? tab.start[kColSZ] + (k - c0)
                      : k < c2 ? tab.start[kColXX] + (k - c1)
                               : tab.start[kColZZ] + (k - c2);
        v = side ? term_value(tab.term[t], R, B, A, true, A.pcore) : term_value(tab.term[t], R, A, B, true, B.pcore);
      }
      s.v[j] = v;
    }
    OverlapSums o = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double R2 = Rv[0] * Rv[0] + Rv[1] * Rv[1] + Rv[2] * Rv[2];
    for (int k = lane; k < 144; k += 32) overlap_accumulate<false>(A, B, k / 36, (k % 36) / 6, k % 6, R2, o);
    o.ss = warp_total(o.ss);
    o.sp = warp_total(o.sp);
    o.ps = warp_total(o.ps);
    o.pp = warp_total(o.pp);
    o.pp0 = warp_total(o.pp0);
    __syncwarp();
    // entry sums: lanes 0-20 the evaluated local integrals, lanes 21-28 the
    // core sigma entries (ss, sz, xx, zz of side 0, then of side 1)
    double lcv = 0.0;
    if (lane < kLocalUnique) {
      const int t0 = tab.start[lane], t1 = t0 + tab.count[lane];
      double acc = 0.0;
      for (int t = t0; t < t1; ++t) acc += s.v[t];
      s.L[tab.row[lane] * 10 + tab.col[lane]] = acc;
    } else if (lane < kLocalUnique + 8) {
      const int q = lane - kLocalUnique, e = q & 3;
      const int lo = e == 0 ? 0 : (e == 1 ? c0 : (e == 2 ? c1 : c2));
      const int hi = e == 0 ? c0 : (e == 1 ? c1 : (e == 2 ? c2 : nc));
      const double* vs = s.v + nT + (q >> 2) * nc;
      for (int k = lo; k < hi; ++k) lcv += vs[k];
    }
    double lc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) lc[q] = __shfl_sync(0xffffffffu, lcv, kLocalUnique + q);
    __syncwarp();
    if (lane < 12) {
      s.L[kLocalCopies[lane][0]] = s.L[kLocalCopies[lane][1]];
    } else if (lane == 12) {
      s.L[44] = 0.5 * (s.L[22] - s.L[25]);
    }
    __syncwarp();
    // T = L W^T (in the term slots), then G = W T
    double* T = s.v;
    for (int k = lane; k < 100; k += 32) {
      const int r = k / 10, c = k % 10;
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < 10; ++q) t = fma(s.L[r * 10 + q], s.W[c * 10 + q], t);
      T[k] = t;
    }
    __syncwarp();
    double* out = ints + s.ioff[i];
    for (int k = lane; k < 100; k += 32) {
      const int r = k / 10, c = k % 10;
      double g = 0.0;
#pragma unroll
      for (int q = 0; q < 10; ++q) g = fma(s.W[r * 10 + q], T[q * 10 + c], g);
      out[k] = g;
    }
    const int p = s.pair[i];
    if (lane < 10) {
      vcore[(size_t)p * 20 + lane] = (-B.core) * sigma_entry(rot, lane, lc[0], lc[1], lc[2], lc[3]);
    } else if (lane < 20) {
      vcore[(size_t)p * 20 + lane] = (-A.core) * sigma_entry(rot, lane - 10, lc[4], -lc[5], lc[6], lc[7]);
    }
    if (lane < 16) ovl[(size_t)p * 16 + lane] = overlap_from_sums(o, Rv, lane >> 2, lane & 3);
    __syncwarp();
  }
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
    // shell pairs ss, and sp or ps when one atom has p functions
    const double Rv[3] = {X, Y, Z};
    const double R2v = X * X + Y * Y + Z * Z;
    OverlapSums o = {0.0, 0.0, 0.0, 0.0, 0.0}, mo = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int shell2 = nB == 4 ? 1 : (nA == 4 ? 2 : -1);
    for (int k = 0; k < 36; ++k) overlap_accumulate<true>(A, B, 0, k / 6, k % 6, R2v, o, &mo);
    if (shell2 > 0)
      for (int k = 0; k < 36; ++k) overlap_accumulate<true>(A, B, shell2, k / 6, k % 6, R2v, o, &mo);
    overlap_gradient(o, mo, f, Rv, g);
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

// Value and d/dR of one point-charge term (local_entry's summand).
__device__ __forceinline__ void term_value_grad(const LocalTerm& T, double R, const ElemDev& A, const ElemDev& B,
                                                bool coreB, double rhoCoreB, double& v, double& dv) {
  const double rA = A.rho[T.c1];
  const double rB = coreB ? rhoCoreB : B.rho[T.c2];
  const double D1 = A.D[T.c1];
  const double d2 = coreB ? 0.0 : B.D[T.c2];
  const double dx = d2 * T.x2 - D1 * T.x1;
  const double dy = d2 * T.y2 - D1 * T.y1;
  const double dz = R + d2 * T.z2 - D1 * T.z1;
  const double rr = rA + rB;
  const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + rr * rr);
  v = T.q * inv;
  dv = -dz * T.q * inv * inv * inv;
}

// Pair gradient, reverse mode, for pairs of two s/p atoms: a warp per group
// of 32 pairs.  First thread per pair: the core-repulsion derivative of the
// lane's pair, staged in shared memory.  Then pair by pair the warp shares
// the work with the 10 x 10 blocks in shared memory:
//   - the point-charge terms (value and d/dR) of the 21 evaluated local
//     integrals and of the two core-attraction sigma columns, one term per
//     lane (coalesced reads of g_local_terms), summed per entry;
//   - the 4 x 36 primitive products of the overlap block, one exponential
//     each, reduced over the warp into the sums of overlap_gradient;
//   - both frame rotations with their derivatives (lanes 30 and 31 in one
//     pass), the 100-entry matrices and products and the rotation adjoints;
// each lane's partial gradient is summed across the warp at the end.
constexpr int kGradWarps = 4;
constexpr int kGradGroup = 32;
struct HeavyGradShared {
  double dErep[kGradGroup];
  double v[kPairTermSlots], dv[kPairTermSlots];  // term values and derivatives, then T1 = F W, T2 = F^T W
  double L[100], dL[100], W[100], F[100];
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
  const int g0 = (blockIdx.x * kGradWarps + warp) * kGradGroup;
  if (g0 >= nhh) return;  // uniform per warp
  HeavyGradShared& s = shm[warp];
  const int ng = min(kGradGroup, nhh - g0);
  if (lane < ng) {
    const PairDev pr = pairs[hh[g0 + lane]];
    const AtomDev a = atoms[pr.a], b = atoms[pr.b];
    const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
    double E, dE;
    core_repulsion(method, elems[a.slot], elems[b.slot], diat[a.slot * kMaxElementSlots + b.slot],
                   sqrt(X * X + Y * Y + Z * Z), E, dE);
    s.dErep[lane] = dE;
  }
  const LocalTermTable& tab = g_local_terms;
  const int nT = tab.n_terms;
  const int c0 = tab.count[kColSS], c1 = c0 + tab.count[kColSZ], c2 = c1 + tab.count[kColXX];
  const int nc = c2 + tab.count[kColZZ];
  const int njobs = nT + 2 * nc;
  for (int i = 0; i < ng; ++i) {
    const int p = hh[g0 + i];
    const PairDev pr = pairs[p];
    const AtomDev a = atoms[pr.a], b = atoms[pr.b];
    const ElemDev& A = elems[a.slot];
    const ElemDev& B = elems[b.slot];
    const MolDev m = mols[pr.mol];
    const int N = m.nao;
    const double* P = Pall + m.mat_off;
    const double X = b.x - a.x, Y = b.y - a.y, Z = b.z - a.z;
    const double R = sqrt(X * X + Y * Y + Z * Z);
    __syncwarp();  // the previous pair's shared blocks are no longer read
    if (lane < 16) {
      const int r = lane >> 2, c = lane & 3;
      s.PA[r][c] = P[(size_t)(a.ao0 + r) * N + a.ao0 + c];
      s.PB[r][c] = P[(size_t)(b.ao0 + r) * N + b.ao0 + c];
      s.PAB[r][c] = P[(size_t)(a.ao0 + r) * N + b.ao0 + c];
      const size_t rc = m.mat_off + (size_t)(a.ao0 + r) * N + b.ao0 + c;
      s.SAB[r][c] = Paall ? Paall[rc] - Pball[rc] : 0.0;
    } else if (lane >= 30) {
      // lane 31: the reversed frame (vector B -> A), differentiated with respect to B - A
      const double sg = lane == 31 ? -1.0 : 1.0;
      rotation_grad(Dual3(sg * X, sg, 0, 0), Dual3(sg * Y, 0, sg, 0), Dual3(sg * Z, 0, 0, sg),
                    lane == 31 ? s.rb : s.ra);
    }
    for (int k = lane; k < 100; k += 32) s.L[k] = s.dL[k] = 0.0;
    if (lane < 10) s.Lc[lane] = s.dLc[lane] = s.Lcb[lane] = s.dLcb[lane] = 0.0;
    for (int j = lane; j < njobs; j += 32) {
      double v, dv;
      if (j < nT) {
        term_value_grad(tab.term[j], R, A, B, false, 0.0, v, dv);
      } else {
        const int side = j - nT >= nc, k = j - nT - side * nc;
        const int t = k < c0   ? tab.start[kColSS] + k
                      : k < c1 ? tab.start[kColSZ] + (k - c0)
                      : k < c2 ? tab.start[kColXX] + (k - c1)
                               : tab.start[kColZZ] + (k - c2);
        if (side) term_value_grad(tab.term[t], R, B, A, true, A.pcore, v, dv);
        else term_value_grad(tab.term[t], R, A, B, true, B.pcore, v, dv);
      }
      s.v[j] = v;
      s.dv[j] = dv;
    }
    OverlapSums o = {0.0, 0.0, 0.0, 0.0, 0.0}, mo = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double R2 = X * X + Y * Y + Z * Z;
    for (int k = lane; k < 144; k += 32) overlap_accumulate<true>(A, B, k / 36, (k % 36) / 6, k % 6, R2, o, &mo);
    o.ss = warp_total(o.ss);
    o.sp = warp_total(o.sp);
    o.ps = warp_total(o.ps);
    o.pp = warp_total(o.pp);
    o.pp0 = warp_total(o.pp0);
    mo.ss = warp_total(mo.ss);
    mo.sp = warp_total(mo.sp);
    mo.ps = warp_total(mo.ps);
    mo.pp = warp_total(mo.pp);
    mo.pp0 = warp_total(mo.pp0);
    __syncwarp();
    // entry sums: lanes 0-20 the evaluated local integrals, lanes 21-28 the
    // core sigma entries (ss, sz, xx, zz of A against B's core, then of B
    // against A's), stored by orbital-pair index
    if (lane < kLocalUnique) {
      const int t0 = tab.start[lane], t1 = t0 + tab.count[lane];
      double acc = 0.0, dacc = 0.0;
      for (int t = t0; t < t1; ++t) {
        acc += s.v[t];
        dacc += s.dv[t];
      }
      s.L[tab.row[lane] * 10 + tab.col[lane]] = acc;
      s.dL[tab.row[lane] * 10 + tab.col[lane]] = dacc;
    } else if (lane < kLocalUnique + 8) {
      const int q = lane - kLocalUnique, e = q & 3, side = q >> 2;
      const int lo = e == 0 ? 0 : (e == 1 ? c0 : (e == 2 ? c1 : c2));
      const int hi = e == 0 ? c0 : (e == 1 ? c1 : (e == 2 ? c2 : nc));
      const int idx = tab.row[e == 0 ? kColSS : (e == 1 ? kColSZ : (e == 2 ? kColXX : kColZZ))];
      const double* vs = s.v + nT + side * nc;
      const double* dvs = s.dv + nT + side * nc;
      double acc = 0.0, dacc = 0.0;
      for (int k = lo; k < hi; ++k) {
        acc += vs[k];
        dacc += dvs[k];
      }
      (side ? s.Lcb : s.Lc)[idx] = acc;
      (side ? s.dLcb : s.dLc)[idx] = dacc;
    }
    __syncwarp();
    // symmetry copies, all from evaluated entries; density factors and W
    if (lane < 12) {
      s.L[kLocalCopies[lane][0]] = s.L[kLocalCopies[lane][1]];
      s.dL[kLocalCopies[lane][0]] = s.dL[kLocalCopies[lane][1]];
    } else if (lane == 12) {
      s.L[44] = 0.5 * (s.L[22] - s.L[25]);
      s.dL[44] = 0.5 * (s.dL[22] - s.dL[25]);
    } else if (lane == 13) {
      s.Lc[5] = s.Lc[2];
      s.dLc[5] = s.dLc[2];
    } else if (lane == 14) {
      s.Lcb[5] = s.Lcb[2];
      s.dLcb[5] = s.dLcb[2];
    }
    for (int k = lane; k < 100; k += 32) {
      s.W[k] = w_entry(s.ra.r, k / 10, k % 10);
      s.F[k] = Paall ? density_factor_uhf(s.PA, s.PB, s.PAB, s.SAB, k / 10, k % 10)
                     : density_factor(s.PA, s.PB, s.PAB, k / 10, k % 10);
    }
    __syncwarp();
    // T1 = F W, T2 = F^T W (in the term slots)
    double* T1 = s.v;
    double* T2 = s.dv;
    for (int k = lane; k < 100; k += 32) {
      const int r = k / 10, c = k % 10;
      double t1 = 0, t2 = 0;
      for (int l = 0; l < 10; ++l) {
        t1 += s.F[r * 10 + l] * s.W[l * 10 + c];
        t2 += s.F[l * 10 + r] * s.W[l * 10 + c];
      }
      T1[k] = t1;
      T2[k] = t2;
    }
    __syncwarp();
    double adjA[4][4] = {}, adjB[4][4] = {};
    double dR = 0, g[3] = {0, 0, 0};
    // two-centre: dE/dW[p][q] = sum_j T1[p][j] L[q][j] + sum_a T2[p][a] L[a][q];
    // dE/dL[x][y] = sum_g W[g][x] T1[g][y]
    for (int k = lane; k < 100; k += 32) {
      const int pp = k / 10, qq = k % 10;
      double adw = 0;
      for (int j = 0; j < 10; ++j) adw += T1[pp * 10 + j] * s.L[qq * 10 + j] + T2[pp * 10 + j] * s.L[j * 10 + qq];
      if (adw != 0.0) w_adjoint(s.ra.r, pp, qq, adw, adjA);
      if (s.dL[k] != 0.0) {
        double mm = 0;
        for (int g2 = 0; g2 < 10; ++g2) mm += s.W[g2 * 10 + pp] * T1[g2 * 10 + qq];
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
    if (lane == 0) {
      // overlap (resonance integrals) from the reduced sums, core repulsion
      double f[4][4];
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
          f[r][c] = ((r == 0 ? A.betaS : A.betaP) + (c == 0 ? B.betaS : B.betaP)) * s.PAB[r][c];
      const double Rv[3] = {X, Y, Z};
      overlap_gradient(o, mo, f, Rv, g);
      dR += s.dErep[i];
    }
    g[0] += dR * X / R;
    g[1] += dR * Y / R;
    g[2] += dR * Z / R;
    add_rotation_gradient(s.ra, adjA, g);
    add_rotation_gradient(s.rb, adjB, g);
    for (int k = 0; k < 3; ++k) g[k] = warp_total(g[k]);
    if (lane == 0) {
      gpair[(size_t)p * 3 + 0] = g[0];
      gpair[(size_t)p * 3 + 1] = g[1];
      gpair[(size_t)p * 3 + 2] = g[2];
    }
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
    k_pair_values_heavy<<<(b.nhh_total + kValWarps * kValGroup - 1) / (kValWarps * kValGroup), kValWarps * 32, 0, s>>>(
        b.hh_pairs, b.nhh_total, b.pairs, b.atoms, b.elems, b.diat, b.method, b.ints, b.vcore, b.ovl, b.erep);
}

void launch_gradient(const DeviceBatch& b, cudaStream_t s) {
  if (b.npairs > 0) {
    const int th = 128;
    k_pair_gradient_light<<<(b.npairs + th - 1) / th, th, 0, s>>>(b.pairs, b.npairs, b.atoms, b.elems, b.diat, b.mols,
                                                                   b.method, b.P, b.uhf ? b.Pa : nullptr,
                                                                   b.uhf ? b.Pb : nullptr, b.gpair);
  }
  if (b.nhh_total > 0) {
    k_pair_gradient_heavy<<<(b.nhh_total + kGradWarps * kGradGroup - 1) / (kGradWarps * kGradGroup), kGradWarps * 32,
                            0, s>>>(
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
