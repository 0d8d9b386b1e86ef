// One-electron assembly and the persistent batched SCF kernel.
//
// The SCF kernel runs one CTA per molecule: CTAs take molecules from a work
// counter (largest first) and iterate each to self-consistency on the device
// with no host round trips.  Per iteration (restricted, orthonormal NDDO
// basis):
//   F = H + G(P), E_el = 1/2 sum P (H + F)        TwoElectronMatrix.cpp:63-166,
//                                                 NDDOElectronicEnergyCalculator.cpp:48-67
//   Pulay DIIS on the commutator FP - PF          (restated; the reference's
//                                                 SCF driver is in scine_utilities)
//   F_mo = C^T F C, cyclic parallel Jacobi, C <- C J (warm start from the
//   previous orbitals), aufbau occupation of the n_occ lowest orbitals
//   P = 2 C_occ C_occ^T, convergence on |dE| and rms(dP)
// and, after convergence, G is rebuilt from the final density
// (FockMatrix::finalize, FockMatrix.cpp:147-150).
#include <cuda_runtime.h>

#include <cstdio>

#include "kernels.h"
#include "nddo_math.cuh"

namespace sgb {

constexpr int kScfThreads = 256;
constexpr int kJacobiMaxPairs = 512;  // supports N <= 1024
constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16;

// ---------------------------------------------------------------------------
// CTA helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum; every thread gets the result.
__device__ double cta_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  return s;
}
__device__ double cta_max(double v, double* red) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s = fmax(s, red[i]);
  return s;
}

// C = alpha * op(A) * op(B) + beta * C, row-major, op(X) = X or X^T.
// 64x64 output tiles, 256 threads with a 4x4 register tile each.
__device__ void cta_gemm(int M, int Nn, int K, double alpha, const double* __restrict__ A, int lda, bool tA,
                         const double* __restrict__ B, int ldb, bool tB, double beta, double* C, int ldc,
                         double* smA, double* smB) {
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  for (int m0 = 0; m0 < M; m0 += kGemmBM)
    for (int n0 = 0; n0 < Nn; n0 += kGemmBN) {
      double acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0;
      for (int k0 = 0; k0 < K; k0 += kGemmBK) {
        // stage op(A)[m0:m0+64, k0:k0+16] as smA[k][m]
        for (int e = tid; e < kGemmBM * kGemmBK; e += kScfThreads) {
          int mm, kk;
          if (!tA) { mm = e / kGemmBK; kk = e % kGemmBK; }
          else { kk = e / kGemmBM; mm = e % kGemmBM; }
          int gm = m0 + mm, gk = k0 + kk;
          double v = 0;
          if (gm < M && gk < K) v = tA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
          smA[kk * (kGemmBM + 1) + mm] = v;
        }
        // stage op(B)[k0:k0+16, n0:n0+64] as smB[k][n]
        for (int e = tid; e < kGemmBK * kGemmBN; e += kScfThreads) {
          int nn, kk;
          if (!tB) { kk = e / kGemmBN; nn = e % kGemmBN; }
          else { nn = e / kGemmBK; kk = e % kGemmBK; }
          int gn = n0 + nn, gk = k0 + kk;
          double v = 0;
          if (gn < Nn && gk < K) v = tB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
          smB[kk * (kGemmBN + 1) + nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGemmBK; ++kk) {
          double a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = smA[kk * (kGemmBM + 1) + ty * 4 + i];
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = smB[kk * (kGemmBN + 1) + tx * 4 + j];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          int gm = m0 + ty * 4 + i, gn = n0 + tx * 4 + j;
          if (gm < M && gn < Nn) {
            double* c = &C[(size_t)gm * ldc + gn];
            *c = beta == 0.0 ? alpha * acc[i][j] : alpha * acc[i][j] + beta * (*c);
          }
        }
    }
  __syncthreads();
}

__device__ __forceinline__ long long pair_slot(const MolDev& m, int lo, int hi) {
  return (long long)m.pair0 + (long long)lo * m.nat - (long long)lo * (lo + 1) / 2 + (hi - lo - 1);
}

// ---------------------------------------------------------------------------
// One-electron matrix, start density and repulsion energy (one CTA per molecule)
// ---------------------------------------------------------------------------
// H (OneElectronMatrix.cpp:43-134, both triangles):
//   same atom:  U on the diagonal + sum over other atoms B of V^B[p(mu,nu)]
//   two atoms:  1/2 (beta_mu + beta_nu) S_mu,nu
// start density (NDDODensityGuess.cpp:31-66): S * n_el / (2N) between atoms,
// zero within an atom off the diagonal, core charge / n_AO on the diagonal.
__global__ void __launch_bounds__(kScfThreads) k_one_electron(const MolDev* __restrict__ mols,
                                                              const AtomDev* __restrict__ atoms,
                                                              const ElemDev* __restrict__ elems,
                                                              const PairDev* __restrict__ pairs,
                                                              const int* __restrict__ ao_atom,
                                                              const double* __restrict__ vcore,
                                                              const double* __restrict__ ovl,
                                                              const double* __restrict__ erep, double* Hall,
                                                              double* Pall, MolResult* res, int write_guess) {
  __shared__ double red[32];
  const MolDev m = mols[blockIdx.x];
  const int N = m.nao;
  double* H = Hall + m.mat_off;
  double* P = Pall + m.mat_off;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx / N, j = idx % N;
    const int A = ao_atom[m.ao_base + i], B = ao_atom[m.ao_base + j];
    const AtomDev aA = atoms[A], aB = atoms[B];
    const ElemDev& eA = elems[aA.slot];
    const int mu = i - aA.ao0, nu = j - aB.ao0;
    double h, p;
    if (A == B) {
      h = (mu == nu) ? (mu == 0 ? eA.Uss : eA.Upp) : 0.0;
      const int a = A - m.atom0;
      const int pk = pair_index(mu, nu);
      for (int c = 0; c < m.nat; ++c) {
        if (c == a) continue;
        long long s = a < c ? pair_slot(m, a, c) : pair_slot(m, c, a);
        h += vcore[s * 20 + (a < c ? 0 : 10) + pk];
      }
      p = (mu == nu) ? eA.core / eA.nao : 0.0;
    } else {
      const ElemDev& eB = elems[aB.slot];
      const int a = A - m.atom0, b = B - m.atom0;
      double s = a < b ? ovl[pair_slot(m, a, b) * 16 + mu * 4 + nu] : ovl[pair_slot(m, b, a) * 16 + nu * 4 + mu];
      double ba = mu == 0 ? eA.betaS : eA.betaP, bb = nu == 0 ? eB.betaS : eB.betaP;
      h = 0.5 * (ba + bb) * s;
      p = s * m.nel / (2.0 * N);
    }
    H[idx] = h;
    if (write_guess) P[idx] = p;
  }
  double e = 0;
  for (int k = threadIdx.x; k < m.npairs; k += blockDim.x) e += erep[m.pair0 + k];
  e = cta_sum(e, red);
  if (threadIdx.x == 0) res[blockIdx.x].e_rep = e;
}

void launch_one_electron(const DeviceBatch& b, cudaStream_t s) {
  if (b.nmol == 0) return;
  k_one_electron<<<b.nmol, kScfThreads, 0, s>>>(b.mols, b.atoms, b.elems, b.pairs, b.ao_atom, b.vcore, b.ovl,
                                                b.erep, b.H, b.P, b.res, b.use_guess);
}

// ---------------------------------------------------------------------------
// Fock matrix F = H + G(P) and the electronic energy 1/2 sum P (H + F)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double one_centre_g(const ElemDev& e, int mu, int nu, const double* P, int N, int o) {
  auto Pm = [&](int i, int j) { return P[(o + i) * N + o + j]; };
  if (e.nao == 1) return 0.5 * Pm(0, 0) * e.gss;
  if (mu == nu) {
    if (mu == 0) return 0.5 * Pm(0, 0) * e.gss + (Pm(1, 1) + Pm(2, 2) + Pm(3, 3)) * (e.gsp - 0.5 * e.hsp);
    double g = Pm(0, 0) * (e.gsp - 0.5 * e.hsp) + 0.5 * Pm(mu, mu) * e.gpp;
    for (int q = 1; q < 4; ++q)
      if (q != mu) g += Pm(q, q) * (e.gp2 - 0.5 * e.hpp);
    return g;
  }
  if (mu == 0 || nu == 0) return Pm(mu, nu) * (1.5 * e.hsp - 0.5 * e.gsp);
  return Pm(mu, nu) * (1.5 * e.hpp - 0.5 * e.gp2);
}

__device__ double build_fock(const MolDev& m, const AtomDev* __restrict__ atoms, const ElemDev* __restrict__ elems,
                             const PairDev* __restrict__ pairs, const double* __restrict__ ints,
                             const int* __restrict__ ao_atom, const double* __restrict__ H,
                             const double* __restrict__ P, double* F, double* red) {
  const int N = m.nao;
  double e = 0;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int i = idx / N, j = idx % N;
    const int A = ao_atom[m.ao_base + i], B = ao_atom[m.ao_base + j];
    const AtomDev aA = atoms[A], aB = atoms[B];
    const ElemDev& eA = elems[aA.slot];
    const int mu = i - aA.ao0, nu = j - aB.ao0;
    const double h = H[idx];
    double g;
    if (A == B) {
      g = one_centre_g(eA, mu, nu, P, N, aA.ao0);
      const int a = A - m.atom0, pk = pair_index(mu, nu), dA = eA.nao == 1 ? 1 : 10;
      for (int c = 0; c < m.nat; ++c) {
        if (c == a) continue;
        const AtomDev aC = atoms[m.atom0 + c];
        const int nC = elems[aC.slot].nao, dC = nC == 1 ? 1 : 10, oc = aC.ao0;
        const bool first = a < c;
        const double* W = ints + pairs[first ? pair_slot(m, a, c) : pair_slot(m, c, a)].int_off;
        for (int la = 0; la < nC; ++la)
          for (int si = la; si < nC; ++si) {
            const int pl = pair_index(la, si);
            const double w = first ? W[pk * dC + pl] : W[pl * dA + pk];
            g += (la == si ? 1.0 : 2.0) * P[(oc + la) * N + oc + si] * w;
          }
      }
    } else {
      const int nA = eA.nao, nB = elems[aB.slot].nao;
      const int dA = nA == 1 ? 1 : 10, dB = nB == 1 ? 1 : 10;
      const int a = A - m.atom0, b = B - m.atom0;
      const bool first = a < b;
      const double* W = ints + pairs[first ? pair_slot(m, a, b) : pair_slot(m, b, a)].int_off;
      double k = 0;
      for (int n2 = 0; n2 < nA; ++n2)
        for (int s2 = 0; s2 < nB; ++s2) {
          const int p1 = pair_index(mu, n2), p2 = pair_index(nu, s2);
          const double w = first ? W[p1 * dB + p2] : W[p2 * dA + p1];
          k += P[(aA.ao0 + n2) * N + aB.ao0 + s2] * w;
        }
      g = -0.5 * k;
    }
    const double f = h + g;
    F[idx] = f;
    e += 0.5 * P[idx] * (h + f);
  }
  __syncthreads();
  return cta_sum(e, red);
}

// ---------------------------------------------------------------------------
// Cyclic Jacobi on the symmetric A (N x N) with rotations applied to C's columns
// ---------------------------------------------------------------------------
struct JacobiShared {
  double c[kJacobiMaxPairs], s[kJacobiMaxPairs], t[kJacobiMaxPairs];
  int p[kJacobiMaxPairs], q[kJacobiMaxPairs];
};

// Returns the number of sweeps, or -1 if not converged within max_sweeps.
__device__ int jacobi_eigh(int N, double* A, double* C, JacobiShared& js, double* red, int max_sweeps, double tol) {
  const int Ne = N + (N & 1);
  const int npair = Ne / 2;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double offmax = 0;
    for (int r = 0; r < Ne - 1; ++r) {
      for (int k = threadIdx.x; k < npair; k += blockDim.x) {
        int p, q;
        if (k == 0) { p = Ne - 1; q = r; }
        else { p = (r + k) % (Ne - 1); q = (r - k + Ne - 1) % (Ne - 1); }
        if (p > q) { int t = p; p = q; q = t; }
        double c = 1, s = 0, t = 0;
        if (q < N) {
          const double apq = A[(size_t)p * N + q];
          offmax = fmax(offmax, fabs(apq));
          if (apq != 0.0) {
            const double app = A[(size_t)p * N + p], aqq = A[(size_t)q * N + q];
            const double tau = (aqq - app) / (2.0 * apq);
            t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        js.p[k] = p;
        js.q[k] = q < N ? q : -1;
        js.c[k] = c;
        js.s[k] = s;
        js.t[k] = t;
      }
      __syncthreads();
      // A <- J^T A J on 2x2 blocks of pair k1 (rows) and pair k2 (columns), k1 <= k2
      const int nblk = npair * (npair + 1) / 2;
      for (int bidx = threadIdx.x; bidx < nblk; bidx += blockDim.x) {
        // map triangular index to (k1, k2)
        int k1 = (int)((sqrt(8.0 * bidx + 1.0) - 1.0) * 0.5);
        while ((k1 + 1) * (k1 + 2) / 2 <= bidx) ++k1;
        while (k1 * (k1 + 1) / 2 > bidx) --k1;
        const int k2 = bidx - k1 * (k1 + 1) / 2;  // k2 <= k1
        const int p1 = js.p[k1], q1 = js.q[k1], p2 = js.p[k2], q2 = js.q[k2];
        if (q1 < 0 && q2 < 0) {
          continue;  // both pairs carry the padding index: only the (p, p) entry, untouched
        }
        const double c1 = js.c[k1], s1 = js.s[k1], c2 = js.c[k2], s2 = js.s[k2];
        if (k1 == k2) {
          if (q1 < 0) continue;
          const double t = js.t[k1];
          const double apq = A[(size_t)p1 * N + q1];
          A[(size_t)p1 * N + p1] -= t * apq;
          A[(size_t)q1 * N + q1] += t * apq;
          A[(size_t)p1 * N + q1] = 0.0;
          A[(size_t)q1 * N + p1] = 0.0;
          continue;
        }
        // rows {p1, q1}, cols {p2, q2}; a padding index has no row/column
        const double m00 = A[(size_t)p1 * N + p2];
        const double m01 = q2 >= 0 ? A[(size_t)p1 * N + q2] : 0.0;
        const double m10 = q1 >= 0 ? A[(size_t)q1 * N + p2] : 0.0;
        const double m11 = (q1 >= 0 && q2 >= 0) ? A[(size_t)q1 * N + q2] : 0.0;
        const double x00 = c1 * m00 - s1 * m10, x01 = c1 * m01 - s1 * m11;
        const double x10 = s1 * m00 + c1 * m10, x11 = s1 * m01 + c1 * m11;
        const double n00 = x00 * c2 - x01 * s2, n01 = x00 * s2 + x01 * c2;
        const double n10 = x10 * c2 - x11 * s2, n11 = x10 * s2 + x11 * c2;
        A[(size_t)p1 * N + p2] = n00;
        A[(size_t)p2 * N + p1] = n00;
        if (q2 >= 0) { A[(size_t)p1 * N + q2] = n01; A[(size_t)q2 * N + p1] = n01; }
        if (q1 >= 0) { A[(size_t)q1 * N + p2] = n10; A[(size_t)p2 * N + q1] = n10; }
        if (q1 >= 0 && q2 >= 0) { A[(size_t)q1 * N + q2] = n11; A[(size_t)q2 * N + q1] = n11; }
      }
      // C <- C J
      for (int e = threadIdx.x; e < N * npair; e += blockDim.x) {
        const int row = e / npair, k = e % npair;
        const int q = js.q[k];
        if (q < 0) continue;
        const int p = js.p[k];
        const double c = js.c[k], s = js.s[k];
        const double cp = C[(size_t)row * N + p], cq = C[(size_t)row * N + q];
        C[(size_t)row * N + p] = c * cp - s * cq;
        C[(size_t)row * N + q] = s * cp + c * cq;
      }
      __syncthreads();
    }
    offmax = cta_max(offmax, red);
    if (offmax < tol) return sweep + 1;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// Persistent SCF kernel
// ---------------------------------------------------------------------------
struct ScfShared {
  double red[32];
  double bmat[kDiisMax * kDiisMax];
  double sys[(kDiisMax + 1) * (kDiisMax + 2)];
  double coef[kDiisMax + 1];
  double gemmA[kGemmBK * (kGemmBM + 1)];
  double gemmB[kGemmBK * (kGemmBN + 1)];
  JacobiShared js;
  int mol;
  int diis_ok;
};

__global__ void __launch_bounds__(kScfThreads) k_scf(const MolDev* __restrict__ mols, int nmol,
                                                     const int* __restrict__ order, int* counter,
                                                     const AtomDev* __restrict__ atoms,
                                                     const ElemDev* __restrict__ elems,
                                                     const PairDev* __restrict__ pairs,
                                                     const double* __restrict__ ints,
                                                     const int* __restrict__ ao_atom, const double* __restrict__ Hall,
                                                     double* Pall, double* Fall, double* Call, double* W1all,
                                                     double* W2all, double* epsall, double* diisall, MolResult* res,
                                                     ScfParams sp) {
  extern __shared__ unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) {
      int k = atomicAdd(counter, 1);
      sh.mol = k < nmol ? order[k] : -1;
    }
    __syncthreads();
    const int mi = sh.mol;
    __syncthreads();
    if (mi < 0) return;
    const MolDev m = mols[mi];
    const int N = m.nao;
    const size_t NN = (size_t)N * N;
    const double* H = Hall + m.mat_off;
    double* P = Pall + m.mat_off;
    double* F = Fall + m.mat_off;
    double* C = Call + m.mat_off;
    double* W1 = W1all + m.mat_off;
    double* W2 = W2all + m.mat_off;
    double* eps = epsall + m.ao_base;
    double* histF = diisall + m.diis_off;
    double* histE = histF + (size_t)kDiisMax * NN;
    const int msize = sp.diis_size < 1 ? 1 : (sp.diis_size > kDiisMax ? kDiisMax : sp.diis_size);
    int nhist = 0, head = 0;  // ring buffer of DIIS vectors
    bool have_orbitals = false;
    double Eold = 0;
    int it = 0, converged = 0, status = kDevOk;
    double last_dE = 0, last_rms = 0;

    for (it = 1; it <= sp.max_iter; ++it) {
      // F = H + G(P), energy of the current density
      const double E = build_fock(m, atoms, elems, pairs, ints, ao_atom, H, P, F, sh.red);
      __syncthreads();
      // DIIS error e = FP - PF (F, P symmetric: PF = (FP)^T)
      cta_gemm(N, N, N, 1.0, F, N, false, P, N, false, 0.0, W1, N, sh.gemmA, sh.gemmB);
      const int slot = head;
      double* eS = histE + (size_t)slot * NN;
      double* fS = histF + (size_t)slot * NN;
      for (size_t k = tid; k < NN; k += blockDim.x) {
        const int i = (int)(k / N), j = (int)(k % N);
        eS[k] = W1[k] - W1[(size_t)j * N + i];
        fS[k] = F[k];
      }
      __syncthreads();
      head = (head + 1) % msize;
      if (nhist < msize) ++nhist;
      // new row of the B matrix
      for (int j = 0; j < nhist; ++j) {
        const double* eJ = histE + (size_t)j * NN;
        double d = 0;
        for (size_t k = tid; k < NN; k += blockDim.x) d += eS[k] * eJ[k];
        d = cta_sum(d, sh.red);
        if (tid == 0) {
          sh.bmat[slot * kDiisMax + j] = d;
          sh.bmat[j * kDiisMax + slot] = d;
        }
      }
      __syncthreads();
      const double* Fx = F;
      if (nhist >= 2) {
        if (tid == 0) {
          // (n+1) x (n+1) Pulay system, scaled by the largest diagonal entry
          const int n = nhist, ld = n + 2;
          double scale = 0;
          for (int i = 0; i < n; ++i) scale = fmax(scale, fabs(sh.bmat[i * kDiisMax + i]));
          scale = scale > 0 ? 1.0 / scale : 1.0;
          for (int i = 0; i <= n; ++i)
            for (int j = 0; j <= n; ++j) {
              double v;
              if (i < n && j < n) v = sh.bmat[i * kDiisMax + j] * scale;
              else if (i == n && j == n) v = 0;
              else v = -1;
              sh.sys[i * ld + j] = v;
            }
          for (int i = 0; i <= n; ++i) sh.sys[i * ld + n + 1] = (i == n) ? -1.0 : 0.0;
          int ok = 1;
          for (int c = 0; c <= n && ok; ++c) {
            int piv = c;
            for (int r = c + 1; r <= n; ++r)
              if (fabs(sh.sys[r * ld + c]) > fabs(sh.sys[piv * ld + c])) piv = r;
            if (fabs(sh.sys[piv * ld + c]) < 1e-300) { ok = 0; break; }
            if (piv != c)
              for (int k = 0; k <= n + 1; ++k) {
                double t = sh.sys[c * ld + k];
                sh.sys[c * ld + k] = sh.sys[piv * ld + k];
                sh.sys[piv * ld + k] = t;
              }
            for (int r = c + 1; r <= n; ++r) {
              double f = sh.sys[r * ld + c] / sh.sys[c * ld + c];
              for (int k = c; k <= n + 1; ++k) sh.sys[r * ld + k] -= f * sh.sys[c * ld + k];
            }
          }
          if (ok) {
            for (int c = n; c >= 0; --c) {
              double s = sh.sys[c * ld + n + 1];
              for (int k = c + 1; k <= n; ++k) s -= sh.sys[c * ld + k] * sh.coef[k];
              sh.coef[c] = s / sh.sys[c * ld + c];
            }
            for (int i = 0; i < n; ++i)
              if (!isfinite(sh.coef[i])) ok = 0;
          }
          sh.diis_ok = ok;
        }
        __syncthreads();
        if (sh.diis_ok) {
          for (size_t k = tid; k < NN; k += blockDim.x) {
            double s = 0;
            for (int i = 0; i < nhist; ++i) s += sh.coef[i] * histF[(size_t)i * NN + k];
            W1[k] = s;
          }
          Fx = W1;
        }
        __syncthreads();
      }
      // eigen-decomposition of Fx, warm-started from the previous orbitals
      if (!have_orbitals) {
        for (size_t k = tid; k < NN; k += blockDim.x) {
          const int i = (int)(k / N), j = (int)(k % N);
          C[k] = (i == j) ? 1.0 : 0.0;
          W2[k] = Fx[k];
        }
        __syncthreads();
      } else {
        // W2 = C^T Fx C  (Fx may live in W1; use F as the temporary)
        cta_gemm(N, N, N, 1.0, Fx, N, false, C, N, false, 0.0, Fx == F ? W1 : F, N, sh.gemmA, sh.gemmB);
        cta_gemm(N, N, N, 1.0, C, N, true, Fx == F ? W1 : F, N, false, 0.0, W2, N, sh.gemmA, sh.gemmB);
        // symmetrise against rounding
        for (size_t k = tid; k < NN; k += blockDim.x) {
          const int i = (int)(k / N), j = (int)(k % N);
          if (i < j) {
            double v = 0.5 * (W2[k] + W2[(size_t)j * N + i]);
            W2[k] = v;
            W2[(size_t)j * N + i] = v;
          }
        }
        __syncthreads();
      }
      const int sweeps = jacobi_eigh(N, W2, C, sh.js, sh.red, sp.jacobi_max_sweeps, 1e-12);
      if (sweeps < 0) status = kDevJacobiNotConverged;
      have_orbitals = true;
      // sort orbitals by energy: rank of each diagonal entry
      for (int k = tid; k < N; k += blockDim.x) {
        const double ek = W2[(size_t)k * N + k];
        int rank = 0;
        for (int j = 0; j < N; ++j) {
          const double ej = W2[(size_t)j * N + j];
          rank += (ej < ek || (ej == ek && j < k)) ? 1 : 0;
        }
        eps[rank] = ek;
        for (int row = 0; row < N; ++row) W1[(size_t)row * N + rank] = C[(size_t)row * N + k];
      }
      __syncthreads();
      for (size_t k = tid; k < NN; k += blockDim.x) C[k] = W1[k];
      __syncthreads();
      // new density P = 2 C_occ C_occ^T into W1, rms change against P
      cta_gemm(N, N, m.nocc, 2.0, C, N, false, C, N, true, 0.0, W1, N, sh.gemmA, sh.gemmB);
      double d2 = 0;
      for (size_t k = tid; k < NN; k += blockDim.x) {
        const double d = W1[k] - P[k];
        d2 += d * d;
        P[k] = W1[k];
      }
      d2 = cta_sum(d2, sh.red);
      const double rms = sqrt(d2 / (double)NN);
      last_rms = rms;
      last_dE = it > 1 ? fabs(E - Eold) : 0.0;
      const bool dE_ok = it > 1 && fabs(E - Eold) < sp.scc;
      Eold = E;
      if (!isfinite(E) || !isfinite(rms)) { status = kDevNonFinite; break; }
      if (dE_ok && rms < sp.rmsd) { converged = 1; break; }
      __syncthreads();
    }
    if (it > sp.max_iter) it = sp.max_iter;
    __syncthreads();
    // finalize: Fock matrix and energy consistent with the final density
    const double Efin = build_fock(m, atoms, elems, pairs, ints, ao_atom, H, P, F, sh.red);
    if (tid == 0) {
      MolResult& r = res[mi];
      r.e_el = Efin;
      r.energy = Efin + r.e_rep;
      r.iterations = it;
      r.converged = converged;
      r.status = status;
      r.last_dE = last_dE;
      r.last_rmsd = last_rms;
    }
    __syncthreads();
  }
}

int scf_max_grid(int) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(k_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ScfShared));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scf, kScfThreads, sizeof(ScfShared));
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

void launch_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  cudaFuncSetAttribute(k_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ScfShared));
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  k_scf<<<grid, kScfThreads, sizeof(ScfShared), s>>>(b.mols, b.nmol, b.order, b.counter, b.atoms, b.elems, b.pairs,
                                                     b.ints, b.ao_atom, b.H, b.P, b.F, b.C, b.W1, b.W2, b.eps,
                                                     b.diis, b.res, sp);
}

}  // namespace sgb
