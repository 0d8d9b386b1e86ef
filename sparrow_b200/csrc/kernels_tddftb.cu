// Linear-response TD-DFTB on a converged restricted DFTB2/DFTB3 reference:
// batched over molecules, one persistent 512-thread CTA per molecule.
//
// Reference behaviour followed (paths relative to
// src/Sparrow/Sparrow/Implementations/Dftb/):
//   transition charges  Utils/DipoleUtils/TransitionChargesCalculator.h:138-165
//                       q_A^{ia} = 1/2 sum_{mu on A} (C_mu,i (SC)_mu,a + C_mu,a (SC)_mu,i)
//   sigma vectors       TimeDependent/LinearResponse/TDDFTBSigmaVectorEvaluator.cpp:40-110
//                       (Omega t)_ia = Delta_ia^2 t_ia + 4 h_ia . G (h^T t), h = q sqrt(Delta),
//                       G = gamma (singlets) or diag(W_A) (triplets), factor 4 for a
//                       restricted reference (TDDFTBSigmaVectorEvaluator.h:118-120)
//   excited states      TimeDependent/LinearResponse/TDDFTBEigenvalueSolver.h:150-197
//                       omega = sqrt(eigenvalue), c_ia = sqrt(Delta_ia / omega) F_ia
//   dipole matrix       Utils/DipoleUtils/DFTBDipoleMatrixCalculator.cpp:60-84
//                       D_ia = sum_A q_A^{ia} R_A; mu_I = sqrt(2) sum_ia c_ia D_ia
// Per molecule:
//   1. canonical orbitals: F' = X F X of the converged Fock matrix, Jacobi
//      diagonalisations of its occupied and virtual blocks in the basis of the
//      SCF's last orbitals (the rotation-based SCF keeps them only close to
//      canonical; the occupied-virtual block vanishes at convergence), C = X C'.
//   2. SC, the transition charges and dipole vectors of every occupied-virtual
//      pair, h = q sqrt(Delta).
//   3. block Davidson for the lowest n_roots eigenpairs of the symmetric
//      Casida matrix Omega (never formed): sigma vectors through the atoms
//      (n_atoms x n_transitions work per vector), Rayleigh matrix and a dense
//      Jacobi eigensolver in shared memory, residuals preconditioned by
//      1 / (theta - Delta^2), two-pass Gram-Schmidt, restart to the n_roots
//      Ritz vectors when the subspace is full.  The reference's Davidson lives
//      in the un-vendored scine_utilities; converged eigenpairs do not depend
//      on the solver.
//   4. omega, transition dipoles.
// The transitions are indexed k = i * n_virt + a.
#include <cuda_runtime.h>

#include "dftb_math.cuh"
#include "kernels.h"
#include "scf_core.cuh"

namespace sgb {

namespace {

constexpr int kTdMaxRoots = 16;
constexpr int kTdMaxSub = 64;  // Davidson subspace limit

// Shared-memory part of the Davidson state (after the ScfShared block).
struct TdShared {
  double H[kTdMaxSub * kTdMaxSub];   // Rayleigh matrix V^T Omega V
  double Z[kTdMaxSub * kTdMaxSub];   // eigenvectors of H (columns), sorted
  double Wk[kTdMaxSub * kTdMaxSub];  // Jacobi work copy
  double theta[kTdMaxSub];
  double cs[kTdMaxSub];              // rotation (c, s) per pair
  double rnorm[kTdMaxRoots];
  double coef[kTdMaxSub];
  int pq[kTdMaxSub];
  int sel[2 * kTdMaxRoots];
  double rv[32];
  int ri[32];
  int flag;
};

// Index of the smallest v over the CTA (ties: lowest index); every thread gets it.
__device__ int cta_argmin(double v, int idx, TdShared& ts) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov < v || (ov == v && oi < idx)) {
      v = ov;
      idx = oi;
    }
  }
  __syncthreads();
  if (lane == 0) {
    ts.rv[w] = v;
    ts.ri[w] = idx;
  }
  __syncthreads();
  double bv = ts.rv[0];
  int bi = ts.ri[0];
  for (int i = 1; i < (int)(blockDim.x >> 5); ++i)
    if (ts.rv[i] < bv || (ts.rv[i] == bv && ts.ri[i] < bi)) {
      bv = ts.rv[i];
      bi = ts.ri[i];
    }
  return bi;
}

// Eigen-decomposition of the symmetric m x m matrix W (row-major, destroyed)
// by cyclic Jacobi with round-robin pairs; eigenvalues ascending in theta,
// eigenvectors in the columns of Z.  Every thread of the CTA takes part.
__device__ void small_eigh(int m, TdShared& ts, double* red) {
  const int tid = threadIdx.x, nt = blockDim.x;
  double* W = ts.Wk;
  double* V = ts.H;  // accumulated rotations (unsorted), H is rebuilt by the caller
  for (int e = tid; e < m * m; e += nt) V[e] = (e / m == e % m) ? 1.0 : 0.0;
  const int Ne = m + (m & 1), npair = Ne / 2;
  double scale = 0;
  for (int i = tid; i < m; i += nt) scale += W[i * m + i] * W[i * m + i];
  scale = cta_sum(scale, red);
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0;
    for (int e = tid; e < m * m; e += nt)
      if (e / m != e % m) off += W[e] * W[e];
    off = cta_sum(off, red);
    if (off <= 1e-30 * (scale + 1e-300)) break;
    for (int r = 0; r < Ne - 1; ++r) {
      for (int k = tid; k < npair; k += nt) {
        int p, q;
        rr_pair(r, k, Ne, p, q);
        double c = 1, s = 0;
        if (q < m && W[p * m + q] != 0.0) {
          const double apq = W[p * m + q];
          const double tau = (W[q * m + q] - W[p * m + p]) / (2.0 * apq);
          const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        ts.cs[2 * k] = c;
        ts.cs[2 * k + 1] = s;
        ts.pq[2 * k] = p;
        ts.pq[2 * k + 1] = q < m ? q : -1;
      }
      __syncthreads();
      // rows p, q <- J^T
      for (int e = tid; e < npair * m; e += nt) {
        const int k = e / m, col = e % m;
        const int p = ts.pq[2 * k], q = ts.pq[2 * k + 1];
        if (q < 0) continue;
        const double c = ts.cs[2 * k], s = ts.cs[2 * k + 1];
        const double a = W[p * m + col], b = W[q * m + col];
        W[p * m + col] = c * a - s * b;
        W[q * m + col] = s * a + c * b;
      }
      __syncthreads();
      // columns p, q of W and of the accumulated rotations <- J
      for (int e = tid; e < npair * m; e += nt) {
        const int k = e / m, row = e % m;
        const int p = ts.pq[2 * k], q = ts.pq[2 * k + 1];
        if (q < 0) continue;
        const double c = ts.cs[2 * k], s = ts.cs[2 * k + 1];
        const double a = W[row * m + p], b = W[row * m + q];
        W[row * m + p] = c * a - s * b;
        W[row * m + q] = s * a + c * b;
        const double u = V[row * m + p], v = V[row * m + q];
        V[row * m + p] = c * u - s * v;
        V[row * m + q] = s * u + c * v;
      }
      __syncthreads();
    }
  }
  // sort: rank of each eigenvalue, columns of V into Z in ascending order
  for (int i = tid; i < m; i += nt) {
    const double wi = W[i * m + i];
    int rk = 0;
    for (int j = 0; j < m; ++j) {
      const double wj = W[j * m + j];
      rk += (wj < wi || (wj == wi && j < i)) ? 1 : 0;
    }
    ts.theta[rk] = wi;
    ts.pq[i] = rk;
  }
  __syncthreads();
  for (int e = tid; e < m * m; e += nt) {
    const int row = e / m, col = e % m;
    ts.Z[row * m + ts.pq[col]] = V[e];
  }
  __syncthreads();
}

// Status of a molecule's excitations (info[2 * mol + 1]).
enum TdStatus : int {
  kTdOk = 0,
  kTdNotConverged = 1,      // Davidson iteration limit or stagnation
  kTdOrbitals = 2,          // canonical orbitals: Jacobi did not converge
  kTdNonPositive = 3,       // a Casida eigenvalue <= 0
  kTdNoReference = 4,       // the DFTB reference did not converge
};

__global__ void __launch_bounds__(kScfThreads, 1) k_tddftb(
    const MolDev* __restrict__ mols, int nmol, const int* __restrict__ order_list, int* counter,
    const AtomDev* __restrict__ atoms, const DftbElemDev* __restrict__ el, const double* __restrict__ Sall,
    const double* __restrict__ Xall, double* Fall, double* Call, double* W1all, double* W2all, double* epsall,
    double* rotbuf, const double* __restrict__ gamall, const MolResult* __restrict__ res, double* td,
    const long long* __restrict__ td_off, int nroots, int triplet, double tol, int max_iter, double* omega_out,
    double* dip_out, int* info, long long* cycles, size_t region_bytes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  unsigned char* after = smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16;
  TdShared& ts = *reinterpret_cast<TdShared*>(after);  // after the canonicalisation
  double* smemA = reinterpret_cast<double*>(after);     // packed Jacobi blocks during it
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5, nt = blockDim.x;
  while (true) {
    if (tid == 0) sh.mol = atomicAdd(counter, 1);
    __syncthreads();
    const int slot = sh.mol;
    __syncthreads();
    if (slot >= nmol) break;
    const int mi = order_list[slot];
    const MolDev m = mols[mi];
    const int N = m.nao, no = m.nocc, nv = N - no, nat = m.nat;
    const int dim = no * nv;
    const int k = nroots < dim ? nroots : dim;
    const int mmax = td_subspace(dim, k);
    double* om_out = omega_out + (size_t)mi * nroots;
    double* dp_out = dip_out + (size_t)mi * nroots * 3;
    for (int j = tid; j < 4 * nroots; j += nt) {
      if (j < nroots) om_out[j] = 0.0;
      else dp_out[j - nroots] = 0.0;
    }
    if (res[mi].status != kDevOk || !res[mi].converged || dim == 0) {
      if (tid == 0) {
        info[2 * mi] = 0;
        info[2 * mi + 1] = dim == 0 ? kTdOk : kTdNoReference;
      }
      __syncthreads();
      continue;
    }
    const double* S = Sall + m.mat_off;
    const double* X = Xall + m.mat_off;
    double* F = Fall + m.mat_off;
    double* Ct = Call + m.mat_off;
    double* W1 = W1all + m.mat_off;
    double* W2 = W2all + m.mat_off;
    double* eps = epsall + m.ao_base;
    const double* gm = gamall + m.gam_off;
    int status = kTdOk;
    const long long c0 = clock64();

    // 1. canonical orbitals of F' = X F X.  At self-consistency the
    //    occupied-virtual block of F' in the SCF's orbitals vanishes, so the
    //    occupied and the virtual blocks are diagonalised separately (a
    //    quarter of the work of one full diagonalisation, and blocks that fit
    //    shared memory); then C = X C'^T (AO rows, orbital columns) in W1, SC in W2
    cta_gemm(N, N, N, 1.0, F, N, false, X, N, false, 0.0, W1, N, sh.gemm);
    cta_gemm(N, N, N, 1.0, X, N, false, W1, N, false, 0.0, F, N, sh.gemm);
    for (int blk = 0; blk < 2; ++blk) {
      const int r0 = blk ? no : 0, n = blk ? nv : no;
      if (n == 0) continue;
      double* Cb = Ct + (size_t)r0 * N;
      cta_gemm(n, N, N, 1.0, Cb, N, false, F, N, false, 0.0, W1, N, sh.gemm);  // C_b F'
      cta_gemm(n, n, N, 1.0, W1, N, false, Cb, N, true, 0.0, W2, n, sh.gemm);  // C_b F' C_b^T
      const size_t pk_bytes = sizeof(double) * (size_t)n * (n + 1) / 2;
      const bool in_smem = pk_bytes <= region_bytes;
      double* A = in_smem ? smemA : W1;
      for (int e = tid; e < n * (n + 1) / 2; e += nt) {
        int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        while (i * (i + 1) / 2 > e) --i;
        const int j = e - i * (i + 1) / 2;
        A[e] = 0.5 * (W2[(size_t)i * n + j] + W2[(size_t)j * n + i]);
      }
      __syncthreads();
      double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
      const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((n + 1) / 2)));
      double* Afree = in_smem && region_bytes >= sizeof(double) * 32 * (size_t)n ? smemA : nullptr;
      const int sw = jacobi_diagonalise(n, A, Cb, false, rot, cap_rounds, sh.gemm, sizeof(sh.gemm), Afree,
                                        Afree ? region_bytes : 0, sh.rank, eps + r0, sh.js, sh.red, 30, 1e-12, N, N);
      if (sw < 0) status = kTdOrbitals;
    }
    cta_gemm(N, N, N, 1.0, X, N, false, Ct, N, true, 0.0, W1, N, sh.gemm);
    cta_gemm(N, N, N, 1.0, S, N, false, W1, N, false, 0.0, W2, N, sh.gemm);
    const double* C = W1;
    const double* SC = W2;
    const long long c1 = clock64();

    // per-molecule scratch
    double* hT = td + td_off[mi];                 // [nat][dim]  q sqrt(Delta)
    double* dl = hT + (size_t)nat * dim;          // [dim]       Delta
    double* D = dl + dim;                         // [3][dim]    transition dipole vectors
    double* V = D + 3 * (size_t)dim;              // [mmax][dim] subspace
    double* AV = V + (size_t)mmax * dim;          // [mmax][dim] Omega V
    double* T = AV + (size_t)mmax * dim;          // [2k][dim]   residuals / directions / restart
    double* Xa = T + 2 * (size_t)k * dim;         // [nat][mmax] h^T V
    double* Ya = Xa + (size_t)nat * mmax;         // [nat][mmax] G h^T V
    double* R = Ya + (size_t)nat * mmax;          // [mmax][mmax] Rayleigh matrix

    // 2. transition charges, Delta, dipole vectors (positions relative to the first atom)
    const AtomDev a0 = atoms[m.atom0];
    for (int kk = tid; kk < dim; kk += nt) {
      const int i = kk / nv, a = no + kk % nv;
      const double d = eps[a] - eps[i];
      const double sd = sqrt(fmax(d, 0.0));
      dl[kk] = d;
      double dx = 0, dy = 0, dz = 0;
      for (int A = 0; A < nat; ++A) {
        const AtomDev at = atoms[m.atom0 + A];
        const int na = el[at.slot].nao;
        double qa = 0;
        for (int mu = at.ao0; mu < at.ao0 + na; ++mu)
          qa += 0.5 * (C[(size_t)mu * N + i] * SC[(size_t)mu * N + a] + C[(size_t)mu * N + a] * SC[(size_t)mu * N + i]);
        hT[(size_t)A * dim + kk] = qa * sd;
        dx += qa * (at.x - a0.x);
        dy += qa * (at.y - a0.y);
        dz += qa * (at.z - a0.z);
      }
      D[kk] = dx;
      D[dim + kk] = dy;
      D[2 * (size_t)dim + kk] = dz;
    }
    __syncthreads();

    const long long c2 = clock64();

    // 3. start vectors: unit vectors of the m0 smallest Delta
    const int m0 = 2 * k < mmax ? 2 * k : mmax;
    for (int j = 0; j < m0; ++j) {
      double bv = 1e300;
      int bi = 0x7fffffff;
      for (int kk = tid; kk < dim; kk += nt) {
        bool taken = false;
        for (int t = 0; t < j; ++t) taken = taken || ts.sel[t] == kk;
        if (!taken && dl[kk] < bv) {
          bv = dl[kk];
          bi = kk;
        }
      }
      const int pick = cta_argmin(bv, bi, ts);
      if (tid == 0) ts.sel[j] = pick;
      __syncthreads();
    }
    for (int j = 0; j < m0; ++j)
      for (int kk = tid; kk < dim; kk += nt) V[(size_t)j * dim + kk] = kk == ts.sel[j] ? 1.0 : 0.0;
    __syncthreads();

    // 4. block Davidson
    int mcur = m0, mdone = 0, iter = 0, converged = 0;
    for (iter = 1; iter <= max_iter; ++iter) {
      const int nb = mcur - mdone;
      // sigma vectors of the new columns: Xa = h^T V, Ya = G Xa, AV = Delta^2 V + 4 h Ya
      for (int A = warp; A < nat; A += nwarps)
        for (int j0 = 0; j0 < nb; j0 += 8) {
          double acc[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) acc[jj] = 0.0;
          const int jn = nb - j0 < 8 ? nb - j0 : 8;
          for (int kk = lane; kk < dim; kk += 32) {
            const double h = hT[(size_t)A * dim + kk];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
              if (jj < jn) acc[jj] += h * V[(size_t)(mdone + j0 + jj) * dim + kk];
          }
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const double v = warp_sum(acc[jj]);
            if (lane == 0 && jj < jn) Xa[(size_t)A * mmax + j0 + jj] = v;
          }
        }
      __syncthreads();
      for (int e = tid; e < nat * nb; e += nt) {
        const int A = e / nb, j = e % nb;
        double y;
        if (triplet) {
          y = el[atoms[m.atom0 + A].slot].w * Xa[(size_t)A * mmax + j];
        } else {
          y = 0;
          for (int B = 0; B < nat; ++B) y += gm[(size_t)A * nat + B] * Xa[(size_t)B * mmax + j];
        }
        Ya[(size_t)A * mmax + j] = y;
      }
      __syncthreads();
      for (int kk = tid; kk < dim; kk += nt) {
        const double d2 = dl[kk] * dl[kk];
        for (int j0 = 0; j0 < nb; j0 += 8) {
          double acc[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) acc[jj] = 0.0;
          const int jn = nb - j0 < 8 ? nb - j0 : 8;
          for (int A = 0; A < nat; ++A) {
            const double h = hT[(size_t)A * dim + kk];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
              if (jj < jn) acc[jj] += h * Ya[(size_t)A * mmax + j0 + jj];
          }
          for (int jj = 0; jj < jn; ++jj) {
            const size_t o = (size_t)(mdone + j0 + jj) * dim + kk;
            AV[o] = d2 * V[o] + 4.0 * acc[jj];
          }
        }
      }
      __syncthreads();
      // Rayleigh matrix: R[i][j] = <V_i, AV_j> for the new columns j (i <= j among new ones)
      for (int e = warp; e < mcur * nb; e += nwarps) {
        const int i = e / nb, j = mdone + e % nb;
        if (i >= mdone && i > j) continue;
        double acc = 0;
        for (int kk = lane; kk < dim; kk += 32) acc += V[(size_t)i * dim + kk] * AV[(size_t)j * dim + kk];
        acc = warp_sum(acc);
        if (lane == 0) {
          R[(size_t)i * mmax + j] = acc;
          R[(size_t)j * mmax + i] = acc;
        }
      }
      __syncthreads();
      mdone = mcur;
      // eigenpairs of the Rayleigh matrix
      for (int e = tid; e < mcur * mcur; e += nt) ts.Wk[e] = R[(size_t)(e / mcur) * mmax + e % mcur];
      __syncthreads();
      small_eigh(mcur, ts, sh.red);
      // residuals r_j = (AV - theta_j V) z_j of the k lowest, into T[j]
      double rn[kTdMaxRoots];
#pragma unroll
      for (int j = 0; j < kTdMaxRoots; ++j) rn[j] = 0.0;
      for (int kk = tid; kk < dim; kk += nt) {
#pragma unroll
        for (int j = 0; j < kTdMaxRoots; ++j) {
          if (j >= k) break;
          double r = 0;
          for (int i = 0; i < mcur; ++i)
            r += (AV[(size_t)i * dim + kk] - ts.theta[j] * V[(size_t)i * dim + kk]) * ts.Z[i * mcur + j];
          T[(size_t)j * dim + kk] = r;
          rn[j] += r * r;
        }
      }
      if (tid < kTdMaxRoots) ts.rnorm[tid] = 0.0;
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kTdMaxRoots; ++j) {
        if (j >= k) break;
        const double v = warp_sum(rn[j]);
        if (lane == 0) atomicAdd(&ts.rnorm[j], v);
      }
      __syncthreads();
      int nconv = 0;
      for (int j = 0; j < k; ++j) nconv += sqrt(ts.rnorm[j]) < tol ? 1 : 0;
      if (nconv == k) {
        converged = 1;
        break;
      }
      // restart when the new directions do not fit: V, AV <- the k Ritz vectors
      const int nnew = k - nconv;
      if (mcur + nnew > mmax) {
        for (int pass = 0; pass < 2; ++pass) {
          double* B = pass ? AV : V;
          for (int kk = tid; kk < dim; kk += nt)
            for (int j = 0; j < k; ++j) {
              double v = 0;
              for (int i = 0; i < mcur; ++i) v += B[(size_t)i * dim + kk] * ts.Z[i * mcur + j];
              T[(size_t)(k + j) * dim + kk] = v;
            }
          __syncthreads();
          for (int j = 0; j < k; ++j)
            for (int kk = tid; kk < dim; kk += nt) B[(size_t)j * dim + kk] = T[(size_t)(k + j) * dim + kk];
          __syncthreads();
        }
        for (int e = tid; e < k * k; e += nt) {
          const int i = e / k, j = e % k;
          R[(size_t)i * mmax + j] = i == j ? ts.theta[i] : 0.0;
        }
        mcur = mdone = k;
        __syncthreads();
      }
      // preconditioned directions of the unconverged roots, orthonormalised into V
      int added = 0;
      for (int j = 0; j < k; ++j) {
        if (sqrt(ts.rnorm[j]) < tol) continue;
        if (mcur >= mmax) break;
        double* t = T + (size_t)j * dim;
        const double th = ts.theta[j];
        for (int kk = tid; kk < dim; kk += nt) {
          double den = th - dl[kk] * dl[kk];
          if (fabs(den) < 1e-8) den = den < 0 ? -1e-8 : 1e-8;
          t[kk] /= den;
        }
        __syncthreads();
        double nrm0 = 0;
        for (int kk = tid; kk < dim; kk += nt) nrm0 += t[kk] * t[kk];
        nrm0 = sqrt(cta_sum(nrm0, sh.red));
        for (int pass = 0; pass < 2; ++pass) {
          for (int i = warp; i < mcur; i += nwarps) {
            double acc = 0;
            for (int kk = lane; kk < dim; kk += 32) acc += V[(size_t)i * dim + kk] * t[kk];
            acc = warp_sum(acc);
            if (lane == 0) ts.coef[i] = acc;
          }
          __syncthreads();
          for (int kk = tid; kk < dim; kk += nt) {
            double v = t[kk];
            for (int i = 0; i < mcur; ++i) v -= ts.coef[i] * V[(size_t)i * dim + kk];
            t[kk] = v;
          }
          __syncthreads();
        }
        double nrm = 0;
        for (int kk = tid; kk < dim; kk += nt) nrm += t[kk] * t[kk];
        nrm = sqrt(cta_sum(nrm, sh.red));
        if (nrm > 1e-10 * nrm0 && nrm > 1e-300) {
          const double inv = 1.0 / nrm;
          for (int kk = tid; kk < dim; kk += nt) V[(size_t)mcur * dim + kk] = t[kk] * inv;
          ++mcur;
          ++added;
        }
        __syncthreads();
      }
      if (added == 0) {
        // nothing new to add: the subspace is the whole space (exact) or stagnated
        converged = mcur >= dim ? 1 : 0;
        break;
      }
    }
    if (!converged) status = status == kTdOk ? kTdNotConverged : status;

    // 5. excitation energies and transition dipoles of the k lowest roots
    for (int j = 0; j < k; ++j) {
      const double th = ts.theta[j];
      if (!(th > 0)) {
        status = kTdNonPositive;
        continue;
      }
      const double w = sqrt(th);
      double mx = 0, my = 0, mz = 0;
      for (int kk = tid; kk < dim; kk += nt) {
        double x = 0;
        for (int i = 0; i < mdone; ++i) x += V[(size_t)i * dim + kk] * ts.Z[i * mdone + j];
        const double c = sqrt(fmax(dl[kk], 0.0) / w) * x;
        mx += c * D[kk];
        my += c * D[dim + kk];
        mz += c * D[2 * (size_t)dim + kk];
      }
      mx = cta_sum(mx, sh.red);
      my = cta_sum(my, sh.red);
      mz = cta_sum(mz, sh.red);
      if (tid == 0) {
        om_out[j] = w;
        if (!triplet) {
          const double r2 = 1.4142135623730951;  // spin-adapted singlet: sqrt(2)
          dp_out[3 * j + 0] = r2 * mx;
          dp_out[3 * j + 1] = r2 * my;
          dp_out[3 * j + 2] = r2 * mz;
        }
      }
    }
    if (tid == 0) {
      info[2 * mi] = iter;
      info[2 * mi + 1] = status;
      cycles[3 * mi + 0] = c1 - c0;
      cycles[3 * mi + 1] = c2 - c1;
      cycles[3 * mi + 2] = clock64() - c2;
    }
    __syncthreads();
  }
}

// ScfShared, then one region for the packed Jacobi blocks of the
// canonicalisation and, afterwards, the Davidson state: all the opt-in shared
// memory that is left (at least the Davidson state).
size_t tddftb_smem_bytes(size_t* region_bytes) {
  const size_t base = ((sizeof(ScfShared) + 15) / 16) * 16;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  size_t region = (size_t)optin > base ? (((size_t)optin - base) / 16) * 16 : 0;
  if (region < sizeof(TdShared)) region = sizeof(TdShared);
  *region_bytes = region;
  return base + region;
}

}  // namespace

void launch_tddftb(const DeviceBatch& b, double* td, const long long* td_off, int nroots, int triplet, double tol,
                   int max_iter, double* omega, double* dip, int* info, long long* cycles, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  size_t region = 0;
  const size_t bytes = tddftb_smem_bytes(&region);
  cudaFuncSetAttribute(k_tddftb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  k_tddftb<<<grid, kScfThreads, bytes, s>>>(b.mols, b.nmol, b.order, b.counter, b.atoms, b.delems, b.S, b.X, b.F, b.C,
                                            b.W1, b.W2, b.eps, b.rotbuf, b.gam, b.res, td, td_off, nroots, triplet, tol,
                                            max_iter, omega, dip, info, cycles, region);
}

}  // namespace sgb
