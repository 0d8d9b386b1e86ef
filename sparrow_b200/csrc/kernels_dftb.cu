// DFTB2 / DFTB3 kernels: Slater-Koster pair blocks, on-site terms, the
// persistent self-consistent-charge kernel and the nuclear gradient.
//
// Reference behaviour followed (paths relative to
// src/Sparrow/Sparrow/Implementations/Dftb/):
//   H0, S                  Utils/ZeroOrderMatricesCalculator.cpp:56-232
//   gamma, gamma^h, Gamma  Utils/SecondOrderFock.cpp:53-113, Utils/ThirdOrderFock.cpp:55-155
//   charges, Fock          Utils/ScfFock.cpp:50-103 (Mulliken q = Z - N),
//                          SecondOrderFock.cpp:115-145, ThirdOrderFock.cpp:157-200
//   energy                 SecondOrderFock.cpp:178-195, ThirdOrderFock.cpp:228-255
//   density guess          Utils/DensityGuess.cpp:22-40
//   gradient               ZeroOrderMatricesCalculator.cpp:431-460,
//                          SecondOrderFock.cpp:148-176, ThirdOrderFock.cpp:202-226
// The self-consistent-charge Fock matrix is F = H0 + S o (s_a + s_b): every
// density-dependent term of DFTB2 and DFTB3 is a per-atom shift s_a, so one
// iteration costs an N^2 pass plus the atom-matrix products.  The
// generalised eigenproblem is solved in the Loewdin basis, X = S^-1/2 from a
// coupled Newton-Schulz iteration (GEMMs only), with the same DIIS, Jacobi
// cold start and occupied-virtual rotation as the NDDO kernel.  The
// energy-weighted density of the gradient is W = 1/2 P F P.
#include <cuda_runtime.h>

#include "dftb_math.cuh"
#include "kernels.h"
#include "scf_core.cuh"

namespace sgb {

namespace {

// ---------------------------------------------------------------------------
// Pair terms: S / H0 off-diagonal blocks, gamma (Gamma) entries, repulsion
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_dftb_pairs(const PairDev* __restrict__ pairs, int npairs,
                                                    const AtomDev* __restrict__ atoms, const MolDev* __restrict__ mols,
                                                    const DftbElemDev* __restrict__ el,
                                                    const DftbPairDev* __restrict__ pp, const double* __restrict__ table,
                                                    const DftbSplineDev* __restrict__ spl, int order, double* H0all,
                                                    double* Sall, double* gam, double* Gam, double* erep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev pr = pairs[p];
  const AtomDev A = atoms[pr.a], B = atoms[pr.b];
  const MolDev m = mols[pr.mol];
  const DftbElemDev ea = el[A.slot], eb = el[B.slot];
  const bool flip = ea.Z > eb.Z;  // the atom of lower Z comes first in the tables
  const double R[3] = {B.x - A.x, B.y - A.y, B.z - A.z};
  const double dist = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
  const double Rf[3] = {flip ? -R[0] : R[0], flip ? -R[1] : R[1], flip ? -R[2] : R[2]};
  const DftbPairDev& pf = flip ? pp[B.slot * kMaxElementSlots + A.slot] : pp[A.slot * kMaxElementSlots + B.slot];
  double me[2][4][4];
  dftb_blocks<double>(pf, table, flip ? eb.nao : ea.nao, flip ? ea.nao : eb.nao, Rf, me);
  const int N = m.nao;
  double* H0 = H0all + m.mat_off;
  double* S = Sall + m.mat_off;
  for (int i = 0; i < ea.nao; ++i)
    for (int j = 0; j < eb.nao; ++j) {
      const double s = flip ? me[0][j][i] : me[0][i][j];
      const double h = flip ? me[1][j][i] : me[1][i][j];
      const size_t u = A.ao0 + i, v = B.ao0 + j;
      S[u * N + v] = S[v * N + u] = s;
      H0[u * N + v] = H0[v * N + u] = h;
    }
  const int ia = pr.a - m.atom0, ib = pr.b - m.atom0, nat = m.nat;
  const DftbPairDev& pab = pp[A.slot * kMaxElementSlots + B.slot];
  if (order == 3) {
    double o[6];
    dftb_gamma3(ea, eb, pab, dist, o);
    gam[m.gam_off + (size_t)ia * nat + ib] = gam[m.gam_off + (size_t)ib * nat + ia] = o[0];
    Gam[m.gam_off + (size_t)ia * nat + ib] = o[2];
    Gam[m.gam_off + (size_t)ib * nat + ia] = o[4];
  } else {
    double g, dg;
    dftb_gamma2(ea, eb, pab, dist, g, dg);
    gam[m.gam_off + (size_t)ia * nat + ib] = gam[m.gam_off + (size_t)ib * nat + ia] = g;
  }
  double E, dE;
  dftb_repulsion(pab, spl, dist, E, dE);
  erep[p] = E;
}

// ---------------------------------------------------------------------------
// On-site blocks, gamma_aa (Gamma_aa), start density, repulsion energy
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dftb_onsite(const MolDev* __restrict__ mols, const AtomDev* __restrict__ atoms,
                                                     const DftbElemDev* __restrict__ el,
                                                     const int* __restrict__ ao_atom, const double* __restrict__ erep,
                                                     int order, double* H0all, double* Sall, double* gam, double* Gam,
                                                     double* Pall, MolResult* res, int write_guess) {
  __shared__ double red[32];
  const MolDev m = mols[blockIdx.x];
  const int N = m.nao, nat = m.nat;
  double* H0 = H0all + m.mat_off;
  double* S = Sall + m.mat_off;
  for (int a = threadIdx.x; a < nat; a += blockDim.x) {
    const AtomDev A = atoms[m.atom0 + a];
    const DftbElemDev e = el[A.slot];
    for (int i = 0; i < e.nao; ++i)
      for (int j = 0; j < e.nao; ++j) {
        const size_t u = A.ao0 + i, v = A.ao0 + j;
        H0[u * N + v] = i == j ? (i == 0 ? e.es : e.ep) : 0.0;
        S[u * N + v] = i == j ? 1.0 : 0.0;
      }
    gam[m.gam_off + (size_t)a * nat + a] = e.U;
    if (order == 3) Gam[m.gam_off + (size_t)a * nat + a] = 0.5 * e.hd;
  }
  if (write_guess) {
    // neutral atoms: the core charge spread over the atom's orbitals
    double* P = Pall + m.mat_off;
    for (int k = threadIdx.x; k < N * N; k += blockDim.x) {
      const int i = k / N, j = k % N;
      double v = 0.0;
      if (i == j) {
        const AtomDev A = atoms[ao_atom[m.ao_base + i]];
        const DftbElemDev e = el[A.slot];
        v = e.occ / e.nao;
      }
      P[k] = v;
    }
  }
  double s = 0;
  for (int k = threadIdx.x; k < m.npairs; k += blockDim.x) s += erep[m.pair0 + k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    res[blockIdx.x].e_rep = t;
  }
}

// ---------------------------------------------------------------------------
// Persistent self-consistent-charge kernel
// ---------------------------------------------------------------------------
// X = S^-1/2 by the coupled Newton-Schulz iteration Y <- Y T, Z <- T Z with
// T = (3 I - Z Y) / 2, Y0 = S / c, Z0 = I, c a Gershgorin bound on the largest
// eigenvalue of S; Z converges quadratically to (S / c)^-1/2.  Buffers:
// Y in {y0, y1}, Z in {X, z1}, T in t.  Returns the iterations used, or -1.
__device__ int inverse_sqrt(int N, const double* S, double* X, double* y0, double* y1, double* z1, double* t,
                            ScfShared& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int NN = N * N;
  double c = 0;
  for (int i = warp; i < N; i += nwarps) {
    double r = 0;
    for (int j = lane; j < N; j += 32) r += fabs(S[(size_t)i * N + j]);
    c = fmax(c, warp_sum(r));
  }
  c = cta_max(c, sh.red);
  const double ic = 1.0 / c;
  for (int k = tid; k < NN; k += blockDim.x) {
    y0[k] = S[k] * ic;
    X[k] = (k % (N + 1) == 0) ? 1.0 : 0.0;
  }
  __syncthreads();
  double *Y = y0, *Yn = y1, *Z = X, *Zn = z1;
  int it = 0, extra = -1;
  for (; it < 100; ++it) {
    for (int k = tid; k < NN; k += blockDim.x) t[k] = (k % (N + 1) == 0) ? 1.5 : 0.0;
    __syncthreads();
    cta_gemm(N, N, N, -0.5, Z, N, false, Y, N, false, 1.0, t, N, sh.gemm);  // T = 3/2 I - 1/2 Z Y
    double err = 0;
    for (int k = tid; k < NN; k += blockDim.x) err = fmax(err, fabs(t[k] - ((k % (N + 1) == 0) ? 1.0 : 0.0)));
    err = cta_max(err, sh.red);
    cta_gemm(N, N, N, 1.0, Y, N, false, t, N, false, 0.0, Yn, N, sh.gemm);
    cta_gemm(N, N, N, 1.0, t, N, false, Z, N, false, 0.0, Zn, N, sh.gemm);
    double* s1 = Y;
    Y = Yn;
    Yn = s1;
    double* s2 = Z;
    Z = Zn;
    Zn = s2;
    if (!isfinite(err)) return -1;
    if (extra < 0 && err < 1e-10) extra = 2;  // two more quadratic steps reach rounding level
    if (extra >= 0 && extra-- == 0) break;
  }
  const double sc = sqrt(ic);
  for (int k = tid; k < NN; k += blockDim.x) X[k] = Z[k] * sc;
  __syncthreads();
  return it < 100 ? it + 1 : -1;
}

// Mulliken charges, atom shifts and the per-atom energy terms for the AO
// density P.  Shift layout per atom: {s_a, V_a, A_a, unused} with
// V_a = -sum_i gamma_ai q_i, A_a = sum_i Gamma_ai q_i (DFTB3) and
// s_a = V_a / 2 + (2 q_a A_a + sum_i Gamma_ia q_i^2) / 6.  Returns
// sum_a (-1/2 q_a V_a - 1/3 q_a^2 A_a), i.e. E2 (+ E3).  pop: N scratch.
__device__ double charges_and_shifts(const MolDev& m, int order, const AtomDev* atoms, const DftbElemDev* el,
                                     const double* P, const double* S, const double* gm, const double* Gm, double* pop,
                                     double* q, double* sh4, double* red) {
  const int N = m.nao, nat = m.nat;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  for (int i = warp; i < N; i += nwarps) {
    double s = 0;
    for (int j = lane; j < N; j += 32) s += P[(size_t)i * N + j] * S[(size_t)i * N + j];
    s = warp_sum(s);
    if (lane == 0) pop[i] = s;
  }
  __syncthreads();
  for (int a = tid; a < nat; a += blockDim.x) {
    const AtomDev A = atoms[m.atom0 + a];
    const DftbElemDev e = el[A.slot];
    double n = 0;
    for (int k = 0; k < e.nao; ++k) n += pop[A.ao0 + k];
    q[a] = e.occ - n;
  }
  __syncthreads();
  double e23 = 0;
  for (int a = warp; a < nat; a += nwarps) {
    double V = 0, Aa = 0, Ba = 0;
    for (int i = lane; i < nat; i += 32) {
      V -= gm[(size_t)a * nat + i] * q[i];
      if (order == 3) {
        Aa += Gm[(size_t)a * nat + i] * q[i];
        Ba += Gm[(size_t)i * nat + a] * q[i] * q[i];
      }
    }
    V = warp_sum(V);
    Aa = warp_sum(Aa);
    Ba = warp_sum(Ba);
    if (lane == 0) {
      const double qa = q[a];
      sh4[4 * a + 0] = 0.5 * V + (order == 3 ? (2.0 * qa * Aa + Ba) / 6.0 : 0.0);
      sh4[4 * a + 1] = V;
      sh4[4 * a + 2] = Aa;
      e23 += -0.5 * qa * V - (order == 3 ? qa * qa * Aa / 3.0 : 0.0);
    }
  }
  return cta_sum(e23, red);
}

// F = H0 + S o (s_a + s_b) (warp per row); returns sum H0 o P.
__device__ double dftb_fock(const MolDev& m, const int* ao_atom, const double* H0, const double* S, const double* P,
                            const double* sh4, double* F, double* red) {
  const int N = m.nao;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  double eb = 0;
  for (int i = warp; i < N; i += nwarps) {
    const double si = sh4[4 * (ao_atom[m.ao_base + i] - m.atom0)];
    for (int j = lane; j < N; j += 32) {
      const size_t k = (size_t)i * N + j;
      const double sj = sh4[4 * (ao_atom[m.ao_base + j] - m.atom0)];
      F[k] = H0[k] + S[k] * (si + sj);
      eb += H0[k] * P[k];
    }
  }
  return cta_sum(eb, red);
}

__global__ void __launch_bounds__(kScfThreads, 1) k_dftb_scf(
    const MolDev* __restrict__ mols, int nmol, const int* __restrict__ order_list, int* counter,
    const AtomDev* __restrict__ atoms, const DftbElemDev* __restrict__ el, const int* __restrict__ ao_atom,
    const double* __restrict__ H0all, const double* __restrict__ Sall, double* Xall, double* Pall, double* Ppall,
    double* Fall, double* Call, double* W1all, double* W2all, double* epsall, double* diisall, double* rotbuf,
    const double* __restrict__ gamall, const double* __restrict__ Gamall, double* qall, double* shall,
    MolResult* res, ScfParams sp, int packed_in_smem, int order) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  double* smemA = reinterpret_cast<double*>(smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16);
  const int tid = threadIdx.x;
  while (true) {
    if (tid == 0) sh.mol = atomicAdd(counter, 1);
    __syncthreads();
    const int slot = sh.mol;
    __syncthreads();
    if (slot >= nmol) break;
    const int mi = order_list[slot];
    const MolDev m = mols[mi];
    const int N = m.nao, no = m.nocc;
    const size_t NN = (size_t)N * N;
    const double* H0 = H0all + m.mat_off;
    const double* S = Sall + m.mat_off;
    double* X = Xall + m.mat_off;
    double* P = Pall + m.mat_off;
    double* Pp = Ppall + m.mat_off;
    double* F = Fall + m.mat_off;
    double* Ct = Call + m.mat_off;
    double* W1 = W1all + m.mat_off;
    double* W2 = W2all + m.mat_off;
    // The buffers of F, C, W1, W2 and P trade roles during the SCF instead of
    // being copied into each other: role r lives in buffer (roles >> 3r) & 7
    // of Fall, Call, W1all, W2all, Pall.
    int roles = 0 | (1 << 3) | (2 << 6) | (3 << 9) | (4 << 12);
    auto buf = [&](int r) -> double* {
      const int b = (roles >> (3 * r)) & 7;
      double* base = b == 0 ? Fall : b == 1 ? Call : b == 2 ? W1all : b == 3 ? W2all : Pall;
      return base + m.mat_off;
    };
    auto trade = [&](int r1, int r2) {
      const int b1 = (roles >> (3 * r1)) & 7, b2 = (roles >> (3 * r2)) & 7;
      roles &= ~((7 << (3 * r1)) | (7 << (3 * r2)));
      roles |= (b2 << (3 * r1)) | (b1 << (3 * r2));
    };
    constexpr int kRF = 0, kRC = 1, kRW1 = 2, kRW2 = 3, kRP = 4;
    double* eps = epsall + m.ao_base;
    double* histF = diisall + m.diis_off;
    double* histE = histF + (size_t)kDiisMax * NN;
    const double* gm = gamall + m.gam_off;
    const double* Gm = Gamall + (order == 3 ? m.gam_off : 0);
    double* q = qall + m.atom0;
    double* sh4 = shall + 4 * (size_t)m.atom0;
    double* Apk = packed_in_smem ? smemA : nullptr;
    const size_t packed_bytes = sizeof(double) * (size_t)N * (N + 1) / 2;
    double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
    const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((N + 1) / 2)));
    const int msize = scf_diis_size(sp, N);
    const int cold_sweeps = sp.cold_sweeps > 0 ? sp.cold_sweeps : 6;
    int status = kDevOk;

    // Loewdin orthogonaliser (W1, F, Ct, W2 serve as Newton-Schulz buffers)
    const int ns_it = inverse_sqrt(N, S, X, W1, F, Ct, W2, sh);
    if (ns_it < 0) status = kDevNonFinite;

    int nhist = 0, head = 0, it = 0, converged = 0, nfull = 0, nsweeps = 0;
    bool have_orbitals = false;
    double drift = 0, Eold = 0, last_dE = 0, last_rms = 0;
    for (it = 1; it <= sp.max_iter && status == kDevOk; ++it) {
      F = buf(kRF);
      Ct = buf(kRC);
      W1 = buf(kRW1);
      W2 = buf(kRW2);
      P = buf(kRP);
      const double e23 = charges_and_shifts(m, order, atoms, el, P, S, gm, Gm, W2, q, sh4, sh.red);
      const double eb = dftb_fock(m, ao_atom, H0, S, P, sh4, F, sh.red);
      const double E = eb + e23;
      // F' = X F X
      cta_gemm(N, N, N, 1.0, F, N, false, X, N, false, 0.0, W1, N, sh.gemm);
      cta_gemm(N, N, N, 1.0, X, N, false, W1, N, false, 0.0, F, N, sh.gemm);
      if (have_orbitals) {
        const double* Fx = diis_step(N, F, Pp, W1, W2, histF, histE, msize, nhist, head, sh);
        if (Fx != F) {  // F and W2 trade buffers
          trade(kRF, kRW2);
          F = buf(kRF);
          W2 = buf(kRW2);
        }
      }
      int need_full = !have_orbitals;
      if (have_orbitals) {
        int sw = 0;
        need_full = ov_rotation(N, no, F, Ct, W1, W2, eps, drift, sh, nullptr, &sw);
        if (sw & 1) trade(kRC, kRF);
        if (sw & 2) trade(kRC, kRW2);
        F = buf(kRF);
        Ct = buf(kRC);
        W2 = buf(kRW2);
      }
      if (need_full && scf_eig_mode(sp, N) != kEigRotation) {
        // every eigenpair of F' by the tridiagonal solver; the rotations take over
        need_full = eigh_tridiag(N, F, N, N, Ct, N, eps, sh.gemm, eig_workspace_doubles(sh, smem_raw), W2, W1, Ct, F,
                                 sh.red, &sh.flag);
        if (need_full) {
          have_orbitals = false;  // the solver used Ct as scratch: the fallback starts cold
        } else {
          have_orbitals = true;
          drift = 0;
          ++nfull;
        }
      }
      if (need_full) {
        const int sw = full_diagonalise(N, F, Ct, W1, W2, eps, Apk ? Apk : F, Apk ? packed_bytes : 0, have_orbitals,
                                        rot, cap_rounds, have_orbitals ? sp.jacobi_max_sweeps : cold_sweeps,
                                        have_orbitals ? 1e-10 : 1e-3, sh);
        if (sw < 0 && have_orbitals) status = kDevJacobiNotConverged;
        nsweeps += sw < 0 ? (have_orbitals ? sp.jacobi_max_sweeps : cold_sweeps) : sw;
        ++nfull;
        have_orbitals = true;
        drift = 0;
      }
      // P' = 2 C'_occ C'_occ^T, P = X P' X
      cta_gemm(N, N, no, 2.0, Ct, N, true, Ct, N, false, 0.0, Pp, N, sh.gemm, true);
      cta_gemm(N, N, N, 1.0, X, N, false, Pp, N, false, 0.0, W1, N, sh.gemm);
      cta_gemm(N, N, N, 1.0, W1, N, false, X, N, false, 0.0, W2, N, sh.gemm, true);
      double d2 = 0;
#pragma unroll 4
      for (size_t k = tid; k < NN; k += blockDim.x) {
        const double d = W2[k] - P[k];
        d2 += d * d;
      }
      d2 = cta_sum(d2, sh.red);
      trade(kRP, kRW2);  // the new density's buffer becomes P's
      const double rms = sqrt(d2 / (double)NN);
      last_rms = rms;
      last_dE = it > 1 ? fabs(E - Eold) : 0.0;
      const bool dE_ok = it > 1 && fabs(E - Eold) < sp.scc;
      Eold = E;
      if (!isfinite(E) || !isfinite(rms)) {
        status = kDevNonFinite;
        break;
      }
      if (dE_ok && rms < sp.rmsd) {
        converged = 1;
        break;
      }
      __syncthreads();
    }
    if (it > sp.max_iter) it = sp.max_iter;
    __syncthreads();
    // Back to the home buffers: the density to Pall's, the orbitals to
    // Call's (the canonical-orbital and TD-DFTB kernels read them); F, W1 and
    // W2 take theirs for the closing products (the gradient reads W1's).
    // W2's buffer holds nothing live and takes the orbitals when they sit in
    // the density's.
    {
      double* const bP = Pall + m.mat_off;
      double* const bC = Call + m.mat_off;
      P = buf(kRP);
      Ct = buf(kRC);
      if (P != bP) {
        if (Ct == bP) {
          W2 = buf(kRW2);
          for (size_t k = tid; k < NN; k += blockDim.x) W2[k] = Ct[k];
          __syncthreads();
          Ct = W2;
        }
        for (size_t k = tid; k < NN; k += blockDim.x) bP[k] = P[k];
        __syncthreads();
      }
      if (Ct != bC) {
        for (size_t k = tid; k < NN; k += blockDim.x) bC[k] = Ct[k];
        __syncthreads();
      }
      P = bP;
      Ct = bC;
      F = Fall + m.mat_off;
      W1 = W1all + m.mat_off;
      W2 = W2all + m.mat_off;
    }
    // final charges, Fock matrix and energy of the converged density; W = 1/2 P F P into W1
    const double e23 = charges_and_shifts(m, order, atoms, el, P, S, gm, Gm, W2, q, sh4, sh.red);
    const double eb = dftb_fock(m, ao_atom, H0, S, P, sh4, F, sh.red);
    cta_gemm(N, N, N, 1.0, F, N, false, P, N, false, 0.0, W2, N, sh.gemm);
    cta_gemm(N, N, N, 0.5, P, N, false, W2, N, false, 0.0, W1, N, sh.gemm, true);
    if (tid == 0) {
      MolResult& r = res[mi];
      r.e_el = eb + e23;
      r.energy = r.e_el + r.e_rep;
      r.iterations = it;
      r.converged = converged;
      r.status = status;
      r.last_dE = last_dE;
      r.last_rmsd = last_rms;
      r.full_diag = nfull;
      r.jacobi_sweeps = nsweeps;
      r.cycles[0] = ns_it;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Nuclear gradient per pair (dE/dR_b, R = R_b - R_a)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64) k_dftb_gradient(const PairDev* __restrict__ pairs, int npairs,
                                                      const AtomDev* __restrict__ atoms,
                                                      const MolDev* __restrict__ mols,
                                                      const DftbElemDev* __restrict__ el,
                                                      const DftbPairDev* __restrict__ pp,
                                                      const double* __restrict__ table,
                                                      const DftbSplineDev* __restrict__ spl, int order,
                                                      const double* __restrict__ Pall, const double* __restrict__ Wall,
                                                      const double* __restrict__ qall,
                                                      const double* __restrict__ shall, double* __restrict__ gpair) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev pr = pairs[p];
  const AtomDev A = atoms[pr.a], B = atoms[pr.b];
  const MolDev m = mols[pr.mol];
  const DftbElemDev ea = el[A.slot], eb = el[B.slot];
  const bool flip = ea.Z > eb.Z;
  const double R[3] = {B.x - A.x, B.y - A.y, B.z - A.z};
  const double dist = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
  const double Rf[3] = {flip ? -R[0] : R[0], flip ? -R[1] : R[1], flip ? -R[2] : R[2]};
  const DftbPairDev& pf = flip ? pp[B.slot * kMaxElementSlots + A.slot] : pp[A.slot * kMaxElementSlots + B.slot];
  Dual3 me[2][4][4];
  const int nz = dftb_blocks<Dual3>(pf, table, flip ? eb.nao : ea.nao, flip ? ea.nao : eb.nao, Rf, me);
  const int N = m.nao;
  const double* P = Pall + m.mat_off;
  const double* W = Wall + m.mat_off;
  const double sab = shall[4 * (size_t)pr.a] + shall[4 * (size_t)pr.b];
  const double sgn = flip ? -1.0 : 1.0;  // blocks were differentiated with respect to -R when flipped
  double d[3] = {0, 0, 0};
  if (nz)
    for (int i = 0; i < ea.nao; ++i)
      for (int j = 0; j < eb.nao; ++j) {
        const Dual3& s = flip ? me[0][j][i] : me[0][i][j];
        const Dual3& h = flip ? me[1][j][i] : me[1][i][j];
        const size_t u = A.ao0 + i, v = B.ao0 + j;
        const double Puv = P[u * N + v];
        const double Wm = W[u * N + v] - sab * Puv;
        d[0] += 2.0 * sgn * (Puv * h.dx - Wm * s.dx);
        d[1] += 2.0 * sgn * (Puv * h.dy - Wm * s.dy);
        d[2] += 2.0 * sgn * (Puv * h.dz - Wm * s.dz);
      }
  const double qa = qall[pr.a], qb = qall[pr.b];
  const DftbPairDev& pab = pp[A.slot * kMaxElementSlots + B.slot];
  double coef;
  if (order == 3) {
    double o[6];
    dftb_gamma3(ea, eb, pab, dist, o);
    // the reference's pair term: q_a q_b gamma' + q_a q_b / 3 (q_b Gamma_ba' - q_a Gamma_ab')
    coef = qa * qb * o[1] + (qa * qb / 3.0) * (qb * o[5] - qa * o[3]);
  } else {
    double g, dg;
    dftb_gamma2(ea, eb, pab, dist, g, dg);
    coef = qa * qb * dg;
  }
  double E, dE;
  dftb_repulsion(pab, spl, dist, E, dE);
  coef += dE;
  for (int k = 0; k < 3; ++k) gpair[(size_t)p * 3 + k] = d[k] + coef * R[k] / dist;
}

// ---------------------------------------------------------------------------
// Spin-polarised (unrestricted) DFTB, Utils/SDFTB.cpp:64-293 and
// Utils/ScfFock.cpp:50-103: the spin Fock matrices are the restricted SCC
// Fock matrix of the total density plus / minus spinC o S,
//   spinC_mu,nu = 1/2 (eps_{a(mu),l(mu)} + eps_{b(nu),l(nu)}),
//   eps_{a,l} = sum_l' W_a(l, l') pdif_{a,l'},
//   pdif_{a,l} = sum_{mu in (a, l)} sum_nu (P_a - P_b)_mu,nu S_mu,nu,
// with the energy 1/2 sum_a sum_{l,l'} pdif_{a,l} W_a(l, l') pdif_{a,l'}.
// ---------------------------------------------------------------------------
// Shell shifts eps_{a,s}, eps_{a,p} of the molecule's atoms into sps (2 per
// atom); pop: N doubles of scratch.  Returns the spin energy.
__device__ double dftb_spin_shifts(const MolDev& m, const AtomDev* __restrict__ atoms,
                                   const DftbElemDev* __restrict__ el, const double* Pa, const double* Pb,
                                   const double* S, double* pop, double* sps, double* red) {
  const int N = m.nao;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  for (int i = warp; i < N; i += nwarps) {
    double s = 0;
    for (int j = lane; j < N; j += 32) {
      const size_t ij = (size_t)i * N + j;
      s += (Pa[ij] - Pb[ij]) * S[ij];
    }
    s = warp_sum(s);
    if (lane == 0) pop[i] = s;
  }
  __syncthreads();
  double e = 0;
  for (int a = tid; a < m.nat; a += blockDim.x) {
    const AtomDev A = atoms[m.atom0 + a];
    const DftbElemDev& E = el[A.slot];
    const double ps = pop[A.ao0];
    const double pp = E.nao == 4 ? pop[A.ao0 + 1] + pop[A.ao0 + 2] + pop[A.ao0 + 3] : 0.0;
    const double es = E.wss * ps + E.wsp * pp, ep = E.wps * ps + E.wpp * pp;
    sps[2 * a] = es;
    sps[2 * a + 1] = ep;
    e += 0.5 * (ps * es + pp * ep);
  }
  __syncthreads();
  return cta_sum(e, red);
}

// spinC of AO pair (u, v) from the shell shifts
__device__ __forceinline__ double dftb_spin_c(const MolDev& m, const AtomDev* __restrict__ atoms,
                                              const int* __restrict__ ao_atom, const double* sps, int u, int v) {
  const int A = ao_atom[m.ao_base + u], B = ao_atom[m.ao_base + v];
  const double eu = sps[2 * (A - m.atom0) + (u == atoms[A].ao0 ? 0 : 1)];
  const double ev = sps[2 * (B - m.atom0) + (v == atoms[B].ao0 ? 0 : 1)];
  return 0.5 * (eu + ev);
}

__global__ void __launch_bounds__(kScfThreads, 1) k_dftb_uhf_scf(
    const MolDev* __restrict__ mols, int nmol, const int* __restrict__ order_list, int* counter,
    const AtomDev* __restrict__ atoms, const DftbElemDev* __restrict__ el, const int* __restrict__ ao_atom,
    const double* __restrict__ H0all, const double* __restrict__ Sall, double* Xall, double* Pall, double* Ppall,
    double* Fall, double* Call, double* W1all, double* W2all, double* epsall, double* diisall, double* Paall,
    double* Pball, double* Ppball, double* Fball, double* Cball, double* epsball, double* diisball, double* sshall,
    double* rotbuf, const double* __restrict__ gamall, const double* __restrict__ Gamall, double* qall, double* shall,
    MolResult* res, ScfParams sp, int packed_in_smem, int order, int spin_given) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  double* smemA = reinterpret_cast<double*>(smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16);
  const int tid = threadIdx.x;
  while (true) {
    if (tid == 0) sh.mol = atomicAdd(counter, 1);
    __syncthreads();
    const int slot = sh.mol;
    __syncthreads();
    if (slot >= nmol) break;
    const int mi = order_list[slot];
    const MolDev m = mols[mi];
    const int N = m.nao, na = m.nocc, nb = m.nocc_b;
    const size_t NN = (size_t)N * N;
    const double* H0 = H0all + m.mat_off;
    const double* S = Sall + m.mat_off;
    double* X = Xall + m.mat_off;
    double* P = Pall + m.mat_off;
    double* Pa = Paall + m.mat_off;
    double* Pb = Pball + m.mat_off;
    double* Ppa = Ppall + m.mat_off;
    double* Ppb = Ppball + m.mat_off;
    double* Fa = Fall + m.mat_off;
    double* Fb = Fball + m.mat_off;
    double* Ca = Call + m.mat_off;
    double* Cb = Cball + m.mat_off;
    double* W1 = W1all + m.mat_off;
    double* W2 = W2all + m.mat_off;
    double* epsa = epsall + m.ao_base;
    double* epsb = epsball + m.ao_base;
    double* histFa = diisall + m.diis_off;
    double* histEa = histFa + (size_t)kDiisMax * NN;
    double* histFb = diisball + m.diis_off;
    double* histEb = histFb + (size_t)kDiisMax * NN;
    const double* gm = gamall + m.gam_off;
    const double* Gm = Gamall + (order == 3 ? m.gam_off : 0);
    double* q = qall + m.atom0;
    double* sh4 = shall + 4 * (size_t)m.atom0;
    double* sps = sshall + 2 * (size_t)m.atom0;
    double* Apk = packed_in_smem ? smemA : nullptr;
    const size_t packed_bytes = sizeof(double) * (size_t)N * (N + 1) / 2;
    double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
    const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((N + 1) / 2)));
    const int msize = scf_diis_size(sp, N);
    const int cold_sweeps = sp.cold_sweeps > 0 ? sp.cold_sweeps : 6;
    int status = kDevOk;
    const int ns_it = inverse_sqrt(N, S, X, W1, Fa, Ca, W2, sh);
    if (ns_it < 0) status = kDevNonFinite;
    if (!spin_given)  // given spin densities (warm start) keep their polarisation
      for (size_t k = tid; k < NN; k += blockDim.x) Pa[k] = Pb[k] = 0.5 * P[k];
    __syncthreads();
    int nhist = 0, head = 0, it = 0, converged = 0, nfull = 0, nsweeps = 0;
    bool have_a = false, have_b = false;
    double drift_a = 0, drift_b = 0, Eold = 0, last_dE = 0, last_rms = 0;
    for (it = 1; it <= sp.max_iter && status == kDevOk; ++it) {
      const double e23 = charges_and_shifts(m, order, atoms, el, P, S, gm, Gm, W2, q, sh4, sh.red);
      const double eb = dftb_fock(m, ao_atom, H0, S, P, sh4, Fa, sh.red);
      const double es = dftb_spin_shifts(m, atoms, el, Pa, Pb, S, W2, sps, sh.red);
      for (size_t k = tid; k < NN; k += blockDim.x) {
        const int u = (int)(k / N), v = (int)(k % N);
        const double c = dftb_spin_c(m, atoms, ao_atom, sps, u, v) * S[k];
        const double fr = Fa[k];
        Fa[k] = fr + c;
        Fb[k] = fr - c;
      }
      __syncthreads();
      const double E = eb + e23 + es;
      // F'_s = X F_s X
      cta_gemm(N, N, N, 1.0, Fa, N, false, X, N, false, 0.0, W1, N, sh.gemm);
      cta_gemm(N, N, N, 1.0, X, N, false, W1, N, false, 0.0, Fa, N, sh.gemm);
      cta_gemm(N, N, N, 1.0, Fb, N, false, X, N, false, 0.0, W1, N, sh.gemm);
      cta_gemm(N, N, N, 1.0, X, N, false, W1, N, false, 0.0, Fb, N, sh.gemm);
      if (have_a && have_b)
        diis_step_uhf(N, Fa, Ppa, Fb, Ppb, W1, histFa, histEa, histFb, histEb, msize, nhist, head, sh);
      const bool warm_a = have_a, warm_b = have_b;
      const size_t wsd = eig_workspace_doubles(sh, smem_raw);
      int sw = uhf_orbitals(N, na, Fa, Ca, W1, W2, epsa, Apk, packed_bytes, have_a, drift_a, rot, cap_rounds, sp,
                            cold_sweeps, nfull, sh, sh.gemm, wsd);
      if (sw < 0 && warm_a) status = kDevJacobiNotConverged;
      nsweeps += sw < 0 ? -sw : sw;
      sw = uhf_orbitals(N, nb, Fb, Cb, W1, W2, epsb, Apk, packed_bytes, have_b, drift_b, rot, cap_rounds, sp,
                        cold_sweeps, nfull, sh, sh.gemm, wsd);
      if (sw < 0 && warm_b) status = kDevJacobiNotConverged;
      nsweeps += sw < 0 ? -sw : sw;
      // P'_s = C'_occ C'_occ^T, P_s = X P'_s X; rms of the AO spin densities
      double d2max = 0;
      for (int spin = 0; spin < 2; ++spin) {
        double* Pps = spin ? Ppb : Ppa;
        double* Ps = spin ? Pb : Pa;
        uhf_density(N, spin ? nb : na, spin ? Cb : Ca, Pps, W1, sh);
        cta_gemm(N, N, N, 1.0, X, N, false, Pps, N, false, 0.0, W1, N, sh.gemm);
        cta_gemm(N, N, N, 1.0, W1, N, false, X, N, false, 0.0, W2, N, sh.gemm, true);
        double d2 = 0;
        for (size_t k = tid; k < NN; k += blockDim.x) {
          const double d = W2[k] - Ps[k];
          d2 += d * d;
          Ps[k] = W2[k];
        }
        d2max = fmax(d2max, cta_sum(d2, sh.red));
      }
      for (size_t k = tid; k < NN; k += blockDim.x) P[k] = Pa[k] + Pb[k];
      __syncthreads();
      const double rms = sqrt(d2max / (double)NN);
      last_rms = rms;
      last_dE = it > 1 ? fabs(E - Eold) : 0.0;
      const bool dE_ok = it > 1 && fabs(E - Eold) < sp.scc;
      Eold = E;
      if (!isfinite(E) || !isfinite(rms)) {
        status = kDevNonFinite;
        break;
      }
      if (dE_ok && rms < sp.rmsd) {
        converged = 1;
        break;
      }
    }
    if (it > sp.max_iter) it = sp.max_iter;
    __syncthreads();
    // final charges, spin Fock matrices and energy of the converged densities;
    // the gradient's overlap multiplier into W1:
    //   P_a F_a P_a + P_b F_b P_b - spinC o (P_a - P_b)
    // (energy-weighted densities; SDFTB.cpp:60-83 adds 2 (P_a - P_b) spinC dS)
    const double e23 = charges_and_shifts(m, order, atoms, el, P, S, gm, Gm, W2, q, sh4, sh.red);
    const double eb = dftb_fock(m, ao_atom, H0, S, P, sh4, Fa, sh.red);
    const double es = dftb_spin_shifts(m, atoms, el, Pa, Pb, S, W2, sps, sh.red);
    for (size_t k = tid; k < NN; k += blockDim.x) {
      const int u = (int)(k / N), v = (int)(k % N);
      const double c = dftb_spin_c(m, atoms, ao_atom, sps, u, v) * S[k];
      const double fr = Fa[k];
      Fa[k] = fr + c;
      Fb[k] = fr - c;
    }
    __syncthreads();
    cta_gemm(N, N, N, 1.0, Fa, N, false, Pa, N, false, 0.0, W2, N, sh.gemm);
    cta_gemm(N, N, N, 1.0, Pa, N, false, W2, N, false, 0.0, W1, N, sh.gemm, true);
    cta_gemm(N, N, N, 1.0, Fb, N, false, Pb, N, false, 0.0, W2, N, sh.gemm);
    cta_gemm(N, N, N, 1.0, Pb, N, false, W2, N, false, 1.0, W1, N, sh.gemm, true);
    for (size_t k = tid; k < NN; k += blockDim.x) {
      const int u = (int)(k / N), v = (int)(k % N);
      W1[k] -= dftb_spin_c(m, atoms, ao_atom, sps, u, v) * (Pa[k] - Pb[k]);
    }
    __syncthreads();
    if (tid == 0) {
      MolResult& r = res[mi];
      r.e_el = eb + e23 + es;
      r.energy = r.e_el + r.e_rep;
      r.iterations = it;
      r.converged = converged;
      r.status = status;
      r.last_dE = last_dE;
      r.last_rmsd = last_rms;
      r.full_diag = nfull;
      r.jacobi_sweeps = nsweeps;
      r.cycles[0] = ns_it;
    }
    __syncthreads();
  }
}

// Canonical orbitals after a DFTB convergence (ScfParams::canonical): F' =
// X F X of each spin's final Fock matrix (left in F / Fb by the SCC kernels)
// into the orthogonal-basis density buffer (free after convergence), then a
// warm diagonalisation with W2 and W3 as scratch.  F / Fb (read by TD-DFTB)
// and W1 (the gradient's energy-weighted density) stay intact.
__global__ void __launch_bounds__(kScfThreads, 1) k_dftb_canonical(
    const MolDev* __restrict__ mols, int nmol, const int* __restrict__ order_list, int* counter,
    const double* __restrict__ Xall, const double* __restrict__ Fall, double* Call, double* Ppall, double* W2all,
    double* W3all, double* epsall, const double* __restrict__ Fball, double* Cball, double* Ppball, double* epsball,
    double* rotbuf, ScfParams sp, int packed_in_smem) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScfShared& sh = *reinterpret_cast<ScfShared*>(smem_raw);
  double* smemA = reinterpret_cast<double*>(smem_raw + ((sizeof(ScfShared) + 15) / 16) * 16);
  for (;;) {
    if (threadIdx.x == 0) {
      const int k = atomicAdd(counter, 1);
      sh.mol = k < nmol ? order_list[k] : -1;
    }
    __syncthreads();
    const int mi = sh.mol;
    __syncthreads();
    if (mi < 0) return;
    const MolDev m = mols[mi];
    const int N = m.nao;
    const double* X = Xall + m.mat_off;
    double* W2 = W2all + m.mat_off;
    double* W3 = W3all + m.mat_off;
    double* Apk = packed_in_smem ? smemA : nullptr;
    const size_t packed_bytes = sizeof(double) * (size_t)N * (N + 1) / 2;
    double* rot = rotbuf + (size_t)blockIdx.x * (kRotBudgetBytes / sizeof(double));
    const int cap_rounds = (int)((kRotBudgetBytes / sizeof(double)) / (2 * ((N + 1) / 2)));
    for (int spin = 0; spin < (Fball ? 2 : 1); ++spin) {
      const double* F = (spin ? Fball : Fall) + m.mat_off;
      double* Fp = (spin ? Ppball : Ppall) + m.mat_off;
      cta_gemm(N, N, N, 1.0, F, N, false, X, N, false, 0.0, W2, N, sh.gemm);
      cta_gemm(N, N, N, 1.0, X, N, false, W2, N, false, 0.0, Fp, N, sh.gemm);
      double* Ct = (spin ? Cball : Call) + m.mat_off;
      double* eps = (spin ? epsball : epsall) + m.ao_base;
      // every eigenpair of F' by the tridiagonal solver; clustered spectra by a
      // Jacobi diagonalisation from scratch (the solver used Ct as scratch)
      const int st = eigh_tridiag(N, Fp, N, N, Ct, N, eps, sh.gemm, eig_workspace_doubles(sh, smem_raw), W2, W3, Ct,
                                  Fp, sh.red, &sh.flag);
      if (st != 0)
        full_diagonalise(N, Fp, Ct, W3, W2, eps, Apk ? Apk : Fp, Apk ? packed_bytes : 0, false, rot, cap_rounds,
                         sp.jacobi_max_sweeps, 1e-10, sh);
    }
    __syncthreads();
  }
}


// One CTA per SM: the persistent kernels take all the opt-in shared memory
// (the Jacobi solver's packed matrix when it fits, the tridiagonal solver's
// tiles up to 192 AOs).
size_t dftb_smem_bytes(int max_nao, int* packed_in_smem) {
  const size_t base = ((sizeof(ScfShared) + 15) / 16) * 16;
  const size_t pk = sizeof(double) * (size_t)max_nao * (max_nao + 1) / 2;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  *packed_in_smem = base + pk <= (size_t)optin ? 1 : 0;
  return (size_t)optin > base ? (size_t)optin : base;
}

}  // namespace

void launch_dftb_setup(const DeviceBatch& b, cudaStream_t s) {
  if (b.npairs > 0) {
    const int th = 128;
    k_dftb_pairs<<<(b.npairs + th - 1) / th, th, 0, s>>>(b.pairs, b.npairs, b.atoms, b.mols, b.delems, b.dpairs,
                                                         b.dtable, b.dsplines, b.dftb_order, b.H, b.S, b.gam, b.Gam,
                                                         b.erep);
  }
  k_dftb_onsite<<<b.nmol, 256, 0, s>>>(b.mols, b.atoms, b.delems, b.ao_atom, b.erep, b.dftb_order, b.H, b.S, b.gam,
                                       b.Gam, b.P, b.res, b.use_guess);
}

void launch_dftb_canonical(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  int in_smem = 0;
  const size_t bytes = dftb_smem_bytes(b.max_nao, &in_smem);
  cudaFuncSetAttribute(k_dftb_canonical, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  k_dftb_canonical<<<grid, kScfThreads, bytes, s>>>(b.mols, b.nmol, b.order, b.counter, b.X, b.F, b.C, b.Pp, b.W2,
                                                    b.W3, b.eps, b.uhf ? b.Fb : nullptr, b.Cb, b.Ppb, b.epsb,
                                                    b.rotbuf, sp, in_smem);
}

void launch_dftb_scf(const DeviceBatch& b, const ScfParams& sp, int grid, cudaStream_t s) {
  if (b.nmol == 0) return;
  int in_smem = 0;
  const size_t bytes = dftb_smem_bytes(b.max_nao, &in_smem);
  cudaFuncSetAttribute(k_dftb_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaMemsetAsync(b.counter, 0, sizeof(int), s);
  if (grid > b.nmol) grid = b.nmol;
  if (b.uhf) {
    cudaFuncSetAttribute(k_dftb_uhf_scf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    k_dftb_uhf_scf<<<grid, kScfThreads, bytes, s>>>(
        b.mols, b.nmol, b.order, b.counter, b.atoms, b.delems, b.ao_atom, b.H, b.S, b.X, b.P, b.Pp, b.F, b.C, b.W1,
        b.W2, b.eps, b.diis, b.Pa, b.Pb, b.Ppb, b.Fb, b.Cb, b.epsb, b.diisb, b.sshift, b.rotbuf, b.gam, b.Gam, b.qat,
        b.ashift, b.res, sp, in_smem, b.dftb_order, b.spin_given);
    return;
  }
  k_dftb_scf<<<grid, kScfThreads, bytes, s>>>(b.mols, b.nmol, b.order, b.counter, b.atoms, b.delems, b.ao_atom, b.H,
                                              b.S, b.X, b.P, b.Pp, b.F, b.C, b.W1, b.W2, b.eps, b.diis, b.rotbuf,
                                              b.gam, b.Gam, b.qat, b.ashift, b.res, sp, in_smem, b.dftb_order);
}

void launch_dftb_gradient(const DeviceBatch& b, cudaStream_t s) {
  if (b.npairs > 0) {
    const int th = 64;
    k_dftb_gradient<<<(b.npairs + th - 1) / th, th, 0, s>>>(b.pairs, b.npairs, b.atoms, b.mols, b.delems, b.dpairs,
                                                            b.dtable, b.dsplines, b.dftb_order, b.P, b.W1, b.qat,
                                                            b.ashift, b.gpair);
  }
  launch_gather_gradient(b, s);
}

}  // namespace sgb
