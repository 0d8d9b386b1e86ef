// Allocation-free single-molecule entry point (sg_calculate_static).
//
// This entry point has no counterpart in the reference.  It runs the same
// kernels as the batched engine (pair integrals, one-electron assembly,
// persistent SCF, gradient) for one molecule, but every device buffer lives in
// one file-scope __device__ array of fixed size and every host-side table in a
// file-scope host array: no cudaMalloc / cudaFree / cudaMallocHost and no heap
// use on the per-call path.
//
// Set-up: the first call on a device (with that device current) looks up the
// scratch array's address with cudaGetSymbolAddress and builds the local
// multipole term table on the host; make that first call before any stream
// capture begins.  Every call (the first included) repeats the address lookup,
// uploads the term table to constant memory from pageable host memory and
// synchronises the stream before it returns, so the entry point stays valid
// after a cudaDeviceReset.  Calls that overlap in time (from two host threads,
// or on two streams of one device) share the scratch and race; callers
// serialise them.
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/sparrow_b200.h"
#include "engine.h"
#include "kernels.h"
#include "nddo_math.cuh"
#include "params.h"

namespace sgb {

void build_local_term_table(LocalTermTable& tab);

namespace {

constexpr int kStaticMaxAtoms = SG_STATIC_MAX_ATOMS;
constexpr int kStaticMaxAos = SG_STATIC_MAX_AOS;
constexpr int kStaticMaxPairs = kStaticMaxAtoms * (kStaticMaxAtoms - 1) / 2;
constexpr int kMaxDevices = 64;

constexpr size_t al256(size_t x) { return (x + 255) / 256 * 256; }

// Byte offsets of every buffer inside the scratch array; the first
// header_end bytes are the descriptor tables, uploaded with one copy.
struct StaticLayout {
  size_t mols, atoms, pairs, elems, diat, ao, order, hh, header_end;
  size_t counter, ints, vcore, jbuf, ovl, erep, gpair, H, P, F, C, W1, W2, eps, diis, grad, rot, res, total;
};

constexpr StaticLayout static_layout(size_t nat, size_t npair, size_t nao, size_t nint) {
  StaticLayout L{};
  size_t off = 0;
  const size_t np = npair > 0 ? npair : 1;
  const size_t mat = sizeof(double) * nao * nao;
  L.mols = off; off = al256(off + sizeof(MolDev));
  L.atoms = off; off = al256(off + sizeof(AtomDev) * nat);
  L.pairs = off; off = al256(off + sizeof(PairDev) * np);
  L.elems = off; off = al256(off + sizeof(ElemDev) * kMaxElementSlots);
  L.diat = off; off = al256(off + sizeof(DiatomicDev) * kMaxElementSlots * kMaxElementSlots);
  L.ao = off; off = al256(off + sizeof(int) * nao);
  L.order = off; off = al256(off + sizeof(int));
  L.hh = off; off = al256(off + sizeof(int) * np);
  L.header_end = off;
  L.counter = off; off = al256(off + sizeof(int));
  L.ints = off; off = al256(off + sizeof(double) * (nint > 0 ? nint : 1));
  L.vcore = off; off = al256(off + sizeof(double) * 20 * np);
  L.jbuf = off; off = al256(off + sizeof(double) * 20 * np);
  L.ovl = off; off = al256(off + sizeof(double) * 16 * np);
  L.erep = off; off = al256(off + sizeof(double) * np);
  L.gpair = off; off = al256(off + sizeof(double) * 3 * np);
  L.H = off; off = al256(off + mat);
  L.P = off; off = al256(off + mat);
  L.F = off; off = al256(off + mat);
  L.C = off; off = al256(off + mat);
  L.W1 = off; off = al256(off + mat);
  L.W2 = off; off = al256(off + mat);
  L.eps = off; off = al256(off + sizeof(double) * nao);
  L.diis = off; off = al256(off + sizeof(double) * 2 * kDiisMax * nao * nao);
  L.grad = off; off = al256(off + sizeof(double) * 3 * nat);
  L.rot = off; off = al256(off + kScfRotationBytesPerCta);  // recorded Jacobi rotations of the one SCF CTA
  L.res = off; off = al256(off + sizeof(MolResult));
  L.total = off;
  return L;
}

// Every buffer grows monotonically with the sizes, so the layout at the
// limits bounds every admissible molecule.
constexpr StaticLayout kMaxLayout =
    static_layout(kStaticMaxAtoms, kStaticMaxPairs, kStaticMaxAos, (size_t)kStaticMaxPairs * 100);
static_assert(kMaxLayout.total <= (size_t)SG_STATIC_SCRATCH_BYTES, "static scratch smaller than its layout");

// The device scratch (one per device context) and the host staging of the
// descriptor tables.
__device__ __align__(256) unsigned char g_static_scratch[SG_STATIC_SCRATCH_BYTES];
alignas(256) unsigned char g_host_header[al256(kMaxLayout.header_end)];

unsigned char* g_scratch_ptr[kMaxDevices];
LocalTermTable g_static_terms;
bool g_static_terms_built = false;

void set_error(char* buf, int cap, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
void set_error(char* buf, int cap, const char* fmt, ...) {
  if (!buf || cap <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, (size_t)cap, fmt, ap);
  va_end(ap);
}

bool parse_method_cstr(const char* s, Method& m) {
  if (!s) return false;
  char t[8];
  size_t n = std::strlen(s);
  if (n == 0 || n >= sizeof(t)) return false;
  for (size_t i = 0; i <= n; ++i) t[i] = (char)std::toupper((unsigned char)s[i]);
  if (!std::strcmp(t, "MNDO")) m = kMNDO;
  else if (!std::strcmp(t, "AM1")) m = kAM1;
  else if (!std::strcmp(t, "PM6")) m = kPM6;
  else return false;
  return true;
}

}  // namespace
}  // namespace sgb

extern "C" int32_t sg_calculate_static(const char* method, int32_t n_atoms, const int32_t* atomic_numbers,
                                       const double* xyz_bohr, int32_t charge, double self_consistence_criterion,
                                       double density_rmsd_criterion, int32_t max_scf_iterations,
                                       uint32_t properties, void* stream, double* energy, double* gradients,
                                       int32_t* iterations, int32_t* converged, char* error_message,
                                       int32_t error_capacity) {
  using namespace sgb;
  if (error_message && error_capacity > 0) error_message[0] = 0;
  Method m;
  if (!parse_method_cstr(method, m)) {
    set_error(error_message, error_capacity, "unknown method '%s' (MNDO, AM1, PM6)", method ? method : "(null)");
    return SG_ERR_UNKNOWN_METHOD;
  }
  if (n_atoms <= 0 || !atomic_numbers || !xyz_bohr) {
    set_error(error_message, error_capacity, "empty molecular structure");
    return SG_ERR_EMPTY_STRUCTURE;
  }
  if (n_atoms > kStaticMaxAtoms) {
    set_error(error_message, error_capacity, "%d atoms exceed the allocation-free limit of %d atoms", (int)n_atoms,
              kStaticMaxAtoms);
    return SG_ERR_INVALID_ARGUMENT;
  }
  if (!(self_consistence_criterion > 0) || !(density_rmsd_criterion > 0) || max_scf_iterations < 1) {
    set_error(error_message, error_capacity, "SCF criteria must be positive and the iteration limit at least 1");
    return SG_ERR_INVALID_ARGUMENT;
  }
  if ((properties & SG_PROP_GRADIENTS) && !gradients) {
    set_error(error_message, error_capacity, "gradients requested without an output buffer");
    return SG_ERR_INVALID_ARGUMENT;
  }

  // ---- descriptor tables in the host staging array ----
  int slot_Z[kMaxElementSlots];
  int n_slots = 0;
  int atom_slot[kStaticMaxAtoms];
  ElemDev elems[kMaxElementSlots];
  int nao = 0;
  double ncore = 0;
  for (int a = 0; a < n_atoms; ++a) {
    const int z = atomic_numbers[a];
    int s = -1;
    for (int k = 0; k < n_slots; ++k)
      if (slot_Z[k] == z) s = k;
    if (s < 0) {
      if (engine_n_aos(m, z) == 0) {
        set_error(error_message, error_capacity, "no %s s/p parameters for element Z=%d", method_name(m), z);
        return SG_ERR_UNSUPPORTED_ELEMENT;
      }
      std::string unused;  // stays empty: make_elem only writes it for elements rejected above
      if (n_slots >= kMaxElementSlots || !make_elem(m, z, elems[n_slots], unused)) {
        set_error(error_message, error_capacity, "element Z=%d cannot be set up", z);
        return SG_ERR_UNSUPPORTED_ELEMENT;
      }
      slot_Z[n_slots] = z;
      s = n_slots++;
    }
    atom_slot[a] = s;
    nao += elems[s].nao;
    ncore += elems[s].core;
  }
  if (nao > kStaticMaxAos) {
    set_error(error_message, error_capacity, "%d AOs exceed the allocation-free limit of %d AOs", nao, kStaticMaxAos);
    return SG_ERR_INVALID_ARGUMENT;
  }
  // 64-bit count: any int charge is range-checked before it sizes the occupied block
  const long long nel_ll = std::llround(ncore) - (long long)charge;
  if (nel_ll < 0 || (nel_ll & 1) || nel_ll / 2 > nao) {
    set_error(error_message, error_capacity,
              "%lld electrons in %d orbitals: the restricted closed-shell SCF needs an even, non-negative count of "
              "at most two per orbital", nel_ll, nao);
    return SG_ERR_ODD_ELECTRONS;
  }
  const int nel = (int)nel_ll;
  DiatomicDev diat[kMaxElementSlots * kMaxElementSlots];
  for (int i = 0; i < kMaxElementSlots * kMaxElementSlots; ++i) diat[i] = DiatomicDev();
  for (int i = 0; i < n_slots; ++i)
    for (int j = 0; j < n_slots; ++j) {
      const DiatomicDev d = make_diatomic(m, slot_Z[i], slot_Z[j]);
      if (m == kPM6 && !d.present) {
        set_error(error_message, error_capacity, "no PM6 diatomic parameters for the element pair Z=%d, Z=%d",
                  slot_Z[i], slot_Z[j]);
        return SG_ERR_UNSUPPORTED_ELEMENT;
      }
      diat[i * kMaxElementSlots + j] = d;
    }
  const int npairs = n_atoms * (n_atoms - 1) / 2;
  long long nint = 0;
  for (int a = 0; a < n_atoms; ++a)
    for (int b = a + 1; b < n_atoms; ++b)
      nint += (elems[atom_slot[a]].nao == 1 ? 1 : 10) * (elems[atom_slot[b]].nao == 1 ? 1 : 10);
  const StaticLayout L = static_layout(n_atoms, npairs, nao, (size_t)nint);

  unsigned char* h = g_host_header;
  std::memset(h, 0, L.header_end);
  MolDev md{};
  md.nat = n_atoms;
  md.nao = nao;
  md.nel = nel;
  md.nocc = nel / 2;
  md.npairs = npairs;
  AtomDev* atoms = reinterpret_cast<AtomDev*>(h + L.atoms);
  int* ao_atom = reinterpret_cast<int*>(h + L.ao);
  for (int a = 0, ao = 0; a < n_atoms; ++a) {
    AtomDev ad{};
    ad.x = xyz_bohr[3 * a];
    ad.y = xyz_bohr[3 * a + 1];
    ad.z = xyz_bohr[3 * a + 2];
    if (!std::isfinite(ad.x) || !std::isfinite(ad.y) || !std::isfinite(ad.z)) {
      set_error(error_message, error_capacity, "non-finite position of atom %d", a);
      return SG_ERR_INVALID_ARGUMENT;
    }
    ad.slot = atom_slot[a];
    ad.ao0 = ao;
    atoms[a] = ad;
    for (int k = 0; k < elems[atom_slot[a]].nao; ++k) ao_atom[ao++] = a;
  }
  PairDev* pairs = reinterpret_cast<PairDev*>(h + L.pairs);
  int* hh = reinterpret_cast<int*>(h + L.hh);
  long long off = 0;
  int k = 0, nhh = 0;
  for (int a = 0; a < n_atoms; ++a)
    for (int b = a + 1; b < n_atoms; ++b, ++k) {
      const double dx = atoms[b].x - atoms[a].x, dy = atoms[b].y - atoms[a].y, dz = atoms[b].z - atoms[a].z;
      if (dx * dx + dy * dy + dz * dz < 1e-12) {
        set_error(error_message, error_capacity, "atoms %d and %d coincide", a, b);
        return SG_ERR_INVALID_ARGUMENT;
      }
      const int na = elems[atom_slot[a]].nao, nb = elems[atom_slot[b]].nao;
      pairs[k] = PairDev{a, b, 0, (int)off};
      off += (na == 1 ? 1 : 10) * (nb == 1 ? 1 : 10);
      if (na == 4 && nb == 4) hh[nhh++] = k;
    }
  md.nhh = nhh;
  std::memcpy(h + L.mols, &md, sizeof(md));
  std::memcpy(h + L.elems, elems, sizeof(ElemDev) * n_slots);
  std::memcpy(h + L.diat, diat, sizeof(diat));
  // order[0] = 0 is already zero

  // ---- once-per-device set-up ----
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error(error_message, error_capacity, "no usable CUDA device: %s",
              e != cudaSuccess ? cudaGetErrorString(e) : "device index out of range");
    return SG_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The scratch address is looked up on every call (a host-side table lookup
  // after the first) and compared with the cached one, and the constant
  // multipole table (a few KB) is uploaded on every call: after a
  // cudaDeviceReset the next call sees the new context's address and refills
  // its constant memory instead of using a stale pointer or an empty table.
  {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      set_error(error_message, error_capacity, "cudaGetSymbolAddress of the static scratch failed: %s",
                cudaGetErrorString(e));
      return SG_ERR_CUDA;
    }
    if (!g_static_terms_built) {
      build_local_term_table(g_static_terms);
      g_static_terms_built = true;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  upload_local_terms(g_static_terms, s);
  unsigned char* base = g_scratch_ptr[dev];

  DeviceBatch d;
  d.method = m;
  d.nmol = 1;
  d.natoms = n_atoms;
  d.npairs = npairs;
  d.nhh_total = nhh;
  d.nao_total = nao;
  d.mat_total = (long long)nao * nao;
  d.diis_total = 2LL * kDiisMax * nao * nao;
  d.int_total = nint;
  d.max_nao = nao;
  d.mols = reinterpret_cast<MolDev*>(base + L.mols);
  d.atoms = reinterpret_cast<AtomDev*>(base + L.atoms);
  d.pairs = reinterpret_cast<PairDev*>(base + L.pairs);
  d.elems = reinterpret_cast<ElemDev*>(base + L.elems);
  d.diat = reinterpret_cast<DiatomicDev*>(base + L.diat);
  d.ao_atom = reinterpret_cast<int*>(base + L.ao);
  d.order = reinterpret_cast<int*>(base + L.order);
  d.hh_pairs = reinterpret_cast<int*>(base + L.hh);
  d.counter = reinterpret_cast<int*>(base + L.counter);
  d.ints = reinterpret_cast<double*>(base + L.ints);
  d.vcore = reinterpret_cast<double*>(base + L.vcore);
  d.jbuf = reinterpret_cast<double*>(base + L.jbuf);
  d.ovl = reinterpret_cast<double*>(base + L.ovl);
  d.erep = reinterpret_cast<double*>(base + L.erep);
  d.gpair = reinterpret_cast<double*>(base + L.gpair);
  d.H = reinterpret_cast<double*>(base + L.H);
  d.P = reinterpret_cast<double*>(base + L.P);
  d.F = reinterpret_cast<double*>(base + L.F);
  d.C = reinterpret_cast<double*>(base + L.C);
  d.W1 = reinterpret_cast<double*>(base + L.W1);
  d.W2 = reinterpret_cast<double*>(base + L.W2);
  d.eps = reinterpret_cast<double*>(base + L.eps);
  d.diis = reinterpret_cast<double*>(base + L.diis);
  d.grad = reinterpret_cast<double*>(base + L.grad);
  d.rotbuf = reinterpret_cast<double*>(base + L.rot);
  d.scf_grid = 1;
  d.res = reinterpret_cast<MolResult*>(base + L.res);
  d.use_guess = 1;

  ScfParams sp;
  sp.scc = self_consistence_criterion;
  sp.rmsd = density_rmsd_criterion;
  sp.max_iter = max_scf_iterations;

  // ---- upload, clear, launch, read back (all on the caller's stream) ----
  e = cudaMemcpyAsync(base, h, L.header_end, cudaMemcpyHostToDevice, s);
  // the result record starts at zero (the SCF kernel fills it; the counter is
  // cleared by the SCF launcher)
  if (e == cudaSuccess) e = cudaMemsetAsync(d.res, 0, sizeof(MolResult), s);
  if (e != cudaSuccess) {
    set_error(error_message, error_capacity, "upload failed: %s", cudaGetErrorString(e));
    return SG_ERR_CUDA;
  }
  launch_pair_values(d, s);
  launch_one_electron(d, s);
  launch_scf(d, sp, 1, s);
  const bool want_grad = (properties & SG_PROP_GRADIENTS) != 0;
  if (want_grad) launch_gradient(d, s);
  e = cudaGetLastError();
  MolResult r;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&r, d.res, sizeof(MolResult), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && want_grad)
    e = cudaMemcpyAsync(gradients, d.grad, sizeof(double) * 3 * n_atoms, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(error_message, error_capacity, "device run failed: %s", cudaGetErrorString(e));
    return SG_ERR_CUDA;
  }
  if (energy) *energy = r.energy;
  if (iterations) *iterations = r.iterations;
  if (converged) *converged = r.converged;
  if (r.status != kDevOk) {
    set_error(error_message, error_capacity, "device SCF failure code %d", r.status);
    return SG_ERR_DEVICE;
  }
  if (!r.converged) {
    set_error(error_message, error_capacity, "SCF not converged in %d iterations", r.iterations);
    return SG_ERR_NOT_CONVERGED;
  }
  return SG_OK;
}
