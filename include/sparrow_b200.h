/*
 * sparrow_b200 C-ABI: batched NDDO (MNDO / AM1 / PM6) single points on one
 * NVIDIA B200 (sm_100a), energy and nuclear gradient.
 *
 * Every entry point returns an int32 status (SG_OK = 0) and copies caller
 * buffers in or out; no pointer into engine memory escapes.  Units: positions
 * in bohr, energies in Hartree, gradients in Hartree/bohr.  A handle is not
 * thread-safe; independent handles may be used from different threads.
 *
 * The entry points replace the reference's Core::Calculator surface as
 * implemented by GenericMethodWrapper / NDDOMethodWrapper (qcscine/sparrow,
 * paths relative to src/Sparrow/Sparrow/):
 *   sg_create                 SparrowModule.cpp:29-49 (ModuleManager::get("calculator", "PM6"))
 *   sg_set_structure          Implementations/GenericMethodWrapper.cpp:101-107 (setStructure)
 *   sg_modify_positions       Implementations/GenericMethodWrapper.h:51-134 (modifyPositions)
 *   sg_get_positions          Implementations/GenericMethodWrapper.h:51-134 (getPositions)
 *   sg_set_setting_*          Implementations/Nddo/NDDOMethodWrapper.cpp:68-103 (settings())
 *   sg_set_required_properties Implementations/GenericMethodWrapper.h:51-134 (setRequiredProperties)
 *   sg_calculate              Implementations/GenericMethodWrapper.cpp:58-99 (calculate)
 *   sg_get_energy / sg_get_gradients / sg_get_scf_info
 *                             Implementations/GenericMethodWrapper.cpp:175-262 (results())
 *   sg_get_density / sg_set_density
 *                             Implementations/GenericMethodWrapper.cpp:268-282 (getState/loadState)
 *   sg_get_orbital_energies   results() OrbitalEnergies
 *   sg_get_beta_orbital_energies  results() OrbitalEnergies (beta, unrestricted)
 *   sg_get_hessian            results() Hessian (GenericMethodWrapper.cpp:58-88: semi-numerical)
 *   sg_get_atomic_charges     results() AtomicCharges (GenericMethodWrapper.cpp:212-214)
 *   sg_get_dipole             results() Dipole (GenericMethodWrapper.cpp:89-92)
 *   sg_get_spin_densities / sg_set_spin_densities
 *                             getState / loadState of an unrestricted calculation
 *   sg_clone                  Implementations/Nddo/Pm6/Wrapper/PM6MethodWrapper.cpp:38-45 (clone)
 * The batch entry points (sg_batch_*) have no counterpart in the reference:
 * they run many independent molecules through one device launch sequence.
 */
#ifndef SPARROW_B200_H
#define SPARROW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SG_OK 0
#define SG_ERR_INVALID_ARGUMENT 1
#define SG_ERR_UNKNOWN_METHOD 2
#define SG_ERR_UNSUPPORTED_ELEMENT 3
#define SG_ERR_EMPTY_STRUCTURE 4
#define SG_ERR_ODD_ELECTRONS 5
#define SG_ERR_NOT_CONVERGED 6 /* informational: results are still available */
#define SG_ERR_CUDA 7
#define SG_ERR_OUT_OF_MEMORY 8
#define SG_ERR_NO_RESULTS 9
#define SG_ERR_UNKNOWN_SETTING 10
#define SG_ERR_DEVICE 11
#define SG_ERR_TIMEOUT 12
#define SG_PENDING 13 /* sg_server_poll: the request is still in flight */
#define SG_ERR_PARAMETERS 14 /* a parameter file is missing or malformed */

/* required-property mask */
#define SG_PROP_ENERGY 1u
#define SG_PROP_GRADIENTS 2u
#define SG_PROP_HESSIAN 4u /* semi-numerical: central differences of analytic gradients */
#define SG_PROP_ATOMIC_CHARGES 8u
#define SG_PROP_DIPOLE 16u

typedef struct sg_calculator sg_calculator;
typedef struct sg_batch sg_batch;

/* version string of the library */
const char* sg_version(void);

/* ---- single-structure calculator (Core::Calculator surface) ---- */
int32_t sg_create(const char* method, sg_calculator** out);
void sg_destroy(sg_calculator* h);
int32_t sg_clone(const sg_calculator* h, sg_calculator** out);
const char* sg_last_error(const sg_calculator* h);

int32_t sg_set_structure(sg_calculator* h, int32_t n_atoms, const int32_t* atomic_numbers, const double* xyz_bohr);
int32_t sg_modify_positions(sg_calculator* h, const double* xyz_bohr);
int32_t sg_get_positions(const sg_calculator* h, double* xyz_bohr);
int32_t sg_get_n_atoms(const sg_calculator* h, int32_t* n_atoms);

/* Settings keys follow the reference: "molecular_charge", "spin_multiplicity",
 * "spin_mode", "self_consistence_criterion", "density_rmsd_criterion",
 * "max_scf_iterations", "scf_mixer", "method_parameters", and one of this
 * engine: "scf_path" = "auto" | "batched" | "large" | "large_mixed" (see
 * sg_batch_set_scf_path).
 * "method_parameters" (empty = the embedded default) is read at sg_calculate,
 * as the reference's method wrappers read it at initialize()
 * (Implementations/Nddo/Pm6/Wrapper/PM6MethodWrapper.cpp:62-75,
 * Implementations/Dftb/Utils/DFTBCommon.cpp:112-120): for MNDO / AM1 / PM6 the
 * path of a parameters.json file in the layout of Nddo/Parameters.cpp:76-93;
 * for DFTB2 / DFTB3 an embedded set name (mio-1-1, 3ob-3-1, 3ob-2-1) or a
 * directory of Slater-Koster files X-Y.skf with optional hubbard.dat and
 * spin.dat (Dftb/ParameterSet.cpp:69-133).  A missing or malformed file makes
 * sg_calculate return SG_ERR_PARAMETERS. */
int32_t sg_set_setting_int(sg_calculator* h, const char* key, int64_t value);
int32_t sg_set_setting_double(sg_calculator* h, const char* key, double value);
int32_t sg_set_setting_string(sg_calculator* h, const char* key, const char* value);
int32_t sg_get_setting_double(const sg_calculator* h, const char* key, double* value);
int32_t sg_get_setting_int(const sg_calculator* h, const char* key, int64_t* value);

int32_t sg_set_required_properties(sg_calculator* h, uint32_t mask);
/* Returns SG_OK, SG_ERR_NOT_CONVERGED (energy still set, like the reference's
 * SuccessfulCalculation = false) or an error. */
int32_t sg_calculate(sg_calculator* h);
int32_t sg_get_energy(const sg_calculator* h, double* energy);
int32_t sg_get_gradients(const sg_calculator* h, double* gradients);
int32_t sg_get_scf_info(const sg_calculator* h, int32_t* iterations, int32_t* converged, int32_t* n_aos,
                        int32_t* n_occupied);
/* Orbital energies (n_aos); SG_ERR_NO_RESULTS after a calculation on the
 * large-molecule path ("scf_path" large / large_mixed, or automatic above 1024
 * AOs), which purifies the density and computes no orbitals. */
int32_t sg_get_orbital_energies(const sg_calculator* h, double* eps);
/* density matrix (n_aos x n_aos, row-major) of the last calculation, and a
 * start density for the next one (warm start) */
/* Linear-response TD-DFTB on the converged DFTB2 / DFTB3 reference of the
 * last sg_calculate (replaces TDDFTBCalculator::calculate,
 * Implementations/Dftb/TimeDependent/LinearResponse/TDDFTBCalculator.cpp:124-158,
 * restricted singlets or triplets, full TD-DFTB, no basis pruning): the
 * nroots (1..16) lowest excitation energies omega (Hartree, ascending) and,
 * for singlets, the transition dipoles (nroots x 3, e bohr; zero for
 * triplets; dipoles may be NULL).  SG_ERR_NOT_CONVERGED when the Davidson
 * solver did not reach its residual tolerance (1e-10 on the Casida matrix). */
int32_t sg_calculate_excitations(sg_calculator* h, int32_t nroots, int32_t triplet, double* omega, double* dipoles);
/* Unrestricted calculations ("spin_mode" = "unrestricted", or "any" with
 * "spin_multiplicity" != 1, as NDDOMethodWrapper.cpp:68-92): the beta orbital
 * energies (N values; sg_get_orbital_energies gives the alpha ones).
 * SG_ERR_NO_RESULTS after a restricted calculation. */
int32_t sg_get_beta_orbital_energies(const sg_calculator* h, double* eps);
/* Unrestricted state (getState / loadState with spin-resolved densities,
 * GenericMethodWrapper.cpp:268-282): the alpha and beta densities (N x N
 * each) of the last calculate(), and start spin densities for the next one
 * (their sum also replaces the sg_set_density state). */
int32_t sg_get_spin_densities(const sg_calculator* h, double* alpha, double* beta);
int32_t sg_set_spin_densities(sg_calculator* h, const double* alpha, const double* beta);
/* Hessian (3 n_atoms x 3 n_atoms row-major, Hartree/bohr^2) of the last
 * calculate() with SG_PROP_HESSIAN required.  Like the reference, which has no
 * analytic Hessian (GenericMethodWrapper.cpp:58-88, 339-341), it is the
 * symmetrised central difference of analytic gradients with a 0.01 bohr
 * step; the 6 n_atoms displaced geometries run as one batch. */
int32_t sg_get_hessian(const sg_calculator* h, double* hessian);
/* Atomic charges (n_atoms) of the last calculate() with SG_PROP_ATOMIC_CHARGES
 * required (results().AtomicCharges, GenericMethodWrapper.cpp:212-214): DFTB
 * the SCC's Mulliken charges, NDDO the core charge minus the atom's diagonal
 * density (Mulliken charges in the orthogonal NDDO basis). */
int32_t sg_get_atomic_charges(const sg_calculator* h, double* charges);
/* Dipole moment (x, y, z in e bohr) of the last calculate() with
 * SG_PROP_DIPOLE required: DFTB sum_a q_a R_a with the Mulliken charges
 * (Dftb/Utils/DipoleUtils/DFTBDipoleMomentCalculator.cpp:23-35); NDDO in the
 * NDDO approximation about the centre of mass, sum_a q_a (R_a - R_cm) -
 * 2 D_sp1 P_{s,p} per s/p atom (Nddo/Utils/DipoleUtils/NDDODipoleMomentCalculator.cpp:76-110). */
int32_t sg_get_dipole(const sg_calculator* h, double* dipole3);
/* One call: the same Hessian for one molecule (method spec as for
 * sg_batch_create; unrestricted != 0 or multiplicity != 1 runs the
 * unrestricted SCF; step <= 0 takes 0.01 bohr).  not_converged (may be NULL)
 * receives the number of displaced geometries whose SCF did not converge. */
int32_t sg_calculate_hessian(const char* method, int32_t n_atoms, const int32_t* atomic_numbers,
                             const double* xyz_bohr, int32_t charge, int32_t multiplicity, int32_t unrestricted,
                             double self_consistence_criterion, double density_rmsd_criterion,
                             int32_t max_iterations, double step, double* hessian, int32_t* not_converged,
                             char* error_message, int32_t error_capacity);
int32_t sg_get_density(const sg_calculator* h, double* P);
int32_t sg_set_density(sg_calculator* h, const double* P);

/* ---- parameter queries (host only, no device use) ---- */
/* Runtime (atomic-unit) parameters of element Z under a method spec as for
 * sg_batch_create, as the engine uploads them.
 * NDDO, SG_NDDO_ELEMENT_VALUES doubles: nao, core charge, U_ss, U_pp, beta_s,
 *   beta_p, alpha, D_sp1, D_pp2, rho_ss0, rho_sp1, rho_pp0, rho_pp2, pcore,
 *   g_ss, g_sp, g_pp, g_p2, h_sp, h_pp, STO-6G s exponents[6], s coefficients[6],
 *   p exponents[6], p coefficients[6], Gaussian term count, a[4], b[4], c[4]
 *   (RawParameterProcessor.cpp:67-188 of Implementations/Nddo/Utils/ParameterUtils).
 * DFTB, SG_DFTB_ELEMENT_VALUES doubles: nao, occupation, e_s, e_p, Hubbard U,
 *   Hubbard derivative, spin constant W, has W (Dftb/Utils/SKAtom.cpp:16-70).
 * Returns SG_ERR_PARAMETERS for an unreadable parameter source and
 * SG_ERR_UNSUPPORTED_ELEMENT when it has no s/p record for Z. */
#define SG_NDDO_ELEMENT_VALUES 57
#define SG_DFTB_ELEMENT_VALUES 8
int32_t sg_element_parameters(const char* method, int32_t Z, double* out, int32_t n_out, char* errmsg,
                              int32_t errcap);
/* PM6 diatomic core-repulsion pair (alpha_AB in 1/bohr, or 1/bohr^2 for X-H
 * with X in C, N, O; x_AB) under a method spec. */
int32_t sg_diatomic_parameters(const char* method, int32_t Z1, int32_t Z2, double* alpha_x, char* errmsg,
                               int32_t errcap);

/* ---- batches: many independent molecules per device launch sequence ---- */
/* Molecule i has n_atoms[i] atoms; atomic_numbers / xyz_bohr are the
 * concatenation over molecules; charges may be NULL (all neutral).  method is
 * "METHOD" or "METHOD:parameters" with parameters as for "method_parameters"
 * (e.g. "DFTB3:3ob-2-1", "PM6:/data/pm6.json"). */
int32_t sg_batch_create(const char* method, int32_t n_molecules, const int32_t* n_atoms,
                        const int32_t* atomic_numbers, const double* xyz_bohr, const int32_t* charges,
                        sg_batch** out);
/* Unrestricted (UHF) batch: molecule i has spin multiplicity multiplicities[i]
 * (NULL: all 1); MNDO / AM1 / PM6 on the batched path (at most 1024 AOs). */
int32_t sg_batch_create_unrestricted(const char* method, int32_t n_molecules, const int32_t* n_atoms,
                                     const int32_t* atomic_numbers, const double* xyz_bohr, const int32_t* charges,
                                     const int32_t* multiplicities, sg_batch** out);
void sg_batch_destroy(sg_batch* b);
const char* sg_batch_last_error(const sg_batch* b);
int32_t sg_batch_set_scf(sg_batch* b, double self_consistence_criterion, double density_rmsd_criterion,
                         int32_t max_scf_iterations);
/* SCF path: 0 automatic (a single NDDO molecule of more than 1024 AOs runs
 * the large-molecule path, everything else the batched persistent kernel),
 * 1 batched kernel, 2 large-molecule path in FP64 (grid-wide Fock build,
 * DIIS, SP2 purification on FP64 GEMMs), 3 large-molecule path with the SP2
 * products in split-BF16 on the tensor cores until rms(dP) < 1e-5, then FP64.
 * Paths 2 and 3 take a batch of one NDDO molecule.  On the large path the
 * scf_stats report iterations with mixed-precision purification as
 * full_diagonalisations and the SP2 steps as jacobi_sweeps. */
int32_t sg_batch_set_scf_path(sg_batch* b, int32_t path);
/* SCF path 3: rms(dP) below which the purification switches from split-BF16
 * to FP64 (default 1e-5; also when the mixed densities stop halving below
 * 1e-4) */
int32_t sg_batch_set_mixed_switch(sg_batch* b, double density_rmsd);
/* Tuning of the batched SCF (no counterpart in the reference, which
 * diagonalises through its SCF library every iteration).  The library
 * carries a table, measured by its autotuner (sparrow_b200/autotune.py), of
 * the orbital update and the Pulay subspace size per molecule-size bin of 32
 * AOs.  sg_batch_set_tuning overrides it for every molecule of the batch:
 * orbital_update one of SG_ORBITALS_EXACT (a full diagonalisation of the
 * extrapolated Fock matrix every iteration, Householder tridiagonal solver),
 * SG_ORBITALS_HYBRID (the tridiagonal solver at the start, then
 * occupied-virtual rotations), SG_ORBITALS_ROTATION (a Jacobi start, then
 * rotations), diis_size 1..6; -1 keeps the table's choice for that knob.
 * Every choice converges to the same fixed point.  sg_tuning_table writes
 * the table (capacity entries at most) and returns its number of bins. */
#define SG_ORBITALS_EXACT 0
#define SG_ORBITALS_HYBRID 1
#define SG_ORBITALS_ROTATION 2
int32_t sg_batch_set_tuning(sg_batch* b, int32_t orbital_update, int32_t diis_size);
int32_t sg_tuning_table(int32_t* orbital_update, int32_t* diis_size, int32_t capacity);
/* TD-DFTB of every molecule of a DFTB batch after sg_batch_run: omega
 * [n_molecules * nroots], dipoles [n_molecules * nroots * 3] (may be NULL),
 * status [n_molecules] (0 ok, 1 not converged, 2 orbital diagonalisation,
 * 3 non-positive eigenvalue, 4 reference not converged; may be NULL).  The
 * call overwrites the batch's orbital scratch; gradients of the preceding
 * run stay valid. */
int32_t sg_batch_excitations(sg_batch* b, int32_t nroots, int32_t triplet, double* omega, double* dipoles,
                             int32_t* status);
/* SM cycles per molecule of the last sg_batch_excitations: canonical
 * orbitals, transition charges, Davidson (3 per molecule) */
int32_t sg_batch_excitation_cycles(sg_batch* b, int64_t* cycles3);
int32_t sg_batch_set_positions(sg_batch* b, const double* xyz_bohr);
/* enqueue integrals -> SCF -> (gradient) on the device; asynchronous */
int32_t sg_batch_run(sg_batch* b, uint32_t properties);
/* wait and copy results: arrays of n_molecules (energies, iterations,
 * converged) and 3 * total atoms (gradients); any pointer may be NULL */
int32_t sg_batch_results(sg_batch* b, double* energies, double* gradients, int32_t* iterations, int32_t* converged);
/* number of device kernel launches issued by the last sg_batch_run */
int32_t sg_batch_launches(const sg_batch* b);
/* CUDA stream (cudaStream_t) the batch runs on */
void* sg_batch_stream(const sg_batch* b);
/* device milliseconds of the stages of the last run: pair integrals,
 * one-electron assembly, SCF, gradient (waits for the run to finish) */
int32_t sg_batch_stage_times(sg_batch* b, double* ms4);
/* timing events on the batch stream: record in slot 0..7, elapsed s0 -> s1 */
int32_t sg_batch_record_event(sg_batch* b, int32_t slot);
int32_t sg_batch_event_elapsed(sg_batch* b, int32_t slot0, int32_t slot1, double* ms);
/* per-molecule SCF diagnostics of the last run: full diagonalisations,
 * Jacobi sweeps, and SM cycles spent in the Fock build, DIIS, occupied-virtual
 * rotation, full diagonalisation and density phases (5 per molecule);
 * any pointer may be NULL */
int32_t sg_batch_scf_stats(sg_batch* b, int32_t* full_diagonalisations, int32_t* jacobi_sweeps, int64_t* cycles5);
/* per-molecule convergence measures of the last SCF iteration of the last
 * run: |E_it - E_it-1| (Hartree) and rms(P_it - P_it-1), the quantities that
 * the settings self_consistence_criterion and density_rmsd_criterion bound;
 * either pointer may be NULL */
int32_t sg_batch_convergence(sg_batch* b, double* last_delta_energy, double* last_rms_density_change);
/* bytes copied host->device and device->host by this batch so far */
int32_t sg_batch_transfer_bytes(const sg_batch* b, int64_t* h2d, int64_t* d2h);
/* free device and pinned host memory cached from destroyed batches */
void sg_release_cached_memory(void);

/* one call from host buffers to host results (create, run, fetch, destroy) */
int32_t sg_batch_calculate(const char* method, int32_t n_molecules, const int32_t* n_atoms,
                           const int32_t* atomic_numbers, const double* xyz_bohr, const int32_t* charges,
                           double self_consistence_criterion, double density_rmsd_criterion,
                           int32_t max_scf_iterations, uint32_t properties, double* energies, double* gradients,
                           int32_t* iterations, int32_t* converged, char* error_message, int32_t error_capacity);

/* ---- request server: continuous batching on one GPU ----
 *
 * No counterpart in the reference (its callers loop over Calculator
 * instances).  A worker thread keeps up to `slots` batches in flight, each on
 * its own stream; free slots are refilled at once with the oldest pending
 * requests of one method, admitted while the estimated device memory of all
 * in-flight batches stays within device_budget_bytes.  Submission validates
 * the request (elements, electron count, coincident atoms) and returns its
 * error at once.  Every function is thread-safe; destroy waits for the
 * requests in flight. */
typedef struct sg_server sg_server;
int32_t sg_server_create(uint64_t device_budget_bytes, int32_t slots, int32_t max_batch,
                         double self_consistence_criterion, double density_rmsd_criterion,
                         int32_t max_scf_iterations, sg_server** out);
void sg_server_destroy(sg_server* s);
/* thread-local text of the last error of a server call on this thread */
const char* sg_server_last_error(void);
int32_t sg_server_submit(sg_server* s, const char* method, int32_t n_atoms, const int32_t* atomic_numbers,
                         const double* xyz_bohr, int32_t charge, uint32_t properties, int64_t* request_id);
/* As sg_server_submit with a spin multiplicity: != 1 runs the unrestricted
 * SCF (the reference's spin mode "any"); batches never mix spin treatments. */
int32_t sg_server_submit_spin(sg_server* s, const char* method, int32_t n_atoms, const int32_t* atomic_numbers,
                              const double* xyz_bohr, int32_t charge, int32_t multiplicity, uint32_t properties,
                              int64_t* request_id);
/* Wait up to timeout_s (< 0: forever) for a request.  Returns SG_OK when the
 * request is finished (its own status in *status: SG_OK, SG_ERR_NOT_CONVERGED
 * with results, or an error), SG_ERR_TIMEOUT, or SG_ERR_INVALID_ARGUMENT for
 * an unknown id.  gradients (3 * n_atoms) is written when requested and
 * non-NULL; latency_s = completion - submission (seconds). */
int32_t sg_server_wait(sg_server* s, int64_t request_id, double timeout_s, double* energy, double* gradients,
                       int32_t* iterations, int32_t* status, double* latency_s);
/* As sg_server_wait without blocking: SG_PENDING while in flight. */
int32_t sg_server_poll(sg_server* s, int64_t request_id, double* energy, double* gradients, int32_t* iterations,
                       int32_t* status, double* latency_s);
/* Block until every submitted request has finished. */
int32_t sg_server_drain(sg_server* s);
/* counters: submitted, completed, batches launched, largest batch */
int32_t sg_server_stats(sg_server* s, int64_t* submitted, int64_t* completed, int64_t* batches, int64_t* max_batch);

/* ---- allocation-free single-molecule call ----
 *
 * No counterpart in the reference.  Energy (and gradient) of one closed-shell
 * molecule with every device buffer in one fixed device array of
 * SG_STATIC_SCRATCH_BYTES (per device context) and every host table in a
 * fixed host array: the call performs no device or pinned allocation.
 * Limits: SG_STATIC_MAX_ATOMS atoms and SG_STATIC_MAX_AOS AOs; larger
 * molecules return SG_ERR_INVALID_ARGUMENT with a message.
 * The first call on a device (with that device current) does the set-up: it
 * looks the scratch array up with cudaGetSymbolAddress; make that first call
 * before any stream capture begins.  Every call repeats that lookup, copies
 * the constant multipole table and the molecule's descriptors from pageable
 * host memory, and synchronises the stream before it returns, so a
 * cudaDeviceReset between calls is safe.  Calls that overlap in time share
 * the scratch and race: serialise them.  stream is a cudaStream_t (NULL = the
 * default stream).  The electron count must be even and fit the orbitals
 * (SG_ERR_ODD_ELECTRONS otherwise, before any device work).
 * Status codes as for sg_batch_results (SG_ERR_NOT_CONVERGED still fills the
 * outputs). */
#define SG_STATIC_MAX_ATOMS 64
#define SG_STATIC_MAX_AOS 256
#define SG_STATIC_SCRATCH_BYTES (14u * 1024u * 1024u)
int32_t sg_calculate_static(const char* method, int32_t n_atoms, const int32_t* atomic_numbers,
                            const double* xyz_bohr, int32_t charge, double self_consistence_criterion,
                            double density_rmsd_criterion, int32_t max_scf_iterations, uint32_t properties,
                            void* stream, double* energy, double* gradients, int32_t* iterations, int32_t* converged,
                            char* error_message, int32_t error_capacity);

#ifdef __cplusplus
}
#endif

#endif /* SPARROW_B200_H */
