/*
 * pm7_b200.h — C ABI of the B200 PM7/NDDO molecular SCF engine.
 *
 * This boundary replaces the Rust entry point of pm7-rs
 *
 *     pub fn run_pm7(molecule: &Molecule, params: &Pm7Parameters,
 *                    options: &Pm7Options) -> Result<Pm7Result>        (src/scf.rs:512-522)
 *
 * with plain pointers and sizes: no Rust or torch types cross it. A Rust
 * host binds it with a small `extern "C"` block (cgo/JNI/ctypes work the
 * same way). All compute behind `pm7_run` runs on one CUDA device; the
 * library has no CPU fallback and returns PM7_ERR_CUDA when no device is
 * usable.
 *
 * Units follow the reference: positions in Bohr, energies in eV, heat of
 * formation in kcal/mol, dipoles in Debye. Dense matrices are row-major
 * nao x nao doubles. MO coefficients are stored with orbitals as COLUMNS,
 * exactly like the reference's `mo_coeff` Matrix (A = V diag(e) V^T).
 */
#ifndef PM7_B200_H
#define PM7_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes. One per `Pm7Error` variant (src/error.rs:8-30) plus the two
 * device-side failures this engine adds. */
typedef enum pm7_status {
  PM7_OK = 0,
  PM7_ERR_INVALID_INPUT = 1,      /* Pm7Error::InvalidInput / Parse      */
  PM7_ERR_MISSING_ELEMENT = 2,    /* Pm7Error::MissingElement(z)         */
  PM7_ERR_MISSING_PARAMETER = 3,  /* Pm7Error::MissingParameter          */
  PM7_ERR_UNSUPPORTED = 4,        /* Pm7Error::UnsupportedFeature        */
  PM7_ERR_LINEAR_ALGEBRA = 5,     /* Pm7Error::LinearAlgebra             */
  PM7_ERR_SCF_NOT_CONVERGED = 6,  /* Pm7Error::ScfNotConverged           */
  PM7_ERR_RESPONSE_FAILED = 7,    /* Pm7Error::ResponseFailed            */
  PM7_ERR_INSUFFICIENT_MEMORY = 8,/* Pm7Error::InsufficientMemory        */
  PM7_ERR_CUDA = 9,               /* CUDA runtime / library failure      */
  PM7_ERR_TIMEOUT = 10            /* a bounded device wait gave up       */
} pm7_status;

/* PM7 family (src/method.rs:8-15). */
typedef enum pm7_method {
  PM7_METHOD_PM7 = 0,
  PM7_METHOD_PM7_TS = 1,
  PM7_METHOD_PM7_SPARKLE = 2,
  PM7_METHOD_PM7_MINUS = 3,
  PM7_METHOD_PM7_HH = 4
} pm7_method;

/* SCF accelerator (src/scf.rs:25-34). */
typedef enum pm7_accelerator {
  PM7_ACCEL_NONE = 0,
  PM7_ACCEL_CDIIS = 1,
  PM7_ACCEL_ADIIS_CDIIS = 2
} pm7_accelerator;

/* Spin treatment (src/scf.rs:38-47). */
typedef enum pm7_reference {
  PM7_REF_AUTO = 0,
  PM7_REF_RESTRICTED = 1,
  PM7_REF_UNRESTRICTED = 2
} pm7_reference;

/* Dipole origin for charged molecules (src/dipole.rs DipoleOrigin). */
typedef enum pm7_dipole_origin {
  PM7_DIPOLE_COORDINATES = 0,
  PM7_DIPOLE_CENTRE_OF_MASS = 1,
  PM7_DIPOLE_CENTRE_OF_CHARGE = 2
} pm7_dipole_origin;

/* Arithmetic of the SCF cycles. FP64 is the plain path; MIXED computes the early
 * cycles' densities (SP2 squarings) and, on the plain path, their DIIS commutator product
 * at FP32 accuracy on the tcgen05 tensor cores (3xTF32, FP32 accumulation), builds their Fock
 * matrices in FP32 while the DIIS error is above 10 eV, and re-converges in FP64 cycles, the
 * only ones that may end the SCF (engine knob; no reference analogue). */
typedef enum pm7_precision {
  PM7_PRECISION_FP64 = 0,
  PM7_PRECISION_MIXED = 1
} pm7_precision;

/* `Molecule` (src/system.rs:21-39): atomic numbers and positions in Bohr.
 * The net charge is NOT read from here: like the reference, `run_pm7` takes
 * charge and multiplicity from the options (src/scf.rs:588-607). */
typedef struct pm7_molecule {
  int32_t n_atoms;
  const uint8_t *z;        /* n_atoms atomic numbers                */
  const double *xyz_bohr;  /* 3*n_atoms, x0 y0 z0 x1 ...            */
} pm7_molecule;

/* `Pm7Options` molecular fields (src/scf.rs:73-188), defaults at
 * src/scf.rs:207-233 via pm7_options_default(). Periodic, field and
 * stability options of the reference are outside this engine's scope. */
typedef struct pm7_options {
  int32_t method;             /* pm7_method, must equal the parameter set's */
  double charge;
  int32_t multiplicity;
  int32_t max_scf;            /* 200    */
  double e_tol;               /* 1e-8 eV */
  double p_tol;               /* 1e-7   */
  int32_t use_diis;           /* 1      */
  int32_t accelerator;        /* pm7_accelerator, ADIIS_CDIIS */
  double adiis_switch;        /* 0.1    */
  double level_shift;         /* 0.0 eV */
  int32_t reference;          /* pm7_reference, AUTO */
  int32_t force_dpath;        /* 0      */
  int32_t smooth_dispersion;  /* 0      */
  int64_t max_memory_mb;      /* <0: no explicit budget (PM7_MEM_BUDGET_MB, then device memory) */
  int32_t dipole_origin;      /* pm7_dipole_origin, CENTRE_OF_MASS */
  const double *initial_density;      /* NULL or nao*nao */
  const double *initial_spin_density; /* NULL or nao*nao (UHF only) */
  /* engine knobs (no reference analogue) */
  int32_t precision;          /* pm7_precision, FP64 */
  int32_t device;             /* CUDA device ordinal, 0 */
  int32_t want_matrices;      /* 1: fill density/mo arrays in the result */
} pm7_options;

/* `Pm7Result` molecular fields (src/scf.rs:261-342). Arrays are owned by the
 * library and released by pm7_result_free(). Absent optionals are NaN
 * (scalars) or NULL (arrays). */
typedef struct pm7_result {
  int32_t n_atoms;
  int32_t nao;
  int32_t n_occ;
  int32_t n_occ_beta;        /* -1 for RHF */
  int32_t unrestricted;
  int32_t iterations;
  int32_t converged;
  double density_error;
  double electronic_ev;
  double core_ev;
  double total_ev;
  double heat_of_formation_kcal;
  double correction_kcal;    /* dispersion + H-bond + MM terms inside total/dHf */
  double homo_ev, lumo_ev, homo_ev_beta, lumo_ev_beta;
  double dipole_debye[3];
  double dipole_magnitude;
  double dipole_point_charge[3];
  double dipole_sp_hybrid[3];
  double dipole_pd_hybrid[3];
  double *charges;            /* n_atoms Mulliken net charges */
  double *density;            /* nao*nao total density           (want_matrices) */
  double *spin_density;       /* nao*nao P_alpha - P_beta, UHF   (want_matrices) */
  double *mo_energies;        /* nao, alpha (or spatial) set, ascending */
  double *mo_coeff;           /* nao*nao, columns are orbitals   (want_matrices) */
  double *mo_energies_beta;   /* nao, UHF */
  double *mo_coeff_beta;      /* nao*nao, UHF                    (want_matrices) */
  /* engine diagnostics */
  double device_ms;           /* wall time of the device SCF, ms */
  int32_t fp32_iterations;    /* cycles run in FP32 (MIXED) */
} pm7_result;

/* Opaque parameter set (`Pm7Parameters`, src/params.rs:104-111), parsed and
 * derived once per method and cached for the process like the reference's
 * OnceLock (src/params.rs:139-155). */
typedef struct pm7_params pm7_params;

/* Replaces `Pm7Parameters::method` (src/params.rs:127-129). The returned
 * pointer is process-global and must not be freed. */
pm7_status pm7_params_load(int32_t method, const pm7_params **out);

/* Fill `Pm7Options::default()` (src/scf.rs:207-233). */
void pm7_options_default(pm7_options *options);

/* Replaces `run_pm7` (src/scf.rs:512-522). On PM7_OK `*result` is filled and
 * must be released with pm7_result_free(). A non-converged SCF returns
 * PM7_ERR_SCF_NOT_CONVERGED with only `iterations` and `density_error` set,
 * mirroring the reference's error-with-no-result (src/scf.rs:770-775). */
pm7_status pm7_run(const pm7_molecule *molecule, const pm7_params *params,
                   const pm7_options *options, pm7_result *result);

/* ---- nuclear gradient ------------------------------------------------------------
 * Hellmann-Feynman gradient dE/dR in eV/Bohr, laid out gradient[3*atom + axis]. */

/* Replaces `closed_form_gradient` (src/gradient.rs:500-561): runs the SCF exactly as
 * pm7_run does (`*result` filled on PM7_OK, same errors) and returns the gradient of
 * result->total_ev at the converged density: core-core, electronic pair terms (RHF, or the
 * spin-resolved UHF form of src/gradient.rs:1249-1350) and the post-SCF corrections
 * (:208-261). `forces` of the reference's GradientResult are -gradient; `max_gradient`
 * (may be NULL) receives the largest |component|. `gradient` holds 3 * n_atoms doubles. */
pm7_status pm7_gradient(const pm7_molecule *molecule, const pm7_params *params,
                        const pm7_options *options, pm7_result *result, double *gradient,
                        double *max_gradient);

/* pm7_run_batch (below) with each molecule's nuclear gradient, as pm7_gradient returns it:
 * gradients[i] points to 3 * molecules[i].n_atoms doubles, filled when statuses[i] is PM7_OK.
 * No counterpart in pm7-rs, whose optimiser and MD loops call closed_form_gradient one
 * molecule at a time (src/optimizer.rs:318). Batched molecules get their gradient at the
 * density the batch converged to; the others go through pm7_gradient. */
pm7_status pm7_run_batch_gradient(int32_t n_molecules, const pm7_molecule *molecules,
                                  const pm7_params *params, const pm7_options *options,
                                  pm7_result *results, pm7_status *statuses, double *const *gradients);

/* Replaces `fixed_density_gradient_with` (src/gradient.rs:638-700) and, with a spin
 * density, `fixed_density_gradient_uhf_with` (:1263-1350): core-core plus electronic
 * gradient at a given density, no corrections. `p_total` (nao^2, row-major) is the total
 * density; `p_spin` is P_alpha - P_beta, or NULL for a closed shell. Host buffers; device 0. */
pm7_status pm7_fixed_density_gradient(const pm7_molecule *molecule, const pm7_params *params,
                                      int32_t force_dpath, const double *p_total,
                                      const double *p_spin, double *gradient);

/* Replaces `correction_gradient` (src/gradient.rs:208-261): the gradient of the post-SCF
 * corrections (dispersion, H-bond, C#C, Si-O-H, PM7-HH H-H) in eV/Bohr; zero for PM7-minus. */
pm7_status pm7_correction_gradient(const pm7_molecule *molecule, int32_t method,
                                   int32_t smooth_dispersion, double *gradient);

/* Release the arrays of a result filled by pm7_run (or the engine). */
void pm7_result_free(pm7_result *result);

/* Message of the last error on the calling thread (`Pm7Error` Display,
 * src/error.rs:32-60). Never NULL. */
const char *pm7_last_error_message(void);

/* Number of CUDA devices the library can see (0 when none). */
int32_t pm7_device_count(void);

/* ---------------------------------------------------------------------
 * Stage entry points: each runs one stage of the device pipeline for one
 * molecule and copies the result to host memory. They exist so the stages
 * can be checked one by one against the reference's own functions.
 * ------------------------------------------------------------------- */

/* The core Hamiltonian H_core (`build_core_generic`, src/hamiltonian.rs:310-638),
 * nao*nao row-major into h_out. *nao_out receives nao. */
pm7_status pm7_stage_core_hamiltonian(const pm7_molecule *molecule, const pm7_params *params,
                                      int32_t force_dpath, double *h_out, int32_t *nao_out);

/* The spin Fock matrix F = H + J(P_tot) - K(P_spin)
 * (`build_fock_spin_x` with no exchange cutoff, src/fock.rs:149-418). */
pm7_status pm7_stage_fock(const pm7_molecule *molecule, const pm7_params *params,
                          int32_t force_dpath, const double *p_tot, const double *p_spin,
                          double *f_out);

/* The same Fock matrix from the FP32 build of the mixed-precision mode's early cycles: the
 * densities and the stored pair integrals read as float and summed in FP32, the output in
 * double (src/fock.rs:149-418 at FP32 accuracy); a stage for accuracy tests. */
pm7_status pm7_stage_fock_fp32(const pm7_molecule *molecule, const pm7_params *params,
                               int32_t force_dpath, const double *p_tot, const double *p_spin,
                               double *f_out);

/* Per-pair two-centre blocks for atoms (i, j) at displacement d = R_j - R_i
 * (Bohr): w (npair_i x npair_j), e1b/e2a (9x9) and the overlap (9x9), all in
 * the i-first orientation (`pair_two_electron_g`, src/integrals.rs:186-271, and
 * `diatom_overlap`, src/overlap.rs:16-40, or their MNDO/d forms). */
pm7_status pm7_stage_pair(const pm7_params *params, int32_t z_i, int32_t z_j, const double d[3],
                          int32_t force_dpath, double *w_out, double *e1b_out, double *e2a_out,
                          double *s_out, int32_t *npair_i, int32_t *npair_j);

/* The mixed-precision SP2 squaring C = X X of a symmetric n x n matrix on the tcgen05
 * tensor cores (3xTF32 split, fp32 accumulation), as a stage for accuracy tests; no
 * counterpart in pm7-rs (its density step diagonalises). */
pm7_status pm7_stage_square_tf32(int32_t n, const double *x, double *c_out);

/* C = A B of two symmetric n x n matrices on the tcgen05 tensor cores (3xTF32), the DIIS
 * commutator product F P of the mixed-precision fp32 cycles; a stage for accuracy tests.
 * Replaces, in those cycles, the product of `commutator_into` (src/scf.rs:1148-1156). */
pm7_status pm7_stage_product_tf32(int32_t n, const double *a, const double *b, double *c_out);

/* One fused FP64-accuracy SP2 step on the tcgen05 integer tensor cores (int8 digit planes,
 * Ozaki-scheme emulation of the fp64 product): x_out = x x (square != 0) or 2 x - x x, for a
 * symmetric n x n x with elements in [-1.98, 1.98]; norms (2 doubles, may be null) receive
 * tr x_out and |x_out|_F^2 from the step's partials. A stage for accuracy tests. */
pm7_status pm7_stage_sp2_step_i8(int32_t n, const double *x, int32_t square, double *x_out, double *norms);

/* Failure drill of the bounded device waits (no counterpart in pm7-rs): runs the tcgen05
 * squaring of an n x n zero matrix (1 <= n <= 4096) with its copy producer withholding
 * every copy, so the pipeline's mbarrier waits never complete. Each wait gives up after its
 * time limit (1 s), the kernel frees its tensor memory and returns, and the call returns
 * PM7_ERR_TIMEOUT, as pm7_run does when a wait expires; the CUDA context stays usable. */
pm7_status pm7_stage_tf32_wait_drill(int32_t n);

/* Eigenvalues (ascending, no eigenvectors) of `count` symmetric matrices, the stage that
 * gives the reported MO energies when no orbitals are returned. Replaces the eigenvalue
 * half of `symmetric_eigen` (src/linalg.rs:231-278, faer self_adjoint_eigen) as used by
 * run_pm7's final step (src/scf.rs:1299-1305). Matrices are packed row-major one after
 * another (orders[i]^2 doubles each; order <= 8192), eigenvalues likewise (orders[i]
 * each). Host buffers; runs on `device`. */
pm7_status pm7_stage_eigenvalues(int32_t count, const int32_t *orders, const double *a, double *w,
                                 int32_t device);

/* Core-core repulsion energy in eV (`core_core_energy`, src/repulsion.rs:16-36). */
pm7_status pm7_stage_core_core(const pm7_molecule *molecule, const pm7_params *params,
                               double *energy_ev);

/* The left-to-right f64 sum of n terms, t_i = a[i] (b NULL) or t_i = a[i] * b[i] (each
 * product rounded, then added), computed on `device` and returned in *out with the exact
 * bits of a serial loop. This is how the engine evaluates the reference's energy folds
 * (`Matrix::frobenius_dot`, src/linalg.rs:138-141; the pair-order sum of
 * `core_core_energy`, src/repulsion.rs:16-36); exposed as a stage for bit-exact tests.
 * Host buffers. */
pm7_status pm7_stage_seqsum(int64_t n, const double *a, const double *b, double *out, int32_t device);

/* Post-SCF corrections in kcal/mol (`correction_energy`, src/scf.rs:907-932):
 * out[0] dispersion, out[1] H-bond, out[2] C#C, out[3] Si-O-H, out[4] PM7-HH. */
pm7_status pm7_stage_corrections(const pm7_molecule *molecule, int32_t method,
                                 int32_t smooth_dispersion, double out[5]);

/* ---------------------------------------------------------------------
 * Engine diagnostics (no reference analogue).
 * ------------------------------------------------------------------- */

/* Number of CUDA kernels this library has launched since the process started. */
int64_t pm7_launch_count(void);

/* The autotuner's decisions so far in this process, as JSON: {"<device>|<kernel key>":
 * variant, ...}. Result-identical launch variants (GEMM tile shapes, warps per block) are
 * timed on first use per size bucket; PM7_AUTOTUNE_CACHE names a JSON file that keeps them
 * across processes. No counterpart in pm7-rs. */
const char *pm7_autotune_report(void);

/* Per-stage device timing with CUDA events on the engine's stream: enable (1) resets
 * and starts recording, 0 stops. Stages: "build", "fock", "commutator_gemm",
 * "density_gemm", "eigensolve", "diis_dots", "combine", "corrections". */
void pm7_profile_enable(int32_t on);
int32_t pm7_profile_count(void);
/* Entry i: name, total device milliseconds and number of timed calls. */
pm7_status pm7_profile_entry(int32_t i, const char **name, double *total_ms, int64_t *calls);

/* ---------------------------------------------------------------------
 * Allocation-free post-SCF corrections. This entry point has no counterpart in
 * the reference; it exists for callers that cannot call cudaMalloc: a host that
 * owns all device memory through its own pool (a framework's caching allocator,
 * a serving process with a fixed HBM budget), or a loop that must not take the
 * implicit synchronisation a device allocation can cause.
 *
 * Same result as pm7_stage_corrections(), but every pointer is a DEVICE pointer
 * supplied by the caller: z_dev (n_atoms int32 atomic numbers), xyz_bohr_dev
 * (3*n_atoms doubles, Bohr) and out_dev (5 doubles, kcal/mol: dispersion, H-bond,
 * C#C, Si-O-H, PM7-HH). Work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns without waiting for it.
 *
 * The kernels' scratch is one static device array sized for at most
 * pm7_corrections_noalloc_max_atoms() atoms (2048, about 1 MB), held by every GPU
 * that loads the library until the process exits; larger molecules are rejected
 * with PM7_ERR_INVALID_INPUT. The first call on each device looks up that array's
 * device address (with the device current), so make that first call before any
 * stream capture. All calls on a device share the one array: calls whose work
 * overlaps on the GPU (different streams, or different host threads) race and must
 * be serialised by the caller. The call allocates nothing: no cudaMalloc, no
 * cudaFree, no library allocator. */
pm7_status pm7_corrections_noalloc(int32_t n_atoms, const int32_t *z_dev, const double *xyz_bohr_dev,
                                   int32_t method, int32_t smooth_dispersion, double *out_dev, void *stream);
/* Message of the last pm7_corrections_noalloc failure on the calling thread. */
const char *pm7_corrections_noalloc_error(void);
/* Largest n_atoms pm7_corrections_noalloc accepts. */
int32_t pm7_corrections_noalloc_max_atoms(void);

/* ---- batched and served solves ------------------------------------------------
 * No counterpart in pm7-rs: its callers (src/python.rs:437, src/bin/pm7_rs.rs:176,
 * src/optimizer.rs:318) loop over run_pm7 one molecule at a time. These entry points
 * give the same per-molecule results (closed-shell RHF in the batch; other requests
 * take the pm7_run path) while many molecules share each SCF-phase launch. */

/* Solves n_molecules independent molecules with options[i] each (options[0].device
 * selects the GPU and options[0].max_memory_mb, when >= 0, caps the HBM the batch
 * holds at once). results[i] / statuses[i] receive what pm7_run would return for
 * molecule i; release each result with pm7_result_free. Returns PM7_OK when the batch
 * ran (per-molecule failures are in statuses), or the error that stopped it. */
pm7_status pm7_run_batch(int32_t n_molecules, const pm7_molecule *molecules, const pm7_params *params,
                         const pm7_options *options, pm7_result *results, pm7_status *statuses);

/* Splits a batch over n_ranks GPUs (or processes) for independent pm7_run_batch calls:
 * greedy longest-processing-time by an estimated cost per molecule (a constant per
 * solve + nao^3 for the dense SCF work + 1000 per atom pair for the integrals), heaviest
 * first, each to the least loaded rank (ties: lowest index). rank_of[i] receives the
 * rank of molecule i; rank_cost (n_ranks entries, may be NULL) the summed cost per rank.
 * Host only: needs no device. Deterministic for equal inputs. Molecules whose elements
 * have no parameters count with one orbital per atom (their solve fails at once). */
pm7_status pm7_batch_partition(int32_t n_molecules, const pm7_molecule *molecules, int32_t method,
                               int32_t n_ranks, int32_t *rank_of, double *rank_cost);

/* A serving engine: a worker thread on one GPU admits submitted closed-shell RHF
 * requests as HBM (their device footprint against hbm_budget_mb, or 80% of free
 * memory when -1) and max_active (0 = unlimited) allow, advances all admitted
 * requests together one SCF iteration per step, and retires each as it converges.
 * Open-shell and forced-UHF requests run one at a time through the pm7_run path on a
 * second worker thread, beside the batch. */
typedef struct pm7_engine pm7_engine;
typedef struct pm7_engine_config {
  int32_t device;
  int32_t method;        /* pm7_method of every request */
  int64_t hbm_budget_mb; /* -1: 80% of the device's free memory at creation */
  int32_t max_active;    /* 0: no limit besides memory */
} pm7_engine_config;

void pm7_engine_config_default(pm7_engine_config *config);
pm7_status pm7_engine_create(const pm7_engine_config *config, pm7_engine **out);
/* Queues one request; *ticket identifies it. Invalid input is reported by poll. */
pm7_status pm7_engine_submit(pm7_engine *engine, const pm7_molecule *molecule, const pm7_options *options,
                             uint64_t *ticket);
/* pm7_engine_submit with the request's nuclear gradient (eV/Bohr, as pm7_gradient returns
 * it): the engine writes 3 * n_atoms doubles to `gradient` before the request is done, so the
 * buffer must stay valid until pm7_engine_poll reports done. No counterpart in pm7-rs; its
 * force callers (src/optimizer.rs:318) call closed_form_gradient per molecule. */
pm7_status pm7_engine_submit_gradient(pm7_engine *engine, const pm7_molecule *molecule,
                                      const pm7_options *options, double *gradient, uint64_t *ticket);

/* *done = 1 when the request finished; the return value is then its pm7_run status,
 * *result is filled (caller frees) and *latency_ms is submit-to-finish time. With
 * wait != 0 the call blocks until the request finishes. A finished ticket is
 * forgotten after it is polled. */
pm7_status pm7_engine_poll(pm7_engine *engine, uint64_t ticket, int32_t wait, int32_t *done, pm7_result *result,
                           double *latency_ms);
/* Admission record of the engine so far: out[0] requests admitted, out[1] the most
 * requests resident on the device at once, out[2] the most device bytes they held at once
 * (their footprints), out[3] the HBM budget in bytes. No counterpart in pm7-rs. */
pm7_status pm7_engine_stats(pm7_engine *engine, int64_t out[4]);
/* Finishes every submitted request, then stops the worker. */
pm7_status pm7_engine_destroy(pm7_engine *engine);

/* ---- divide-and-conquer SCF --------------------------------------------------------
 * `DandcOptions` (src/dandc/mod.rs:62-99); defaults from pm7_dandc_options_default. */
typedef struct pm7_dandc_options {
  double buffer;         /* buffer radius, Bohr (15.0) */
  int32_t core_size;     /* target atoms per core (12) */
  double fermi_width_ev; /* Fermi smearing of the common chemical potential (0.1) */
  int32_t max_scf;       /* (200) */
  double p_tol;          /* RMS density change over the stored blocks (1e-6) */
  double mixing;         /* linear density mixing factor in (0, 1] (0.4) */
} pm7_dandc_options;

void pm7_dandc_options_default(pm7_dandc_options *options);
/* sizeof(pm7_dandc_options), sizeof(pm7_dandc_result): bindings check their mirrors. */
void pm7_dandc_abi_sizes(int64_t out[2]);

/* `DandcResult` (src/dandc/mod.rs:121-140) with `DandcDerivatives` (:438-443). The global
 * density is returned dense (nao x nao, row-major) with zeros outside the stored atom-pair
 * pattern; the caller frees the arrays with pm7_dandc_result_free. */
typedef struct pm7_dandc_result {
  int32_t n_atoms, nao;
  int32_t converged, iterations, subsystems, largest_subsystem, unrestricted;
  double fermi_ev, electronic_ev, density_error;
  double core_core_ev, correction_ev;
  double energy_ev;                 /* electronic + core-core + corrections (dandc_derivatives) */
  int64_t stored_density_elements;  /* SparseDensity::stored_elements */
  double *charges;                  /* n_atoms Mulliken net charges (src/dandc/mod.rs:819-829) */
  double *gradient;                 /* 3 n_atoms eV/Bohr when requested, else NULL */
  double *density;                  /* nao x nao when options->want_matrices, else NULL */
  double *spin_density;             /* nao x nao, unrestricted and options->want_matrices */
} pm7_dandc_result;

/* Replaces `run_dandc` (src/dandc/mod.rs:143-428) and, with want_gradient != 0,
 * `dandc_derivatives` (:446-506) for a molecule: subsystem cores by recursive median
 * bisection with a buffer shell, one Fock build and eigendecomposition per subsystem on the
 * device, one global Fermi level, Dixon-Merz weights normalised per atom pair, linear mixing.
 * A run that reaches max_scf returns PM7_OK with converged = 0, as the reference does.
 * Option errors and a largest subsystem beyond the memory budget are PM7_ERR_INVALID_INPUT. */
pm7_status pm7_run_dandc(const pm7_molecule *molecule, const pm7_params *params,
                         const pm7_options *options, const pm7_dandc_options *dandc,
                         int32_t want_gradient, pm7_dandc_result *result);
void pm7_dandc_result_free(pm7_dandc_result *result);

/* The subsystem partition of pm7_run_dandc alone (host only, no device), for parity tests of
 * `partition` (src/dandc/partition.rs): core_of[atom] = the subsystem whose core holds the atom,
 * sizes[s] = atoms of subsystem s (core and buffer; sizes holds n_atoms entries), the count of
 * subsystems and of stored atom pairs (ordered, the diagonal included). */
pm7_status pm7_stage_dandc_partition(const pm7_molecule *molecule, int32_t core_size, double buffer,
                                     int32_t *core_of, int32_t *sizes, int32_t *n_subsystems,
                                     int64_t *stored_pairs);

#ifdef __cplusplus
}
#endif

#endif /* PM7_B200_H */
