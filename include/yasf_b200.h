/*
 * yasf_b200 — C ABI of the B200-native coupling backend for the T-matrix multiple-sphere solve.
 *
 * Every entry point takes plain pointers and sizes, returns an int status (YASF_OK == 0), never
 * synchronises the host unless stated, and never takes ownership of caller memory. Vectors are
 * device pointers to interleaved complex numbers (re, im), particle-major: element (s, n) sits
 * at s*nmax + n, n = (tau-1)*lmax*(lmax+2) + (l-1)*(l+1) + l + m, exactly the unknown ordering of
 * yasfpy/functions/cpu_numba.py:371-407. `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream). Positions are device float64 (N, 3) row-major, lengths in the
 * same unit as the wavelength; k_medium is the real medium wavenumber (yasfpy/parameters.py:96-100).
 *
 * Precision codes: YASF_C128 computes the translation generation and contraction in complex128;
 * YASF_C64 computes them in complex64 while vectors stay complex128 (inputs are rounded on the
 * way in, outputs widened on the way out).
 */
#ifndef YASF_B200_H
#define YASF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define YASF_ABI_VERSION 1

enum yasf_status {
  YASF_OK = 0,
  YASF_ERR_INVALID_ARGUMENT = 1, /* null pointer, non-positive size, bad enum value */
  YASF_ERR_UNSUPPORTED = 2,      /* lmax outside [1, 8], non-finite k, ... */
  YASF_ERR_ALIGNMENT = 3,        /* pointer not 16-byte aligned */
  YASF_ERR_CUDA = 4,             /* a CUDA runtime call failed (see yasf_last_cuda_error) */
  YASF_ERR_OUT_OF_MEMORY = 5,    /* a device allocation made by the library failed */
  YASF_ERR_WORKSPACE = 6,        /* workspace smaller than the size query returned */
  YASF_ERR_NOT_FINITE = 7,       /* NaN/Inf in the right-hand side or the iteration */
  YASF_ERR_NOT_PREPARED = 8,     /* preconditioner used before prepare */
  YASF_ERR_SCRATCH_LIMIT = 9     /* problem larger than the static scratch of the no-alloc call */
};

enum yasf_precision { YASF_C128 = 0, YASF_C64 = 1 };

typedef struct yasf_plan yasf_plan;         /* per-lmax translation structure on one device */
typedef struct yasf_precond yasf_precond;   /* block-Jacobi preconditioner on one device */

/* ---- library ---------------------------------------------------------------------------- */
int yasf_abi_version(void);
const char* yasf_status_string(int status);
/* Last CUDA error string seen by the library on this thread ("" if none). */
const char* yasf_last_cuda_error(void);
/* Kernels launched by the library in this process so far (all threads). Counterpart of the
 * per-operator matvec_calls / uploads counters of yasfpy/coupling/cuda_dense.py:102-105. */
unsigned long long yasf_kernel_launches(void);

/* Tile shapes for the next launches and workspace-size queries FROM THIS HOST THREAD (0 keeps the
 * built-in rule): contract_waves in {1, 2, 4, 8} sizes the coupling contraction's source chunks for
 * that many waves of resident blocks (rule: 2); dpanel_cols in {32, 64} is the float64 dense panel's
 * column tile (rule: 64 from 64 columns, else 32); panel_groups in {1, 2} is the tensor-core panel's
 * column groups of 64 per block (rule: 2 when there are two, up to lmax 7). Set it before the size
 * query of a solve and keep it for the solve. Chosen per (lmax, N, R) by yasf_b200.autotune; no
 * reference counterpart. */
int yasf_set_tiles(int contract_waves, int dpanel_cols, int panel_groups);

/* Test hook for failure detection; no counterpart in the reference. Every wait inside a kernel of
 * this library is bounded: when it runs out, the kernel records an error word, writes NaN outputs,
 * frees what it holds and returns, so the CUDA context stays usable and the host sees
 * YASF_ERR_NOT_FINITE from a solve. This call makes such a wait run out on purpose for the next
 * launches FROM THIS HOST THREAD: `role` names one producer that never delivers (the first stage
 * copy of every block of the coupling contraction; the pair-table warps of the tensor-core panel;
 * the helper warp of the float64 dense panel; the first tile row of a one-column preconditioner
 * apply, whose sweeps then wait on it and write NaN), `contract_polls` (> 0) replaces the contraction's
 * poll limit per stage wait (2^22) and `panel_wait_seconds` (> 0, <= 10) the wait bound of the
 * panels and of the preconditioner sweeps (1 s). 0 keeps a default. YASF_STALL_NONE restores
 * normal launches. The error word a kernel sets is the int at byte offset (required workspace
 * bytes - 256) of the call's workspace, for the coupling, panel and dense-panel entry points alike
 * (0: every wait completed); a preconditioner apply whose wait ran out leaves NaN in its output. */
enum yasf_stall_role {
  YASF_STALL_NONE = 0,
  YASF_STALL_CONTRACT = 1,
  YASF_STALL_PANEL = 2,
  YASF_STALL_DPANEL = 3,
  YASF_STALL_PRECOND = 4
};
int yasf_test_stall(int role, int contract_polls, double panel_wait_seconds);

/* ---- plan: the a5/b5 translation table in the layout the kernels stream -----------------
 * Replaces the per-Simulation table handling of yasfpy/coupling/cpu_dense.py:45-64 and
 * yasfpy/coupling/cuda_dense.py:52-158. `translation_ab5` is the HOST complex128 array
 * (nmax, nmax, 2*lmax+1) of yasfpy/numerics.py:187-281 (Numerics.translation_ab5), indexed
 * [n_source, n_receiver, p] as the matvec reads it (cpu_numba.py:86). The plan is built for the
 * current CUDA device and allocates its own device memory. */
int yasf_plan_create(int lmax, const double* translation_ab5, yasf_plan** plan);
int yasf_plan_destroy(yasf_plan* plan);
/* nmax, stream entries per source particle (all bundles) and source-side terms per particle of the
 * float64 kernels' stream layout (the complex64 kernel may split the stream into other bundles). */
int yasf_plan_info(const yasf_plan* plan, int* nmax, long long* stream_entries,
                   long long* source_terms);
/* Host-only check (no device, nothing allocated on a GPU): builds the generation layouts a plan
 * derives from `translation_ab5` (the tensor-core panel's schedule with its slot tables and term
 * windows, the float64 dense panel's items) and returns YASF_ERR_INVALID_ARGUMENT if the table
 * breaks the a5/b5 selection rules or mirror relations they rely on, YASF_ERR_NOT_FINITE for
 * non-finite entries; yasf_plan_create runs the same check. No reference counterpart. */
int yasf_plan_check_table(int lmax, const double* translation_ab5);

/* Bytes of caller-provided device workspace needed by the coupling entry points for
 * n_particles spheres and nrhs right-hand sides at `precision`. */
int yasf_coupling_workspace_size(const yasf_plan* plan, int n_particles, int nrhs, int precision,
                                 size_t* bytes);

/* ---- coupling matvec -----------------------------------------------------------------------
 * y = W x with every W_ij generated on the fly (spherical Hankel h_p(k r_ij) by upward
 * recurrence, normalised Legendre P_p^{|m-m'|}(cos theta_ij) by the CELES recurrence, the
 * azimuthal phase e^{i(m'-m) phi_ij}, and the a5/b5 coefficients), summed over s_j != s_i.
 * Replaces particle_interaction_scalar (yasfpy/functions/cpu_numba.py:22-95) behind
 * DenseCouplingOps.matvec (yasfpy/coupling/ops.py:29-49) and CouplingBackend.multiply
 * (yasfpy/coupling/backends.py:47-66).
 * x, y: (n_particles*nmax) complex128 on the device; nrhs columns are stored column after
 * column with leading dimension ld (>= n_particles*nmax). */
int yasf_coupling_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                         double k_medium, const double* x, double* y, int nrhs, long long ld,
                         int precision, void* workspace, size_t workspace_bytes, void* stream);

/* Near-field variant: the same product restricted to the pairs with |pos_i - pos_j| <= radius
 * (self pairs excluded), all others dropped: the semantics of the reference's NearFarCouplingBackend
 * (yasfpy/coupling/backends.py:259-459, numerics.coupling_near_field_radius), which is CPU-only
 * there. Sources that no receiver of a thread block is near are skipped as a whole. Same workspace
 * as yasf_coupling_matvec; radius >= 0 and finite. */
int yasf_coupling_matvec_nearfield(const yasf_plan* plan, int n_particles, const double* positions,
                                   double k_medium, double near_field_radius, const double* x,
                                   double* y, int nrhs, long long ld, int precision, void* workspace,
                                   size_t workspace_bytes, void* stream);

/* No counterpart in the reference. For callers that cannot allocate device memory when they
 * call (all device memory reserved at start-up, an embedding runtime that owns the allocator, or
 * only fixed buffers to hand over): the same y = W x as yasf_coupling_matvec for one right-hand
 * side, with all scratch in one static device array of YASF_STATIC_SCRATCH_BYTES, so nothing is
 * allocated. Returns YASF_ERR_SCRATCH_LIMIT when yasf_coupling_workspace_size exceeds that size.
 * All calls on a device share the array: calls that overlap on the GPU race, so order them on
 * one stream. The first call on each device looks up the array (with that device current); make
 * it before any stream capture. Every GPU that loads the library holds the array until exit. */
#define YASF_STATIC_SCRATCH_BYTES (64u * 1024u * 1024u)
int yasf_coupling_matvec_noalloc(const yasf_plan* plan, int n_particles, const double* positions,
                                 double k_medium, const double* x, double* y, int precision,
                                 void* stream);

/* y = x - T (.) (W x): the master operator of yasfpy/matrix_apply.py:66-120 fused into the
 * reduction epilogue. tmat is (n_particles*nmax) complex128: T[s,n] = mie[sidx[s], n, w]. */
int yasf_master_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                       double k_medium, const double* tmat, const double* x, double* y, int nrhs,
                       long long ld, int precision, void* workspace, size_t workspace_bytes,
                       void* stream);

/* ---- multi-right-hand-side panel on the tensor cores ----------------------------------------
 * The batched form of the coupling matvec for R right-hand sides (incidence directions x
 * polarisations), replacing the multi-channel particle_interaction loop
 * (yasfpy/functions/cpu_numba.py:99-181) for the inner solves of the refined, batched GMRES:
 * every pair block W_ij is generated once in FP32 (as the tau-symmetric P = Wa + Wb, Q = Wa - Wb)
 * and applied to the source's columns, 64 or 128 per block, on tcgen05 tensor cores (TF32 inputs,
 * FP32 accumulation; relative accuracy ~1e-3). y = x - T (.) (W x) when tmat is non-NULL, else
 * y = W x; x and y columns have leading dimensions ldx and ldy. Every lmax of
 * a plan (1..8). */
int yasf_panel_workspace_size(const yasf_plan* plan, int n_particles, int nrhs, size_t* bytes);
int yasf_panel_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                      double k_medium, const double* tmat, const double* x, double* y, int nrhs,
                      long long ldx, long long ldy, void* workspace, size_t workspace_bytes,
                      void* stream);

/* ---- float64 dense multi-column coupling -------------------------------------------------------
 * The multi-channel particle_interaction (yasfpy/functions/cpu_numba.py:99-181) in float64 for
 * nrhs columns at once: every W_ij is formed once per pair (tau-symmetric P = Wa + Wb, Q = Wa - Wb)
 * and applied to blocks of 32 columns. Same arguments and outputs as yasf_panel_matvec
 * (y = x - T (.) W x when tmat is non-NULL, else y = W x), float64 throughout; agrees with
 * yasf_coupling_matvec to rounding. lmax <= 6 (YASF_ERR_UNSUPPORTED otherwise). Used for the
 * float64 residuals of yasf_batched_solve. */
int yasf_dpanel_workspace_size(const yasf_plan* plan, int n_particles, int nrhs, size_t* bytes);
int yasf_dpanel_matvec(const yasf_plan* plan, int n_particles, const double* positions,
                       double k_medium, const double* tmat, const double* x, double* y, int nrhs,
                       long long ldx, long long ldy, void* workspace, size_t workspace_bytes,
                       void* stream);

/* ---- batched right-hand sides: refined lockstep GMRES -----------------------------------------
 * (I - T W) X = B for nrhs columns (incidence directions x polarisations; the reference solves one
 * incidence per Simulation, yasfpy/scattered_field_coefficients.py:95-144 with
 * yasfpy/solver.py:108-121). Float64 iterative refinement: residuals B - A X in float64, inner
 * left-preconditioned GMRES cycles (restart steps, each column its own float64 Krylov basis, all
 * live columns sharing one operator application per step) to inner_rtol on the reduced-precision
 * operator inner_kind: 0 tensor-core TF32 panel, 1 complex64 coupling kernel,
 * 2 complex128 coupling kernel. X0 = 0. Columns leave when ||B_c - A X_c|| <= rtol ||B_c||.
 * stats (host, may be NULL): [0] lockstep inner steps, [1] panel applications, [2] column
 * applications of kinds 1/2, [3] float64 residual column applications (float64 applications to
 * 12 or more columns use yasf_dpanel_matvec when lmax <= 6), [4] worst relative residual,
 * [5] unconverged columns, [6] refinement steps. column_residuals (host, may be NULL): nrhs
 * final relative residuals. Synchronous. */
int yasf_batched_workspace_size(const yasf_plan* plan, int n_particles, int nrhs, int restart,
                                int inner_kind, size_t* bytes);
int yasf_batched_solve(const yasf_plan* plan, int n_particles, const double* positions,
                       double k_medium, const double* tmat, const yasf_precond* pc,
                       const double* b, double* x, int nrhs, double rtol, int restart,
                       int max_refine, double inner_rtol, int inner_kind, void* workspace,
                       size_t workspace_bytes, double* stats, double* column_residuals,
                       void* stream);

/* ---- right-hand sides of R plane-wave incidences ---------------------------------------------
 * Replaces compute_initial_field_coefficients for plane waves (yasfpy/initial_field_coefficients.py:
 * 79-142) and compute_right_hand_side (yasfpy/simulation.py:189-205) for R incidences at once:
 * a[r][s*nmax + n] = coef[r][n] e^{i kvec_r . (pos_s - focal_point)}, b = tmat (.) a.
 * coef (device, nrhs x nmax complex128): 4 E0 e^{-i m alpha_r} B^dagger_{tau l m}(beta_r) per incidence;
 * kvec (device, nrhs x 3): the wave vectors; focal_point: host (3,) or NULL for the origin; positions:
 * device (N, 3). a or b may be NULL (b needs tmat). Columns have leading dimension ld. Asynchronous. */
int yasf_plane_wave_rhs(int lmax, int n_particles, const double* positions, int nrhs,
                        const double* kvec, const double* coef, const double* focal_point,
                        const double* tmat, double* a, double* b, long long ld, void* stream);

/* ---- far field of the scattered wave (consumers of the coefficients) ---------------------------
 * Replaces Optics.compute_scattered_e_field_angle_components (yasfpy/optics.py:178-267; kernels
 * yasfpy/functions/cpu_numba.py:536-601 and cuda_numba.py:824-894) and the Stokes part of
 * compute_polarization_components (cpu_numba.py:604-660) for one wavelength: for every sampling
 * direction a, E_theta(a) and E_phi(a) = sum over particles s and modes n of
 * i^{tau-l-2} coef[s,n] / sqrt(2l(l+1)) e^{i(m phi_a - k r_s.e_r(a))} times the angular functions,
 * and (stokes, may be NULL) I, Q, U, V per direction (4 doubles each). coef: device (N*nmax)
 * complex128, particle-major (the solution vector); positions: device (N, 3); polar, azimuthal:
 * device (n_dirs) radians; pilm, taulm: device (lmax+1, lmax+1, n_dirs) float64, the reference's
 * spherical_functions_trigon arrays (yasfpy/functions/spherical_functions_trigon.py:11-96);
 * e_theta, e_phi: device (n_dirs) complex128. Asynchronous. */
int yasf_far_field(int lmax, int n_particles, const double* positions, double k_medium, const double* coef,
                   int n_dirs, const double* polar, const double* azimuthal, const double* pilm,
                   const double* taulm, double* e_theta, double* e_phi, double* stokes, void* stream);

/* ---- grouped solve: right-hand sides of several aggregates at once -------------------------------
 * No single reference counterpart: the reference solves one aggregate and one incidence per
 * Simulation (yasfpy/scattered_field_coefficients.py:95-144, yasfpy/solver.py:108-121). Here the
 * columns of several aggregates of one lmax (each its own spheres, positions, wavenumber, T and
 * right-hand sides) are solved together by lockstep float64-refined GMRES, every column with its own
 * Krylov basis: each operator application is three launches for all live columns of all aggregates,
 * the middle one a persistent work-queue contraction (resident blocks take (column, receiver tile,
 * source chunk, bundle) items from a device counter), so small aggregates share launches instead of
 * each running its own. Inner operator at inner_precision (YASF_C64 or YASF_C128), float64
 * residuals, X0 = 0, columns leave at ||b - A x|| <= rtol ||b||; no preconditioner.
 * stats (host, may be NULL): [0] lockstep inner steps, [1] inner operator applications (all columns
 * each), [2] float64 applications, [3] worst relative residual, [4] unconverged columns,
 * [5] refinement steps, [6] columns, [7] work items per application. column_residuals (host, may be
 * NULL): final relative residual of every column, aggregate by aggregate. Synchronous.
 * yasf_grouped_workspace_size reads only n_particles and nrhs of each problem (its pointers may be
 * NULL), so a group can be sized before its buffers exist. */
typedef struct {
  int n_particles;
  const double* positions;   /* device (N, 3) */
  double k_medium;
  const double* tmat;        /* device (N*nmax) complex128 */
  const double* b;           /* device, nrhs columns of N*nmax */
  double* x;                 /* device, nrhs columns of N*nmax (output) */
  int nrhs;
} yasf_problem;
int yasf_grouped_workspace_size(const yasf_plan* plan, int n_problems, const yasf_problem* problems,
                                int restart, size_t* bytes);
int yasf_grouped_solve(const yasf_plan* plan, int n_problems, const yasf_problem* problems, double rtol,
                       int restart, int max_refine, double inner_rtol, int inner_precision,
                       void* workspace, size_t workspace_bytes, double* stats, double* column_residuals,
                       void* stream);

/* ---- cross sections (yasfpy/optics.py:55-156) ------------------------------------------------
 * out[0..1] (device) <- sum_{s,n} conj(b) (W_reg b), the bilinear form of
 * compute_scattering_cross_section (yasfpy/functions/cpu_numba.py:410-457): regular spherical
 * Bessel j_p, self pairs included. C_sca = pi/|k|^2 * |out|. */
int yasf_scattering_bilinear(const yasf_plan* plan, int n_particles, const double* positions,
                             double k_medium, const double* b, double* out, void* workspace,
                             size_t workspace_bytes, void* stream);
/* out[0..1] (device) <- sum conj(a) * b over n elements (C_ext = -pi/|k|^2 * Re(out)). */
int yasf_dotc(long long n, const double* a, const double* b, double* out, void* workspace,
              size_t workspace_bytes, void* stream);

/* ---- block-Jacobi preconditioner (yasfpy/preconditioner.py:58-219) ---------------------------
 * Blocks are given as a particle list per block (CSR: block_ptr[n_blocks+1], particles[]); the
 * library assembles M_B = (I - T W)[B,B] on the device with the same generator as the matvec
 * (particle-major rows and columns, receiver Mie factor), factors every block in place with its own
 * batched LU (yasf_precond_factor) and keeps, after finalize, the complex64 factors the solves
 * stream. Protocol: create -> assemble -> factor -> finalize -> apply (any number of times).
 * (A caller may instead invert every block in place between assemble and finalize, with any dense
 * complex128 inversion; finalize then keeps complex128 and complex64 copies of those inverses and
 * apply streams them.)
 * apply: y = M^{-1} x, block by block (x and y must not alias). */
int yasf_precond_create(const yasf_plan* plan, int n_particles, int n_blocks,
                        const int* block_ptr /*host*/, const int* particles /*host*/,
                        yasf_precond** pc);
int yasf_precond_destroy(yasf_precond* pc);
/* Replaces prepare()'s block assembly (yasfpy/preconditioner.py:92-175, 365-442). Asynchronous. */
int yasf_precond_assemble(yasf_precond* pc, const double* positions, double k_medium,
                          const double* tmat, void* stream);
/* Device pointer and order of block `block`: row-major (dim, dim) complex128, dim = n_B*nmax,
 * rows/columns in the block's particle order, particle-major inside. Available from assemble until
 * a complex64 factorisation (or a finalize) releases the complex128 blocks (YASF_ERR_NOT_PREPARED
 * afterwards). */
int yasf_precond_block(const yasf_precond* pc, int block, double** matrix, int* dim);
/* Replaces the block LU of prepare() (yasfpy/preconditioner.py:445-468, scipy.linalg.lu on complex64
 * blocks): every block factored in place, P_B M_B = L_B U_B, by a right-looking tile LU (64 x 64
 * tiles, partial pivoting inside each diagonal tile, so P_B permutes rows only within each tile
 * row); all blocks of the preconditioner in one sequence of launches. By default in complex64, as
 * the reference factors (the complex128 blocks are converted and released first; diagonal-tile
 * steps in float64 arithmetic, trailing updates in FP32); in complex128 when
 * yasf_precond_keep_float64(pc, 1) was called before. Synchronises the stream in complex64 mode
 * (the release), else asynchronous. */
int yasf_precond_factor(yasf_precond* pc, void* stream);
/* Call before factor: 1 factors in complex128 and keeps those factors beside the complex64 copy
 * after finalize (YASF_C128 applies stream them); 0 (default) factors in complex64, halving the
 * resident bytes, and YASF_C128 applies stream the complex64 factors. */
int yasf_precond_keep_float64(yasf_precond* pc, int keep);
/* Call after factor (or after the caller's in-place inversion). Makes the complex64 copy and, after
 * factor, the inverses of the diagonal tiles of L and U; YASF_ERR_NOT_FINITE for a zero pivot.
 * Synchronises the stream. */
int yasf_precond_finalize(yasf_precond* pc, void* stream);
/* Replaces BlockDiagonalPreconditioner.apply (yasfpy/preconditioner.py:177-219, the unit-lower and
 * upper triangular solves of :470-519): gather with the pivots, a forward sweep with L and a
 * backward sweep with U over tile rows (float64 arithmetic on the complex64 factors, or the
 * complex128 ones when kept and precision is YASF_C128), scatter. One column: both sweeps in one
 * launch whose blocks take tile rows in dependency order and wait (bounded, 1 s; NaN output when a
 * wait runs out) on per-block finished-row counters. Several columns: one launch per tile row,
 * captured once per column count as a CUDA graph (on a private stream) and replayed on `stream`.
 * The first apply with more columns than any before allocates the preconditioner's sweep buffer;
 * applies of ONE preconditioner on different streams at the same time race on that buffer and on
 * the one-column counters. */
int yasf_precond_apply(const yasf_precond* pc, const double* x, double* y, int nrhs, long long ld,
                       int precision, void* stream);
/* Device bytes held by the factors. */
int yasf_precond_bytes(const yasf_precond* pc, size_t* bytes);

/* ---- device GMRES (yasfpy/solver.py:65-181 -> scipy.sparse.linalg.gmres) --------------------
 * Restarted, left-preconditioned GMRES with SciPy's stopping rules: the inner loop stops when the
 * preconditioned residual estimate reaches ptol (adapted per restart as SciPy does), every restart
 * cycle ends with the true residual ||b - A x|| checked against rtol*||b||; maxiter counts
 * restart cycles. A = I - T W. x holds x0 on entry and the solution on exit. Arnoldi uses
 * classical Gram-Schmidt with one re-orthogonalisation pass; Givens rotations and the Hessenberg
 * solve run on the device in float64. A preconditioner (pc, may be NULL) is applied from the
 * complex64 copy of its block inverses with float64 arithmetic: a fixed linear operator, half the
 * bytes of the float64 copy (the reference's block factors are complex64 too,
 * yasfpy/preconditioner.py:391).
 * inner_precision: YASF_C128 for the plain solve; YASF_C64 runs the Krylov iterations on the
 * complex64 matvec and wraps them in float64 iterative refinement (true residual, update and
 * stopping test in float64), see the solve stats.
 * stats (host, may be NULL): [0] inner iterations, [1] matvecs at inner precision,
 * [2] float64 matvecs, [3] final ||b - A x|| / ||b||, [4] info (0 converged, else maxiter),
 * [5] refinement steps. */
int yasf_gmres_workspace_size(const yasf_plan* plan, int n_particles, int restart,
                              int inner_precision, size_t* bytes);
int yasf_gmres_solve(const yasf_plan* plan, int n_particles, const double* positions,
                     double k_medium, const double* tmat, const yasf_precond* pc, const double* b,
                     double* x, double rtol, int restart, int maxiter, int inner_precision,
                     void* workspace, size_t workspace_bytes, double* stats, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* YASF_B200_H */
