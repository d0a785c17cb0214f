/* Extensions of the qkrylov C ABI provided by libqkrylov_b200.so.
 *
 * qkrylov's own C ABI (qkrylov_c_api.h) runs in single precision.  The
 * functions here add: double-precision Hamiltonians and solvers (the
 * reference's fp64 C++ namespace: its src/solvers sources compiled with
 * QKRYLOV_DOUBLE_PRECISION), device-pointer H.x for callers that keep
 * vectors in HBM, a multi-temperature FTLM, the OpSum compiler's output for
 * inspection, and library diagnostics.  They reuse the opaque handles of
 * qkrylov_c_api.h.  All return QKRYLOV_SUCCESS / QKRYLOV_ERROR_INVALID_ARG /
 * QKRYLOV_ERROR_EXCEPTION unless stated; qkrylov_b200_last_error() describes
 * the last failure on the calling thread.
 */
#ifndef QKRYLOV_B200_H
#define QKRYLOV_B200_H

#include "qkrylov_c_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Vector element types of the device-pointer entry points. */
#define QKRYLOV_DTYPE_C128 0 /* interleaved complex double */
#define QKRYLOV_DTYPE_C64 1  /* interleaved complex float */
#define QKRYLOV_DTYPE_F64 2  /* real double (real Hamiltonians only) */
#define QKRYLOV_DTYPE_F32 3  /* real float (real Hamiltonians only) */

/* ------------------------------------------------------------ diagnostics */
const char* qkrylov_b200_last_error(void);
/* Kernels launched by this library since it was loaded. */
uint64_t qkrylov_b200_launch_count(void);
int qkrylov_b200_device_count(void);
/* 0 (default): H.x uses the specialised row kernels (one CTA per sector
 * block, x of the block staged in shared memory, per-row class tables)
 * wherever the compiled operator has their tables, with per-die work queues
 * on a two-die GPU; 1: the generic kernel everywhere; 2: as 0 with the
 * blocks handed out in one grid-stride order (no per-die queues); 3: as 0
 * with Hubbard-type operators on the two-part row kernel instead of their
 * spin-product path.  For comparisons; process-wide.  Other values:
 * QKRYLOV_ERROR_INVALID_ARG. */
int qkrylov_b200_set_kernel_policy(int policy);
/* Dies of the current device as the row kernels' topology probe measured
 * them (2 on a B200, 1 where the probe saw one) and the SMs of each (first
 * call on a device: a few probe launches; later calls: cached). */
int qkrylov_b200_die_count(int* sms_die0, int* sms_die1);

/* Select which of N_up / N_dn a sector conserves after
 * qkrylov_sector_set_hubbard_particles (c_api.h:33), which always sets
 * both; qkrylov's C++ Sector allows either alone (sector.hpp:20-24). */
int qkrylov_b200_sector_set_species(qkrylov_sector_h sector, int use_nup, int use_ndn);

/* Site::apply (site.hpp:19-23) for a site handle: one operator on one state. */
int qkrylov_b200_site_apply(qkrylov_site_h site, const char* op, int site_index, uint64_t state, int* valid,
                            uint64_t* new_state, double* matrix_element /* [2] */);

/* ------------------------------------------------------ basis (host only)
 * Replaces the per-state loops a caller of qkrylov_basis_state /
 * qkrylov_basis_index (c_api.h:51-52) would write. */
int qkrylov_basis_states(qkrylov_basis_h basis, uint64_t first, uint64_t count, uint64_t* states_out);
int qkrylov_basis_index_many(qkrylov_basis_h basis, const uint64_t* states, uint64_t n, int64_t* index_out);

/* ------------------------------------------------------------------ OpSum
 * qkrylov_opsum_add_term_nbody (c_api.h:75-76) with double coefficients. */
int qkrylov_opsum_add_term_nbody_f64(qkrylov_opsum_h opsum, double coeff_real, double coeff_imag, int n_factors,
                                     const char** ops, const int* sites);
uint64_t qkrylov_opsum_size(qkrylov_opsum_h opsum);

/* The OpSum compiler's output for (basis, site, opsum), without a GPU.
 * Term t: valid on |s> iff (s & mask[3t]) == mask[3t+1]; element
 * (coef[2t] + i coef[2t+1]) * (-1)^popcount(s & mask[3t+2]); terms
 * [first[g], first[g]+count[g]) of group g reach s ^ flip[g]; check[g] = 1
 * when that target may leave the sector.  Pass NULL arrays to get counts. */
int qkrylov_opsum_compile(qkrylov_basis_h basis, qkrylov_site_h site, qkrylov_opsum_h opsum, int* n_terms,
                          int* n_groups, int* has_diag, int* all_real, uint64_t* mask, double* coef,
                          uint64_t* flip, uint32_t* first, uint32_t* count, uint32_t* check);

/* ------------------------------------------------------------ Hamiltonian
 * qkrylov_hamiltonian_create (c_api.h:81-83) with a precision (32: complex
 * float vectors as the reference C ABI, 64: complex double as the
 * reference's fp64 C++ API) and a CUDA device ordinal. */
qkrylov_hamiltonian_h qkrylov_hamiltonian_create_ex(qkrylov_basis_h basis, qkrylov_site_h site,
                                                   qkrylov_opsum_h opsum, int precision, int device);
int qkrylov_hamiltonian_precision(qkrylov_hamiltonian_h h);
int qkrylov_hamiltonian_all_real(qkrylov_hamiltonian_h h);
uint64_t qkrylov_hamiltonian_device_bytes(qkrylov_hamiltonian_h h);
/* The H.x kernel of this handle: 1 the two-site exchange kernel (spin
 * models in a single-charge sector), 2 the two-part kernel (operators whose
 * terms factorise over the sector split: Hubbard, t-J, fermion hops with
 * Jordan-Wigner signs), 3 the spin-product path (Hubbard-type operators with
 * N_up and N_dn conserved: T_up x 1 + 1 x T_dn + D in the (up, down) order,
 * the vector permuted at the boundary; block applies stay on the two-part
 * kernel), 0 the generic term-table kernel. */
int qkrylov_hamiltonian_kernel(qkrylov_hamiltonian_h h);
/* The CUDA stream (cudaStream_t) the library uses on the handle's device. */
void* qkrylov_hamiltonian_stream(qkrylov_hamiltonian_h h);

/* qkrylov_hamiltonian_apply_complex / _diagonal (c_api.h:94-100) on
 * double host arrays (64-bit Hamiltonians). */
int qkrylov_hamiltonian_apply_complex_f64(qkrylov_hamiltonian_h h, const double* x_complex, double* y_complex);
int qkrylov_hamiltonian_diagonal_complex_f64(qkrylov_hamiltonian_h h, double* diag_complex_out);

/* y = H x on device pointers of `dtype` (any precision handle; real dtypes
 * need a real operator), issued on `stream` (NULL: the library stream)
 * without synchronising.  MatrixFreeHamiltonian::apply(VectorView, VectorView)
 * (matrix_free_hamiltonian.hpp:38) as a C entry point. */
int qkrylov_hamiltonian_apply_device(qkrylov_hamiltonian_h h, int dtype, const void* x, void* y, void* stream);
int qkrylov_hamiltonian_diagonal_device(qkrylov_hamiltonian_h h, int dtype, void* diag, void* stream);
/* Row sharding of H.x over several GPUs (no counterpart in the reference;
 * it parallelises the row loop of matrix_free_hamiltonian.cpp:140-168
 * within one device).  qkrylov_b200_basis_shard_bounds writes nshards + 1
 * row bounds at sector-block boundaries (bounds[0] = 0, bounds[nshards] =
 * dim, shard k = [bounds[k], bounds[k+1]), rows as even as block
 * boundaries allow); host only, no GPU needed.
 * qkrylov_hamiltonian_apply_range_device computes rows [row_lo, row_hi) of
 * y = H x from the complete x (the other rows of y are not written); the
 * bounds must be block boundaries (QKRYLOV_ERROR_INVALID_ARG otherwise). */
int qkrylov_b200_basis_shard_bounds(qkrylov_basis_h basis, int nshards, uint64_t* bounds_out);
int qkrylov_hamiltonian_apply_range_device(qkrylov_hamiltonian_h h, int dtype, const void* x, void* y,
                                           uint64_t row_lo, uint64_t row_hi, void* stream);

/* The block apply's autotuner (no counterpart in the reference; it replaces
 * the one-vector loop of ftlm.cpp:140-157): the fastest timed launch in ms
 * for each shape it tried on this operator, dtype and block size R (32, 64
 * or 128), ms9[3*i + j] for lanes per row 32, 16, 8 (i) and tile code j
 * (CTA tiles of 256, 128, 512 rows); 0 where a shape was not timed or the
 * tuner has not run (it runs on the first batched FTLM or sweep). */
int qkrylov_b200_block_shape_timings(qkrylov_hamiltonian_h h, int dtype, int R, double* ms9);
/* Block H.X on R vectors stored row-interleaved (element (i, r) at
 * X[i*R + r]; R = 32, 64 or 128; device memory, 16-byte aligned, X != Y):
 * Y = H X in one pass that reads each row's terms and target ranks once for
 * all R vectors (the reference applies one vector at a time,
 * matrix_free_hamiltonian.cpp:140-168).  lanes_per_row 8, 16 or 32
 * (R / lanes <= 8) forces a shape, 0 the autotuned one (the first call with
 * 0 tunes on X and Y).  dots_out: NULL, or a host array of 2R doubles that
 * receives <X_r, Y_r> (the call then waits for the stream).  stream: NULL
 * for the library stream. */
int qkrylov_b200_apply_block_device(qkrylov_hamiltonian_h h, int dtype, int R, int lanes_per_row, const void* X,
                                    void* Y, double* dots_out, void* stream);

/* ------------------------------------------------------ device vector ops
 * Multi-vector dot out[2j..2j+1] = <V_j, x> = sum_i conj(V_j[i]) x[i] for
 * j < k (the reorthogonalisation coefficients of vector_ops.hpp:14-30
 * `dot`, k at once), FP64 accumulation, deterministic.  V: host array of k
 * device pointers; x, V_j: n elements of dtype on `device`; out: host
 * array of 2k doubles.  Runs on the library stream and waits for it. */
int qkrylov_b200_multi_dot(int device, int dtype, size_t n, int k, const void* const* V, const void* x,
                           double* out);

/* qkrylov_b200_multi_dot for callers that cannot let the library allocate
 * device memory (their memory is owned by another allocator's pool, or an
 * allocation or free would stall their streams).  No counterpart in the
 * reference.  Same inputs, output and arithmetic as qkrylov_b200_multi_dot,
 * issued on `stream` (NULL: the legacy default stream) and waited for; it
 * calls no cudaMalloc, cudaFree or allocating routine.  All scratch lives in
 * one fixed device array of about 129 KB per GPU, held until exit: k is
 * limited to 16 vectors per call (more is rejected with
 * QKRYLOV_ERROR_INVALID_ARG), calls share the array and must not overlap on
 * the GPU, and the first call on a device sets the array up (make it before
 * any stream capture). */
int qkrylov_b200_multi_dot_noalloc(int device, int dtype, size_t n, int k, const void* const* V, const void* x,
                                   double* out, void* stream);

/* -------------------------------------------------- double-precision solvers */
typedef struct {
  double energy;
  int iterations;
  int converged;
  int n_alpha;
  int n_beta;
} qkrylov_lanczos_result_f64_t;

/* lanczos_ground_state (lanczos.hpp:20-25).  start_complex: NULL for the
 * reference start vector, else dimension() complex doubles.  alphas and
 * betas (maxiter doubles each, may be NULL) receive the tridiagonal. */
int qkrylov_lanczos_ground_state_f64(qkrylov_hamiltonian_h h, int maxiter, double tol, const double* start_complex,
                                     qkrylov_lanczos_result_f64_t* result, double* eigenvector_complex,
                                     double* alphas, double* betas);
/* davidson_lowest (davidson.hpp:21-27) */
int qkrylov_davidson_lowest_f64(qkrylov_hamiltonian_h h, int n_eig, int max_subspace, double tol,
                                double* eigenvalues_out, double* eigenvectors_complex_out,
                                qkrylov_davidson_result_c_t* result_info);
/* continued_fraction_coeffs (dynamics.hpp:21-25) */
int qkrylov_continued_fraction_coeffs_f64(qkrylov_hamiltonian_h h, const double* phi0_complex, int n_iter,
                                          double* alphas_out, double* betas_out, double* norm_phi0_out,
                                          int* n_alpha_out, int* n_beta_out);
/* continued_fraction_coeffs with a checkpoint of its state, for long runs
 * that must survive an interruption.  No counterpart in the reference (its
 * examples/hdf5_storage.py stores final results only).  Starts from
 * phi0_complex, or, when resume_dir is not NULL, continues the run saved
 * there (phi0 is then ignored); runs until n_iter steps in total (or
 * beta < 1e-15); when save_dir is not NULL writes the state there as .npy
 * files numpy reads: alphas.npy, betas.npy, norm_phi0.npy, state.npy
 * ([steps, stopped]) and the current and previous Lanczos vectors v.npy,
 * v_prev.npy (complex128).  A run resumed from a checkpoint gives the same
 * coefficients, bit for bit, as one uninterrupted run.  alphas_out and
 * betas_out hold n_iter doubles; the directories must exist. */
int qkrylov_b200_cf_checkpointed(qkrylov_hamiltonian_h h, const double* phi0_complex, const char* resume_dir,
                                 int n_iter, const char* save_dir, double* alphas_out, double* betas_out,
                                 double* norm_phi0_out, int* n_alpha_out, int* n_beta_out);
/* evaluate_spectral_function (dynamics.hpp:28-38); betas has n-1 entries */
double qkrylov_evaluate_spectral_function_f64(const double* alphas, const double* betas, size_t n,
                                              double norm_phi0, double omega, double E0, double eta);
/* evaluate_spectral_function (dynamics.cpp:61-89) for ncols continued
 * fractions at n_omega frequencies in one call, evaluated on `device`
 * (one GPU thread per fraction and frequency, FP64).  Fraction c has its
 * alphas and betas at c*ld (betas: its first lengths[c]-1 entries),
 * lengths[c] <= ld coefficients (lengths NULL: ld each) and norm
 * norm_phi0[c] (NULL: 1); out[c*n_omega + k] = S_c(omegas[k]).  Host
 * arrays; waits for the result.  No counterpart in the reference (it
 * evaluates one frequency of one fraction per call). */
int qkrylov_b200_spectral_function_batch(int device, int ncols, int ld, const double* alphas, const double* betas,
                                         const int* lengths, const double* norm_phi0, size_t n_omega,
                                         const double* omegas, double E0, double eta, double* out);
/* Apply the operator an OpSum defines on a basis to a device vector, once:
 * y = O x with the reference's H.x convention (y[a] = sum over terms of
 * conj(amplitude) x[T a], matrix_free_hamiltonian.cpp:45-91 and 140-168),
 * without keeping a Hamiltonian handle; e.g. Sz(q)|psi> for a dynamical
 * structure factor, or with `expectation` (2 doubles, may be NULL) the
 * value <x|y> of a correlation function.  x, y: dim elements of dtype on
 * `device` (real dtypes need a real operator); waits for the result.  No
 * counterpart in the reference's C ABI. */
int qkrylov_b200_apply_operator(qkrylov_basis_h basis, qkrylov_site_h site, qkrylov_opsum_h opsum, int device,
                                int dtype, const void* x, void* y, double* expectation);
/* ftlm (ftlm.hpp:21-27) at n_beta inverse temperatures from one set of
 * random-vector tridiagonals; entry q equals ftlm(h, betas[q], ...). */
int qkrylov_ftlm_sweep_f64(qkrylov_hamiltonian_h h, int n_beta, const double* betas, int n_random, int n_steps,
                           double* Z_out, double* U_out, double* Cv_out);

/* ------------------------------------------------ mixed-precision Lanczos
 * No counterpart in the reference.  The iterate psi, its energy E and the
 * residual r = H psi - E psi are FP64 (float64 for a real operator,
 * complex128 otherwise; one FP64 apply per outer step).  Each correction
 * comes from a Lanczos pass on FP32 vectors (float32 / complex64 H.x and
 * vectors; alpha, beta, reorthogonalisation coefficients, norms and the
 * tridiagonal eigensolve in FP64) over the Krylov space of r kept
 * orthogonal to psi, followed by the Rayleigh-Ritz step on span{psi, v_1..
 * v_m}.  It stops when ||H psi - E psi|| / |E| <= tol; a pass stops when
 * its Ritz residual estimate drops below max(0.3 tol, 1e-6 |r| / |E|) or
 * after its length in steps (32 for the first pass, doubled after a pass
 * that cut the residual less than twentyfold, at most maxiter <= 511 and
 * half of the device's free memory); a pass that fails to halve the
 * residual switches the remaining passes to FP64.  Inside a pass the
 * Krylov vectors are kept semi-orthogonal by partial reorthogonalisation
 * (Simon 1984: orthogonalised against psi every step, against all stored
 * vectors only when the omega recurrence's estimate of their loss of
 * orthogonality exceeds the square root of the vectors' unit roundoff, and
 * at the step after); qkrylov_b200_lanczos_mixed_full below orthogonalises
 * every step against all of them.
 *   start: NULL for a random start generated on the GPU from `seed`
 *          (uniform in [-1, 1)), else dimension() elements of the FP32
 *          vector type, in host memory, or in device memory of the
 *          operator's GPU when start_on_device is non-zero.
 *   psi_out: NULL, or host memory for the normalised FP64 ground state.
 *   trace_*: NULL, or trace_cap entries receiving (step, energy or Ritz
 *          value, seconds since the call started) for every FP32 step and
 *          every FP64 residual evaluation. */
typedef struct {
  double energy;
  double residual;      /* explicit ||H psi - E psi|| / |E| of psi_out */
  double seconds_low;   /* wall time in FP32 passes (and start set-up) */
  double seconds_high;  /* wall time in FP64 applies, residuals and passes */
  int iterations_low;   /* FP32 Lanczos steps */
  int iterations_high;  /* FP64 Lanczos steps and residual applies */
  int restarts;         /* refinement passes (plain FP64: Lanczos runs) */
  int converged;
  int trace_len;
} qkrylov_b200_mixed_result_t;

int qkrylov_b200_lanczos_mixed(qkrylov_hamiltonian_h h, uint64_t seed, const void* start, int start_on_device,
                               int maxiter, double tol, qkrylov_b200_mixed_result_t* result, void* psi_out,
                               int trace_cap, int* trace_iteration, double* trace_energy, double* trace_seconds);

/* No counterpart in the reference.  qkrylov_b200_lanczos_mixed with every
 * step of every pass orthogonalised against psi and all the pass's stored
 * vectors (classical Gram-Schmidt, a second pass when a vector loses more
 * than 3/4 of its norm): the FP32-vector form with full
 * reorthogonalisation, same arguments and results. */
int qkrylov_b200_lanczos_mixed_full(qkrylov_hamiltonian_h h, uint64_t seed, const void* start,
                                    int start_on_device, int maxiter, double tol,
                                    qkrylov_b200_mixed_result_t* result, void* psi_out, int trace_cap,
                                    int* trace_iteration, double* trace_energy, double* trace_seconds);

/* Plain FP64 Lanczos with full reorthogonalisation from the start (FP64
 * vector type) or a random FP64 start, restarted from its Ritz vector (at
 * most 8 runs of up to maxiter steps) until the explicit residual meets
 * tol: the baseline the mixed form is timed against. */
int qkrylov_b200_lanczos_fp64(qkrylov_hamiltonian_h h, uint64_t seed, const void* start, int start_on_device,
                              int maxiter, double tol, qkrylov_b200_mixed_result_t* result, void* psi_out,
                              int trace_cap, int* trace_iteration, double* trace_energy, double* trace_seconds);

/* ---------------------------------------------------------- block Davidson
 * No counterpart in the reference (its davidson_lowest, davidson.hpp:21-27,
 * has no block size and keeps complex V and HV, 340 GB for Hubbard 4x4).
 * For real operators on float32 (precision 32) or float64 (64) vectors: a
 * seeded random start block of `block` vectors, corrections r / (diag -
 * theta) with the reference's clamp (davidson.cpp:171-175) for the
 * unconverged among the lowest `block` Ritz pairs, orthogonalised against
 * the basis (a second round when the first removed more than half of a
 * correction's squared norm); restart from the lowest 2*block Ritz vectors when the
 * basis would exceed max_subspace (3*block <= max_subspace <= 510).  Only
 * the basis is stored (H is applied again to the Ritz vectors for the
 * residuals).  Converged when the n_eig lowest residual norms
 * ||H u - theta u|| are below tol.  evecs: NULL or n_eig * dimension()
 * doubles (host, vector a at a * dimension()). */
typedef struct {
  int iterations;
  int applies;   /* H.x products */
  int restarts;
  int converged;
  double seconds;
} qkrylov_b200_davidson_info_t;

int qkrylov_b200_davidson_block(qkrylov_hamiltonian_h h, int precision, int n_eig, int block, int max_subspace,
                                double tol, uint64_t seed, int maxiter, double* evals, double* residuals,
                                double* evecs, qkrylov_b200_davidson_info_t* info);

/* ---------------------------------------------------------- batched FTLM
 * No counterpart in the reference (its ftlm, ftlm.hpp:21-27, runs one
 * complex Gaussian vector at a time and one temperature per call).
 * n_random (32, 64 or 128) seeded Rademacher (+-1) vectors advanced together
 * as one block: each of the n_steps Lanczos steps (the reference's
 * recurrence without reorthogonalisation, ftlm.cpp:24-53) is one block H.X
 * with fused column dots, one column update with fused FP64 norms and one
 * column scaling, with alpha and beta kept on the GPU; with use_graph the
 * steps are captured once as a CUDA graph.  The block H.X tile shape (lanes
 * per row) is autotuned on first use.  precision 32: float32 vectors
 * (complex64 for a complex operator), FP64 dots, norms and tridiagonals;
 * 64: float64 / complex128.  For each of the n_temps temperatures T (> 0):
 * logZ = log Z, U = <H>, Cv = beta^2 (<H^2> - <H>^2), beta = 1/T, with
 * Z = (1/R) sum_r sum_i |r|^2 z_0i^2 exp(-beta e_i) evaluated with the
 * lowest Ritz value as energy shift (no overflow at low T). */
typedef struct {
  double seconds;         /* whole call */
  double seconds_device;  /* the Lanczos steps (graph replay: CUDA events) */
  double e_min;           /* lowest Ritz value over all vectors */
  int lanes_per_row;      /* block H.X shape chosen by the autotuner */
  int graph;
  int vectors;
  int steps;
} qkrylov_b200_ftlm_info_t;

int qkrylov_b200_ftlm_block(qkrylov_hamiltonian_h h, int precision, int n_random, int n_steps, uint64_t seed,
                            int n_temps, const double* temps, double* logZ, double* U, double* Cv, int use_graph,
                            qkrylov_b200_ftlm_info_t* info);

/* The same random vectors (columns 0..n_vectors-1 of the n_random block)
 * run one at a time through the single-vector kernels: the one-vector
 * loop the batched form is measured against. */
int qkrylov_b200_ftlm_loop(qkrylov_hamiltonian_h h, int precision, int n_random, int n_steps, uint64_t seed,
                           int n_vectors, int n_temps, const double* temps, double* logZ, double* U, double* Cv,
                           qkrylov_b200_ftlm_info_t* info);

/* ------------------------------------------------------ learned warm start
 * No counterpart in the reference.  An MLP over the spin configurations of
 * a spin-1/2 basis and a coupling J2: inputs the nsites spins as +-1 (bit
 * set = +1) and J2, two hidden layers of 128 with GELU, outputs the
 * log-amplitude o0 and a sign logit o1; BF16 weights, FP32 accumulation.
 * Its start vector is phi(s) = M(s) exp(o0) tanh(o1) with M(s) =
 * (-1)^(number of up spins on odd sites), Marshall's sign rule.  Training
 * (forward, loss, backward, Adam; all on the GPU) fits o0 to log|psi| -
 * log max|psi| and o1 to the sign of psi relative to M on samples drawn by
 * |psi|^2 from each added ground state; per sample
 *   loss = (o0 - a)^2 + c_sign * softplus(-y o1).
 * Parameters (FP32): W1 [128][nsites+1], W2 [128][128], W3 [2][128], b1,
 * b2, b3 (20,098 values for 24 sites). */
/* ------------------------------------------------- block continued fraction
 * qkrylov's continued_fraction_coeffs (dynamics.cpp:12-59: normalise phi0,
 * three-term Lanczos without reorthogonalisation, stop at beta < 1e-15) for
 * n_vectors (32, 64 or 128) start vectors at once, e.g. Sz(q)|psi0> for
 * every momentum q: one block H.X with fused column dots and one column
 * recurrence per step, the n_steps (1..1000) steps captured as one CUDA
 * graph when use_graph.  start: row-interleaved dimension() x n_vectors
 * block (element (i, r) at i * n_vectors + r; float for precision 32,
 * double for 64; complex interleaved for complex operators, or for real
 * ones when complex_vectors != 0), in device memory when start_on_device,
 * else host memory; zero columns give empty fractions.  alphas, betas: n_vectors x n_steps doubles (vector r at
 * r * n_steps; betas[k] is the beta computed at step k); norms: |start_r|
 * (may be NULL); lengths: steps per vector, the last being the one whose
 * beta fell below 1e-15 when the recurrence stopped early (may be NULL).
 * No counterpart in the reference, which runs one start vector per call. */
int qkrylov_b200_cf_block(qkrylov_hamiltonian_h h, int precision, int complex_vectors, int n_vectors, int n_steps,
                          const void* start, int start_on_device, int use_graph, double* alphas, double* betas,
                          double* norms, int* lengths, qkrylov_b200_ftlm_info_t* info);

typedef struct qkrylov_b200_mlp_t* qkrylov_b200_mlp_h;

qkrylov_b200_mlp_h qkrylov_b200_mlp_create(qkrylov_basis_h basis, int device, uint64_t seed);
void qkrylov_b200_mlp_destroy(qkrylov_b200_mlp_h net);
size_t qkrylov_b200_mlp_num_params(qkrylov_b200_mlp_h net);
int qkrylov_b200_mlp_get_params(qkrylov_b200_mlp_h net, float* out);
int qkrylov_b200_mlp_set_params(qkrylov_b200_mlp_h net, const float* in);
/* Inference (qkrylov_b200_mlp_start_vector, qkrylov_b200_lanczos_warm) on
 * the tensor cores (on != 0, the default: tcgen05 MMAs with BF16 weights
 * and activations, FP32 accumulation in tensor memory) or on the CUDA cores
 * (FP32 activations, as in training). */
int qkrylov_b200_mlp_set_tensor_cores(qkrylov_b200_mlp_h net, int on);
/* A real ground state psi (dimension() doubles, host) at coupling j2. */
int qkrylov_b200_mlp_add_target(qkrylov_b200_mlp_h net, double j2, const double* psi);
/* `steps` Adam steps (learning rate lr with cosine decay to lr/20) on
 * minibatches of `batch` samples split evenly over the targets; loss_out:
 * NULL or `steps` doubles. */
int qkrylov_b200_mlp_train(qkrylov_b200_mlp_h net, int steps, int batch, double lr, uint64_t seed, double c_sign,
                           double* loss_out);
/* phi at coupling j2 over the whole basis (not normalised), FP32, into host
 * memory or (out_on_device) device memory of the network's GPU. */
int qkrylov_b200_mlp_start_vector(qkrylov_b200_mlp_h net, double j2, float* out, int out_on_device);
/* Mean loss and its gradient (layout of the parameters) over n explicit
 * samples: states (host), j2 per sample, targets (a, y, weight) per sample. */
int qkrylov_b200_mlp_loss_grad(qkrylov_b200_mlp_h net, int n, const uint64_t* states, const double* j2,
                               const float* targets, double c_sign, float* grad_out, double* loss_out);
/* qkrylov_b200_lanczos_mixed started from the network's start vector at
 * j2 (built on the GPU, its time included in seconds_low and returned in
 * seconds_inference).  The operator must be real and act on the network's
 * basis. */
int qkrylov_b200_lanczos_warm(qkrylov_hamiltonian_h h, qkrylov_b200_mlp_h net, double j2, int maxiter, double tol,
                              qkrylov_b200_mixed_result_t* result, double* seconds_inference);

/* ---------------------------------------------------- batched coupling sweep
 * No counterpart in the reference (its lanczos_ground_state, lanczos.hpp:
 * 11-25, solves one Hamiltonian at a time).  Ground states of
 * H(g) = H0 + g H1 for n_couplings (1..128) values of g at once: h0 and h1
 * are real operators on the same basis (e.g. the J1 and the unit-J2 parts of
 * a J1-J2 chain).  The couplings are the columns of one row-interleaved
 * FP64 block (32, 64 or 128 columns; extra columns repeat the last
 * coupling); each step is one block H.X per operator (the row's tables read
 * once for all columns), a column axpy forming H(g) X, and the three-term
 * update; every column is kept semi-orthogonal against its own Krylov
 * vectors by partial reorthogonalisation (Simon's estimates, classical
 * Gram-Schmidt of the whole block when any column needs it).
 * Each column restarts from its Ritz vector after at most pass_len (2..128)
 * steps; the run ends when every column's explicit residual
 * |H psi - E psi| / |E| is <= tol or after max_passes (1..64) passes.  Start
 * block: uniform [-1, 1) from seed; with a warm-start network (net, on the
 * same basis, NULL for none) column q starts from the network's start
 * vector at coupling g_q (its coupling input is g; inference time is
 * included in seconds and reported in seconds_inference).  Device memory:
 * (pass_len + 4) blocks of dimension() x block doubles.  energies,
 * residuals, converged: n_couplings entries (residuals, converged and info
 * may be NULL). */
typedef struct {
  int block;          /* columns of the block: 32, 64 or 128 */
  int steps;          /* Lanczos steps (all columns advance together) */
  int passes;         /* residual checks (restarts + 1) */
  int applies;        /* block H.X products (two per step and check) */
  int lanes_per_row;  /* tuned block H.X tile shape */
  double seconds;
  double seconds_inference;  /* start vectors from the network (0 without one) */
} qkrylov_b200_sweep_info_t;

int qkrylov_b200_lanczos_sweep(qkrylov_hamiltonian_h h0, qkrylov_hamiltonian_h h1, int n_couplings,
                               const double* couplings, int pass_len, int max_passes, double tol, uint64_t seed,
                               qkrylov_b200_mlp_h net, double* energies, double* residuals, int* converged,
                               qkrylov_b200_sweep_info_t* info);

#ifdef __cplusplus
}
#endif

#endif /* QKRYLOV_B200_H */
