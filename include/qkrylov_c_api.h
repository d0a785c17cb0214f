/* qkrylov C ABI, served by libqkrylov_b200.so on NVIDIA B200 (sm_100a).
 *
 * Every declaration below is the entry point of the same name in qkrylov's
 * include/qkrylov/c_api.h (the line range is given with each group), with
 * the same argument meaning, float precision, status codes and handle
 * ownership, so its FFI callers (the Julia package's ccall wrappers under
 * bindings/julia/src) bind this library unchanged.  The main difference in
 * behaviour is that qkrylov_hamiltonian_diagonal returns real diagonal
 * entries from device memory correctly on GPU builds; the others are
 * noted at the declarations they concern.
 *
 * Extended entry points (double precision, device pointers, batched and
 * mixed-precision solvers) are in qkrylov_b200.h.
 */
#ifndef QKRYLOV_C_API_H
#define QKRYLOV_C_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (c_api.h:14-16) */
#define QKRYLOV_SUCCESS 0
#define QKRYLOV_ERROR_INVALID_ARG -1
#define QKRYLOV_ERROR_EXCEPTION -2

/* Opaque handles (c_api.h:21-25) */
typedef struct qkrylov_sector_t* qkrylov_sector_h;
typedef struct qkrylov_basis_t* qkrylov_basis_h;
typedef struct qkrylov_site_t* qkrylov_site_h;
typedef struct qkrylov_opsum_t* qkrylov_opsum_h;
typedef struct qkrylov_hamiltonian_t* qkrylov_hamiltonian_h;

/* Sector (c_api.h:30-39) */
qkrylov_sector_h qkrylov_sector_create(void);
void qkrylov_sector_destroy(qkrylov_sector_h sector);
int qkrylov_sector_set_sz(qkrylov_sector_h sector, int sz2);
int qkrylov_sector_set_hubbard_particles(qkrylov_sector_h sector, int nup, int ndn);
int qkrylov_sector_set_n(qkrylov_sector_h sector, int n);
int qkrylov_sector_set_nb(qkrylov_sector_h sector, int nb);
int qkrylov_sector_get_sz(qkrylov_sector_h sector, int* sz2_out, int* active_out);
int qkrylov_sector_get_hubbard_particles(qkrylov_sector_h sector, int* nup_out, int* ndn_out, int* active_out);
int qkrylov_sector_get_n(qkrylov_sector_h sector, int* n_out, int* active_out);
int qkrylov_sector_get_nb(qkrylov_sector_h sector, int* nb_out, int* active_out);

/* Basis (c_api.h:44-53) */
qkrylov_basis_h qkrylov_spinhalf_basis_create(int num_sites, qkrylov_sector_h sector);
qkrylov_basis_h qkrylov_fermion_basis_create(int num_sites, qkrylov_sector_h sector);
qkrylov_basis_h qkrylov_hubbard_basis_create(int num_sites, qkrylov_sector_h sector);
qkrylov_basis_h qkrylov_tj_basis_create(int num_sites, qkrylov_sector_h sector);
void qkrylov_basis_destroy(qkrylov_basis_h basis);
uint64_t qkrylov_basis_dimension(qkrylov_basis_h basis);
int qkrylov_basis_nsites(qkrylov_basis_h basis);
uint64_t qkrylov_basis_state(qkrylov_basis_h basis, uint64_t index);
int64_t qkrylov_basis_index(qkrylov_basis_h basis, uint64_t state_bitstring);
int qkrylov_basis_contains(qkrylov_basis_h basis, uint64_t state_bitstring);

/* Site (c_api.h:58-62) */
qkrylov_site_h qkrylov_spinhalf_site_create(void);
qkrylov_site_h qkrylov_fermion_site_create(void);
qkrylov_site_h qkrylov_hubbard_site_create(void);
qkrylov_site_h qkrylov_tj_site_create(void);
void qkrylov_site_destroy(qkrylov_site_h site);

/* OpSum (c_api.h:67-76) */
qkrylov_opsum_h qkrylov_opsum_create(void);
void qkrylov_opsum_destroy(qkrylov_opsum_h opsum);
int qkrylov_opsum_clear(qkrylov_opsum_h opsum);
int qkrylov_opsum_add_term_1body(qkrylov_opsum_h opsum, float coeff_real, float coeff_imag, const char* op1,
                                 int site1);
int qkrylov_opsum_add_term_2body(qkrylov_opsum_h opsum, float coeff_real, float coeff_imag, const char* op1,
                                 int site1, const char* op2, int site2);
int qkrylov_opsum_add_term_nbody(qkrylov_opsum_h opsum, float coeff_real, float coeff_imag, int n_factors,
                                 const char** ops, const int* sites);

/* Matrix-free Hamiltonian (c_api.h:81-100).  Vectors are host arrays of
 * dimension() complex floats.  Differences a caller can see: an unknown
 * operator name, or a site whose bit would not fit a 64-bit state, makes
 * qkrylov_hamiltonian_create return NULL (the reference fails at the first
 * state that reaches the factor); the host-pointer applies reuse device
 * staging buffers held by the handle, so calls on one handle are
 * serialised; qkrylov_hamiltonian_diagonal copies the diagonal from device
 * memory (the reference reads a device View from the host). */
qkrylov_hamiltonian_h qkrylov_hamiltonian_create(qkrylov_basis_h basis, qkrylov_site_h site,
                                                qkrylov_opsum_h opsum);
void qkrylov_hamiltonian_destroy(qkrylov_hamiltonian_h h);
uint64_t qkrylov_hamiltonian_dimension(qkrylov_hamiltonian_h h);
int qkrylov_hamiltonian_apply(qkrylov_hamiltonian_h h, const float* x_real, const float* x_imag, float* y_real,
                              float* y_imag);
int qkrylov_hamiltonian_apply_complex(qkrylov_hamiltonian_h h, const float* x_complex, float* y_complex);
int qkrylov_hamiltonian_diagonal(qkrylov_hamiltonian_h h, float* diag_out);

/* Solvers (c_api.h:105-168) */
typedef struct {
  float energy;
  int iterations;
  int converged;
} qkrylov_lanczos_result_c_t;

typedef struct {
  int iterations;
  int converged;
} qkrylov_davidson_result_c_t;

int qkrylov_lanczos_ground_state(qkrylov_hamiltonian_h h, int maxiter, float tol,
                                 qkrylov_lanczos_result_c_t* result);
int qkrylov_lanczos_ground_state_complex(qkrylov_hamiltonian_h h, int maxiter, float tol,
                                         qkrylov_lanczos_result_c_t* result, float* eigenvector_complex);
int qkrylov_davidson_lowest_complex(qkrylov_hamiltonian_h h, int n_eig, int max_subspace, float tol,
                                    float* eigenvalues_out, float* eigenvectors_complex_out,
                                    qkrylov_davidson_result_c_t* result_info);
int qkrylov_continued_fraction_coeffs_complex(qkrylov_hamiltonian_h h, const float* phi0_complex, int n_iter,
                                              float* alphas_out, float* betas_out, float* norm_phi0_out,
                                              int* num_coeffs_out);
float qkrylov_evaluate_spectral_function(const float* alphas, const float* betas, size_t n, float norm_phi0,
                                         float omega, float E0, float eta);

typedef struct {
  float beta;
  float partition_function;
  float internal_energy;
  float specific_heat;
} qkrylov_ftlm_result_c_t;

int qkrylov_ftlm(qkrylov_hamiltonian_h h, float beta, int n_random, int n_steps, qkrylov_ftlm_result_c_t* result);

#ifdef __cplusplus
}
#endif

#endif /* QKRYLOV_C_API_H */
