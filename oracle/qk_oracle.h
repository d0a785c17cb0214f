/* CPU restatement of qkrylov's matrix-free H.x path and the Krylov solvers
 * above it, used ONLY as the parity checker by tests/, by
 * __graft_entry__.smoke() and as the timed CPU baseline in bench.py.  The
 * product library never links it.
 *
 * Every function restates the reference algorithm it names (file:line in the
 * qkrylov sources).  Complex vectors are interleaved doubles [re, im, ...].
 * Sector array sec[10] = use_sz, sz2, use_nup, nup, use_ndn, ndn, use_n, n,
 * use_nb, nb (include/qkrylov/symmetry/sector.hpp:10-41).
 * Site kinds: 0 spin-1/2, 1 spinless fermion, 2 Hubbard, 3 t-J.
 * Status codes: 0 ok, -1 invalid argument, -2 exception (qko_last_error()).
 */
#ifndef QK_ORACLE_H
#define QK_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

const char* qko_last_error(void);

/* src/sites/{spinhalf,fermion,hubbard,tj}_site.cpp Site::apply */
int qko_site_apply(int kind, const char* op, int site, uint64_t state,
                   int* valid, uint64_t* new_state, double* me /*[2]*/);

/* src/basis/*_basis.cpp: ascending list of sector states */
int64_t qko_basis_count(int kind, int nsites, const int* sec);
int qko_basis_states(int kind, int nsites, const int* sec, uint64_t* out);

/* MatrixFreeHamiltonian (src/hamiltonian/matrix_free_hamiltonian.cpp) */
void* qko_ham_create(int kind, int nsites, const int* sec, int nterms, const double* coef,
                     const int* nfac, const char* const* ops, const int* sites);
void qko_ham_destroy(void* h);
uint64_t qko_ham_dim(void* h);
int qko_ham_states(void* h, uint64_t* out);
int qko_ham_apply(void* h, const double* x, double* y);
int64_t qko_ham_coo_count(void* h);
int qko_ham_coo(void* h, int64_t* rows, int64_t* cols, double* vals);
int qko_ham_diagonal(void* h, double* d);

/* Reference random streams (libstdc++ mt19937 + distributions, the imaginary
 * part drawn before the real part as GCC evaluates KComplex(d(rng), d(rng))). */
int qko_lanczos_start(uint64_t dim, double* v);             /* lanczos.cpp:115-119 */
int qko_ftlm_vectors(uint64_t dim, int n_random, double* v); /* ftlm.cpp:133-142 */

/* src/solvers/lanczos.cpp:101-202 (+ alphas/betas it accumulates) */
int qko_lanczos(void* h, int maxiter, double tol, double* energy, int* iters, int* conv,
                double* evec, double* alphas, double* betas, int* n_alpha, int* n_beta);
/* src/solvers/davidson.cpp:86-227 */
int qko_davidson(void* h, int n_eig, int max_subspace, double tol, double* evals,
                 double* evecs, int* n_out, int* iters, int* conv);
/* src/solvers/dynamics.cpp:12-59 */
int qko_cf(void* h, const double* phi0, int n_iter, double* alphas, double* betas,
           double* norm_phi0, int* n_alpha, int* n_beta);
/* src/solvers/dynamics.cpp:61-89 */
double qko_spectral(const double* alphas, const double* betas, size_t n, double norm_phi0,
                    double omega, double E0, double eta);
/* src/solvers/ftlm.cpp:122-170 */
int qko_ftlm(void* h, double beta, int n_random, int n_steps, double* Z, double* U, double* Cv);
/* ftlm.cpp:24-53 from a caller-given start vector: the tridiagonal only */
int qko_ftlm_tridiag(void* h, const double* v_start, int n_steps, double* alphas,
                     double* betas, int* n_alpha, int* n_beta);
/* lanczos.cpp:25-98 / ftlm.cpp:61-119 (the reference's implicit QL sweeps) */
int qko_tridiag_eig(const double* alphas, const double* betas, int n, double* evals,
                    double* first_comp);
/* davidson.cpp:22-82 (Jacobi rotations on a small Hermitian matrix) */
int qko_jacobi_eig(const double* H /*n*n complex, row major*/, int n, double* evals,
                   double* evecs /*n*n complex, evecs[k*n+j] = component j of vector k*/);

#ifdef __cplusplus
}
#endif
#endif
