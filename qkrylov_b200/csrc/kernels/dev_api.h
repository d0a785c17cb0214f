/* Internal C ABI between the C++ host layer and the CUDA kernels of
 * libqkrylov_b200.so.  Plain pointers, sizes and streams only; every call
 * returns 0 or a negative status (QKD_*) and never throws.
 *
 * Vector dtypes: complex128 (interleaved double pairs), complex64, float64,
 * float32.  Real dtypes are only valid for operators whose compiled
 * coefficients are all real.
 */
#ifndef QKRYLOV_B200_DEV_API_H
#define QKRYLOV_B200_DEV_API_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { QKD_OK = 0, QKD_EINVAL = -1, QKD_ECUDA = -3, QKD_ENOMEM = -4, QKD_ETIMEOUT = -5 };
typedef enum { QK_C128 = 0, QK_C64 = 1, QK_F64 = 2, QK_F32 = 3 } qk_dtype;

static inline size_t qk_dtype_size(qk_dtype t) {
  return t == QK_C128 ? 16 : (t == QK_C64 || t == QK_F64) ? 8 : 4;
}
static inline int qk_dtype_complex(qk_dtype t) { return t == QK_C128 || t == QK_C64; }

/* One compiled term: valid iff (s & cmask) == cval; value
 * (wre + i wim) * (-1)^popcount(s & smask). */
typedef struct { uint64_t cmask, cval, smask; double wre, wim; } qk_term_t;
/* Terms [first, first+count) share the target s ^ flip. */
typedef struct { uint64_t flip; uint32_t first, count, check, pad; } qk_group_t;
/* A run of consecutive rows inside one sector block. */
typedef struct { uint64_t row0; uint32_t h, lstart, count, pad; } qk_tile_t;

typedef struct {
  int nbits, L;
  uint64_t dim;
  const uint64_t* A; uint64_t nA;         /* block offsets | need key << 56 */
  const uint32_t* B; uint64_t nB;         /* low ranks | key << 24 */
  const uint32_t* llist; uint64_t nllist; /* low parts grouped by key */
  const uint32_t* key_off; uint32_t nkeys;
  const qk_term_t* terms; uint32_t nterms;
  const qk_group_t* groups; uint32_t ngroups;
  int has_diag, all_real;
  int pair_sites;  /* 1: two bits per site, up-spin at the even bit (Hubbard, t-J) */
} qk_plan_desc;

typedef struct qk_plan qk_plan;
typedef struct qk_workspace qk_workspace;

int qkd_plan_create(const qk_plan_desc* d, int device, qk_plan** out);
int qkd_plan_destroy(qk_plan* p);
uint64_t qkd_plan_dim(const qk_plan* p);
int qkd_plan_all_real(const qk_plan* p);
size_t qkd_plan_device_bytes(const qk_plan* p);

/* 0: use specialised kernels where the operator qualifies (default);
 * 1: generic kernel only; 2: as 0 without the per-die work queues of the
 * row kernel; 3: as 0 without the spin-product path of Hubbard-type
 * operators (for comparisons). */
int qkd_set_kernel_policy(int policy);
/* Dies of the current device as measured by the row kernels' topology probe
 * (2 or 1) and the SMs on each. */
int qkd_die_count(int* sms_die0, int* sms_die1);
/* 1 when applies of this plan run the specialised two-site spin kernel. */
int qkd_plan_kernel(const qk_plan* p);

/* y = H x (device pointers, n = dim elements of dtype t). */
int qkd_apply(const qk_plan* p, qk_dtype t, const void* x, void* y, cudaStream_t s);
/* Rows [row_lo, row_hi) of y = H x (x complete, other rows of y untouched);
 * the bounds must be sector-block boundaries. */
int qkd_apply_range(const qk_plan* p, qk_dtype t, const void* x, void* y, uint64_t row_lo, uint64_t row_hi,
                    cudaStream_t s);
/* y = H x and dot_out[0..1] = <x, y> (device memory) in the same pass. */
int qkd_apply_dot(const qk_plan* p, qk_workspace* w, qk_dtype t, const void* x, void* y,
                  double* dot_out, cudaStream_t s);
/* Block form: X, Y hold nvec vectors, vector v at X + v*ldx elements. */
int qkd_apply_block(const qk_plan* p, qk_dtype t, int nvec, const void* X, size_t ldx, void* Y,
                    size_t ldy, cudaStream_t s);
/* Block apply on R vectors stored row-interleaved (element (i, r) at
 * i*R + r; R = 32, 64 or 128): Y = H X and, if dots != NULL, dots[2r..2r+1]
 * = <X_r, Y_r> (device memory).  lanes_per_row 8, 16 or 32 (R / lanes <= 8)
 * sets the tile shape; 0 uses the autotuned shape (32 before tuning).
 * diag: NULL, or H's diagonal (dtype t, from qkd_diagonal) used instead of
 * walking the diagonal terms.  X, Y 16-byte aligned. */
int qkd_apply_rows(const qk_plan* p, qk_workspace* w, qk_dtype t, int R, int lanes_per_row, const void* X,
                   void* Y, const void* diag, double* dots, cudaStream_t s);
/* Y += diag(g) (H X) column by column (g: R device doubles), with dots =
 * <X_r, Y_r> of the result, on the row-kernel tables; QKD_EINVAL for plans
 * without them (the caller then applies into a separate block). */
int qkd_apply_rows_acc(const qk_plan* p, qk_workspace* w, qk_dtype t, int R, int lanes_per_row, const void* X,
                       void* Y, const double* g, double* dots, cudaStream_t s);
/* Time every valid lanes-per-row shape on X, Y (three launches each) and
 * keep the fastest for (t, R) in the plan; *chosen receives it.  Waits for
 * the stream. */
int qkd_tune_rows(qk_plan* p, qk_workspace* w, qk_dtype t, int R, const void* X, void* Y, const void* diag,
                  cudaStream_t s, int* chosen);
/* The same for the accumulating form qkd_apply_rows_acc (Y is scratch). */
int qkd_tune_rows_acc(qk_plan* p, qk_workspace* w, qk_dtype t, int R, const void* X, void* Y, const double* g,
                      cudaStream_t s, int* chosen);
/* The tuned lanes per row for (t, R), 0 before tuning. */
/* Block Davidson forms (t = QK_F64 or QK_F32; V, X: device arrays of device
 * pointers; nx <= 8).  qkd_multi_dot: out[2*(i*8 + a)] = <V_i, X_a> for
 * i < m, a < nx (out: 16 * (m rounded up to 8) device doubles; FP64,
 * deterministic).
 * qkd_multi_update: X_a = sum_i c[i*nx + a] V_i (accumulate = 0) or
 * X_a -= sum_i c[i*nx + a] V_i (accumulate = 1); c: m*nx device doubles. */
int qkd_multi_dot(qk_workspace* w, qk_dtype t, size_t n, int m, const void* const* V, int nx, const void* const* X,
                  double* out, cudaStream_t s);
int qkd_multi_update(qk_dtype t, size_t n, int m, const void* const* V, const double* c, int nx, void* const* X,
                     int accumulate, cudaStream_t s);
int qkd_rows_shape(const qk_plan* p, qk_dtype t, int R);
/* The tuner's fastest launch (ms) for lanes per row 32, 16, 8 (rows) x tile
 * code 0, 1, 2 (columns), row-major; 0 where a shape was not timed. */
int qkd_rows_timings(const qk_plan* p, qk_dtype t, int R, float* ms9);
/* diag[i] = <i|H|i> as dtype t. */
int qkd_diagonal(const qk_plan* p, qk_dtype t, void* diag, cudaStream_t s);
/* Number of kernel launches issued by this library since load (for the
 * bench's launch count). */
uint64_t qkd_launch_count(void);

/* ---------------------------------------------------------------- vectors
 * Scalars are complex doubles {re, im}.  Reductions accumulate in FP64 and
 * write their result to `out` (device memory), deterministic for a given
 * n: each block sums a fixed slice, the last block adds the partials in
 * block order.  `ws` is a workspace from qkd_workspace_create(). */
int qkd_workspace_create(int device, qk_workspace** out);
int qkd_workspace_destroy(qk_workspace* w);

int qkd_fill(qk_dtype t, size_t n, void* x, double re, double im, cudaStream_t s);
int qkd_copy(qk_dtype t, size_t n, const void* x, void* y, cudaStream_t s);
int qkd_convert(qk_dtype tin, const void* x, qk_dtype tout, void* y, size_t n, cudaStream_t s);
/* x *= (re + i im) */
int qkd_scal(qk_dtype t, size_t n, double re, double im, void* x, cudaStream_t s);
/* y += (re + i im) x */
int qkd_axpy(qk_dtype t, size_t n, double re, double im, const void* x, void* y, cudaStream_t s);
/* y = a x + b y, complex host scalars */
int qkd_axpby(qk_dtype t, size_t n, double are, double aim, const void* x, double bre, double bim,
              void* y, cudaStream_t s);
/* out[0..1] = sum conj(x_i) y_i, written to device memory `out` */
int qkd_dot(qk_workspace* w, qk_dtype t, size_t n, const void* x, const void* y, double* out,
            cudaStream_t s);
/* Optionally update x first:  x <- x - sum_{m<M} a_m U_m  (M <= 4; U and
 * the complex coefficients a[2M] are HOST arrays), storing x back; then
 * out[2j..2j+1] = <V_j, x> for j < k (V: DEVICE array of k pointers).  One
 * pass over U, V and x. */
int qkd_update_mdot(qk_workspace* w, qk_dtype t, size_t n, int M, const void* const* U,
                    const double* a, int k, const void* const* V, void* x, double* out,
                    cudaStream_t s);
/* x <- x - sum_{j<k} c_j V_j (c: 2k device doubles); if nrm2 != NULL also
 * writes ||x||^2 of the stored result to nrm2[0] (and 0 to nrm2[1]). */
int qkd_mupdate(qk_workspace* w, qk_dtype t, size_t n, int k, const void* const* V,
                const double* c, void* x, double* nrm2, cudaStream_t s);
/* y = x * scale where scale = 1 / sqrt(nrm2[0]) is read on the device. */
int qkd_normalize_into(qk_dtype t, size_t n, const double* nrm2, const void* x, void* y,
                       cudaStream_t s);
/* Davidson correction t = r / (diag - lambda) with the reference's clamp. */
int qkd_dav_precond(qk_dtype t, size_t n, const void* diag, double lambda, const void* r, void* out,
                    cudaStream_t s);
/* Seeded counter-based random vector: kind 0 uniform in [-1, 1) (real and
 * imaginary parts), kind 1 Rademacher +-1 (real). */
int qkd_random(qk_dtype t, size_t n, uint64_t seed, int kind, void* x, cudaStream_t s);
/* x (dtype tx) = sum_{j<k} c_j V_j (dtype tv), c: 2k device doubles. */
int qkd_combine(qk_dtype tv, size_t n, int k, const void* const* V, const double* c, qk_dtype tx, void* x,
                cudaStream_t s);
/* ------------------------------------------------- row-interleaved blocks
 * R vectors of n elements, element (i, r) at i*R + r; R divides 256.
 * W_r <- W_r - a_r V_r - b_r Vp_r for every column r (a: 2R device doubles,
 * complex; b: R device doubles, real; V / Vp with a / b may be NULL), then
 * nrm2[2r] = |W_r|^2 (device, 2R doubles; odd entries 0). */
int qkd_block_update(qk_workspace* w, qk_dtype t, size_t n, int R, const void* V, const double* a, const void* Vp,
                     const double* b, void* W, double* nrm2, cudaStream_t s);
/* One step of R Lanczos recurrences on unnormalised vectors U (v_k = s_k U_k):
 * with raw dots d_r = <U_k,r, Y_r> of Y = H U_k, alpha_r = s_k^2 Re d_r and
 *   W_r = s_k Y_r - alpha_r s_k U_k,r - beta_{k-1},r s_{k-1},r U_{k-1},r
 * written over Y (Ukm1 / beta_prev / s_prev NULL at the first step); then
 * beta_k,r = |W_r|, s_{k+1},r = 1 / beta_k,r (0 and len[r] = min(len[r],
 * step + 1) when beta < 1e-15).  s: scales by step (s[k*R + r]); alpha_out,
 * beta_out: R doubles each of this step (device). */
int qkd_block_lanczos(qk_workspace* w, qk_dtype t, size_t n, int R, const void* Uk, const void* Ukm1,
                      const double* dots, const double* beta_prev, const double* s_prev, const double* s_k,
                      double* s_next, void* Y, double* alpha_out, double* beta_out, int* len, int step,
                      cudaStream_t s);
/* beta_r = sqrt(nrm2[2r]); W_r *= 1 / beta_r, or W_r = 0 and
 * len[r] = min(len[r], step + 1) when beta_r < 1e-15; beta_out[r] = beta_r. */
int qkd_block_scale(qk_dtype t, size_t n, int R, const double* nrm2, void* W, double* beta_out, int* len, int step,
                    cudaStream_t s);
/* out (n elements) = column c of the block X. */
int qkd_block_column(qk_dtype t, size_t n, int R, const void* X, int c, void* out, cudaStream_t s);
/* Column-wise kernels of the batched coupling sweep on real blocks (t =
 * QK_F64 or QK_F32; R divides 256).  Results are column sums reduced in a
 * fixed order from per-CTA partials: partials (device) must hold
 * count * qkd_block_partials_grid(n, R) doubles, count = nv * R for
 * qkd_block_mdot and R otherwise (partials_cap = its size).  Outputs use
 * the (re, im) layout out[2 o], out[2 o + 1] = 0.  V: device array of nv
 * (<= 192) device pointers to blocks.
 *   mdot:      out[2 (j R + c)] = <V_j[:, c], W[:, c]>
 *   mcomb:     W[:, c] = (keep ? W[:, c] : 0) - sum_j coef[2 (j R + c)] V_j[:, c];
 *              nrm2 (may be NULL) = column norms^2 of the result
 *   axpy_cols: Y0[:, c] += g[c] Y1[:, c]; dots = <X[:, c], Y0[:, c]> */
int qkd_block_partials_grid(size_t n, int R);
/* Column c of the block dst (dtype td) = the n-element vector src (dtype
 * ts); (ts, td) = (f32, f64), (f64, f64) or (f32, f32). */
int qkd_block_put_column(qk_dtype ts, const void* src, size_t n, int R, int c, qk_dtype td, void* dst,
                         cudaStream_t s);
int qkd_block_mdot(qk_dtype t, size_t n, int R, int nv, const void* const* V, const void* W, double* partials,
                   size_t partials_cap, double* out, cudaStream_t s);
int qkd_block_mcomb(qk_dtype t, size_t n, int R, int nv, const void* const* V, const double* coef, int keep, void* W,
                    double* partials, size_t partials_cap, double* nrm2, cudaStream_t s);
int qkd_block_axpy_cols(qk_dtype t, size_t n, int R, const double* g, const void* Y1, void* Y0, const void* X,
                        double* partials, size_t partials_cap, double* dots, cudaStream_t s);
/* Device scratch of the workspace: 2*kMaxK+16 doubles for small results. */
double* qkd_workspace_results(qk_workspace* w);
/* S(omega) of ncols continued fractions (column c: alphas/betas at c*ld,
 * len[c] coefficients, NULL: ld; norm nrm[c], NULL: 1) at nw frequencies,
 * the reference's evaluate_spectral_function per pair; out[c*nw + k].
 * Device pointers. */
int qkd_spectral_batch(const double* alphas, const double* betas, const int* len, int ncols, int ld,
                       const double* nrm, const double* omega, size_t nw, double E0, double eta, double* out,
                       cudaStream_t s);

#ifdef __cplusplus
}
#endif
#endif
