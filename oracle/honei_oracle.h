/* honei_oracle.h -- plain-C restatement of the HONEI sparse-solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load this; the product never does.
 *
 * Parity pin: every routine is checked bit-for-bit against the reference's own CPU path
 * (oracle/_ref/libhonei_ref.so, compiled from the unmodified HONEI sources) and against the
 * FEATFLOW2 fixtures the reference's tests use (tests/golden, tests/test_oracle_pin.py).
 *
 * Matrices use the reference ELL layout (honei/la/sparse_matrix_ell-impl.hh:75-122):
 * entry k of row r lives at (k % T) + r*T + (k / T)*stride, Arl[r] = ceil(nnz_r / T),
 * Aj are 64-bit column indices.  All arithmetic is one IEEE rounding per operation, in the
 * order the reference source states it (build with -ffp-contract=off).
 */
#ifndef HONEI_ORACLE_H
#define HONEI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint64_t rows, cols, stride, ncpr, threads;
    const uint64_t *Aj;
    const void *Ax;       /* double* or float* */
    const uint64_t *Arl;
} ora_ell;

/* SparseMatrixCSR<DT> (honei/la/sparse_matrix_csr.hh): Ar[rows + 1] block offsets, Aj[nblocks]
 * the first column of each block, Ax[nblocks * blocksize] (csr::blocksize values per block). */
typedef struct {
    uint64_t rows, cols, blocksize;
    const uint64_t *Ar, *Aj;
    const void *Ax;       /* double* or float* */
} ora_csr;

/* ---- BLAS-1 and SpMV (f64 / f32) ---- */
void   ora_spmv_f64(const ora_ell *A, const double *x, double *y);
void   ora_spmv_f32(const ora_ell *A, const float *x, float *y);
void   ora_defect_f64(const ora_ell *A, const double *b, const double *x, double *r);
void   ora_defect_f32(const ora_ell *A, const float *b, const float *x, float *r);
/* Product<tags::CPU>(DV, SparseMatrixCSR, DV) (honei/la/product.hh:209-242): per row, over its
 * blocks and their lanes in order, sum += Ax * x for lanes whose column is < cols; Defect
 * (honei/math/defect.hh:386-419): r = rhs - that sum. */
void   ora_csr_spmv_f64(const ora_csr *A, const double *x, double *y);
void   ora_csr_spmv_f32(const ora_csr *A, const float *x, float *y);
void   ora_csr_defect_f64(const ora_csr *A, const double *rhs, const double *x, double *r);
void   ora_csr_defect_f32(const ora_csr *A, const float *rhs, const float *x, float *r);
/* BandedMatrixQx<Q1Type> (honei/la/banded_matrix_qx.hh): nine bands of n values in the
 * Q1BandIndex order LL, LD, LU, DL, DD, DU, UL, UD, UU (honei/la/band_type.hh); root =
 * floor(sqrt(n)).  y = A x as Product<tags::CPU> (honei/la/product.hh:371-404); r = b - A x as
 * Defect<tags::CPU> (honei/math/defect.hh:194-199: the product, then Difference). */
void   ora_q1band_spmv_f64(uint64_t n, const double *const *band, const double *x, double *y);
void   ora_q1band_spmv_f32(uint64_t n, const float *const *band, const float *x, float *y);
void   ora_q1band_defect_f64(uint64_t n, const double *const *band, const double *b, const double *x, double *r);
void   ora_q1band_defect_f32(uint64_t n, const float *const *band, const float *b, const float *x, float *r);
/* Geometric transfers of (2^k + 1)^2 grids: Prolongation<Tag, methods::NONE>
 * (honei/math/prolongation.hh:42-139) and Restriction<Tag, methods::NONE>
 * (honei/math/restriction.hh:41-170), each followed by ApplyDirichletBoundaries
 * (honei/math/apply_dirichlet_boundaries.hh) with the 8-entry mask (2 = Dirichlet: zero the
 * corner / edge).  n_fine = fine nodes; the coarse grid has (sqrt(n_fine) - 1) / 2 + 1 nodes per
 * side.  Arithmetic in double, stored as DT (the reference's 0.5 / 0.25 literals are double). */
void   ora_prolongate_f64(uint64_t n_fine, double *fine, const double *coarse, const uint64_t *mask);
void   ora_prolongate_f32(uint64_t n_fine, float *fine, const float *coarse, const uint64_t *mask);
void   ora_restrict_f64(uint64_t n_fine, double *coarse, const double *fine, const uint64_t *mask);
void   ora_restrict_f32(uint64_t n_fine, float *coarse, const float *fine, const uint64_t *mask);
/* FillMatrix<POISSON, DIRICHLET_0> on the banded form (honei/math/fill_matrix.hh:41-77). */
void   ora_q1band_poisson_f64(uint64_t n, double *const *band);
double ora_dot_f64(uint64_t n, const double *x, const double *y);
float  ora_dot_f32(uint64_t n, const float *x, const float *y);
void   ora_scaled_sum_f64(uint64_t n, double *x, const double *y, double b);
void   ora_scaled_sum_f32(uint64_t n, float *x, const float *y, float b);
void   ora_scaled_sum3_f64(uint64_t n, double *r, const double *x, const double *y, double b);
void   ora_scale_f64(uint64_t n, double *x, double a);
void   ora_sum_f64(uint64_t n, double *x, const double *y);
void   ora_difference_f64(uint64_t n, double *r, const double *x, const double *y);
void   ora_element_product_f64(uint64_t n, double *r, const double *x, const double *y);

/* ---- Preconditioner construction ----
 * SPAI2<tags::CPU::SSE>::value(M, A, col_start, col_end) (honei/math/spai2.hh:129-260) on the
 * SparseMatrix made of A (honei/la/sparse_matrix.hh:157-185).  Mx is in A's ELL layout and must
 * hold A's values on entry (M = A.copy()); the entries of columns [col_start, col_end) are
 * overwritten (col_end == 0: every column).  Returns 0, or 1 when A is not square or memory runs
 * out.  The algorithm is restated in ora_spai2.inc. */
int    ora_spai2_f64(const ora_ell *A, double *Mx, uint64_t col_start, uint64_t col_end);
int    ora_spai2_f32(const ora_ell *A, float *Mx, uint64_t col_start, uint64_t col_end);

/* ---- Solvers ----
 * CG returns the number of iterations in *used; hist (optional, max_iters+1 entries) gets
 * sqrt(alpha) after every iteration, hist[0] = initial defect. */
int ora_cg_f64(const ora_ell *A, const double *b, double *x, uint64_t max_iters, double eps,
               uint64_t *used, double *hist);
int ora_cg_f32(const ora_ell *A, const float *b, float *x, uint64_t max_iters, float eps,
               uint64_t *used, float *hist);

/* CGSolver<Tag, methods::VAR> (honei/math/cg.hh:140-219): CG with preconditioner P, either a
 * vector (Pd, the element product z = P r; Pm == NULL) or an ELL matrix (Pm, z = P r). */
int ora_cg_var_f64(const ora_ell *A, const double *Pd, const ora_ell *Pm, const double *b, double *x,
                   uint64_t max_iters, double eps, uint64_t *used);
int ora_cg_var_f32(const ora_ell *A, const float *Pd, const ora_ell *Pm, const float *b, float *x,
                   uint64_t max_iters, float eps, uint64_t *used);

/* MG hierarchy, coarsest level first (level index 0 == HONEI level 1).  prol[l] maps level l
 * to level l+1 (rows = n_{l+1}); res[l] = prol[l]^T.  P[l] = damping / diag(A[l]). */
typedef struct {
    int nlevels;
    const ora_ell *A;
    const ora_ell *prol;
    const ora_ell *res;
    uint64_t max_iters, max_iters_coarse, n_pre, n_post;
} ora_mg;

int ora_mg_f64(const ora_mg *mg, double damping, const double *b, double *x, double eps,
               uint64_t *used, double *rnorm_hist);
int ora_mg_f32(const ora_mg *mg, float damping, const float *b, float *x, float eps,
               uint64_t *used, float *rnorm_hist);

/* IR (honei/math/ir.hh:30-78): FP64 outer defect + update around the FP32 MG above.
 * A64 is the finest FP64 matrix; mg32 the FP32 hierarchy. warm_start != 0 keeps the inner
 * x between outer steps (the reference behaviour); 0 = scaled mode (normalised defect, inner
 * x from zero, correction scaled back by |r|). */
int ora_ir_mg(const ora_ell *A64, const ora_mg *mg32, float damping, const double *b, double *x,
              double eps, float inner_eps, uint64_t max_iters, int warm_start, uint64_t *used,
              double *rnorm_hist);

/* IR with an FP32 CG inner solver in the scaled mode (normalised defect, inner CG from 0). */
int ora_ir_cg(const ora_ell *A64, const ora_ell *A32, const double *b, double *x, double eps,
              float inner_eps, uint64_t inner_max_iters, uint64_t max_iters, uint64_t *used,
              uint64_t *inner_total, double *rnorm_hist);

/* IR (scaled mode) around FP32 CG preconditioned by one V-cycle of mg32 from zero (coarse CG
 * eps 1e-6): the served mixed-precision solve.  *outer_out = outer steps, *inner_total = summed
 * PCG iterations, rnorm_hist[k] = FP64 defect norm before outer step k. */
int ora_ir_pcg(const ora_ell *A64, const ora_mg *mg32, float damping, const double *b, double *x, double eps,
               float inner_eps, uint64_t max_outer, uint64_t max_inner, uint64_t *outer_out, uint64_t *inner_total,
               double *rnorm_hist);

#ifdef __cplusplus
}
#endif
#endif
