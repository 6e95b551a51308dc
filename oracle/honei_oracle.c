/* honei_oracle.c -- plain-C restatement of the HONEI sparse-solver path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker, never the thing measured or shipped.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Pinned against the reference itself: tests/test_oracle_pin.py compares every routine
 * bit-for-bit with oracle/_ref/libhonei_ref.so (the unmodified HONEI CPU path) and with the
 * committed fixtures under tests/golden/.
 *
 * Each routine cites the reference source it restates (paths within the HONEI tree).
 * Build with -ffp-contract=off: the reference rounds once per multiply and once per add.
 */
#include "honei_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------------------
 * ELL SpMV -- honei/la/product.hh:148-204 (Product<tags::CPU>, SparseMatrixELL x DenseVector)
 *   for row: sum = 0; for col < Arl[row]: for thread < T: sum += Ax[j+thread] * x[Aj[j+thread]]
 *   with j = row*T + col*stride.
 * Defect -- honei/math/defect.hh:357-383: temp = A x, then r[i] = b[i] - temp[i].
 * ------------------------------------------------------------------------------------- */
#define ORA_SPMV(SUF, DT)                                                                   \
void ora_spmv_##SUF(const ora_ell *A, const DT *x, DT *y)                                   \
{                                                                                           \
    const DT *ax = (const DT *)A->Ax;                                                       \
    for (uint64_t row = 0; row < A->rows; ++row) {                                          \
        DT sum = 0;                                                                         \
        uint64_t j = row * A->threads;                                                      \
        for (uint64_t col = 0; col < A->Arl[row]; ++col, j += A->stride)                    \
            for (uint64_t t = 0; t < A->threads; ++t)                                       \
                sum += ax[j + t] * x[A->Aj[j + t]];                                         \
        y[row] = sum;                                                                       \
    }                                                                                       \
}                                                                                           \
void ora_defect_##SUF(const ora_ell *A, const DT *b, const DT *x, DT *r)                    \
{                                                                                           \
    DT *temp = (DT *)malloc(sizeof(DT) * (A->rows ? A->rows : 1));                          \
    ora_spmv_##SUF(A, x, temp);                                                             \
    for (uint64_t i = 0; i < A->rows; ++i) r[i] = b[i] - temp[i];                           \
    free(temp);                                                                             \
}
ORA_SPMV(f64, double)
ORA_SPMV(f32, float)

/* Product<tags::CPU>::value(DV, SparseMatrixCSR, DV) -- honei/la/product.hh:209-242, and the
 * CSR Defect -- honei/math/defect.hh:386-419 (the same sum, then rhs - sum in one step). */
#define ORA_CSR(SUF, DT)                                                                    \
static DT ora_csr_row_##SUF(const ora_csr *A, const DT *x, uint64_t row)                    \
{                                                                                           \
    const DT *Ax = (const DT *)A->Ax;                                                       \
    const uint64_t bs = A->blocksize;                                                       \
    DT sum = 0;                                                                             \
    for (uint64_t i = A->Ar[row]; i < A->Ar[row + 1]; ++i)                                  \
        for (uint64_t k = 0; k < bs; ++k)                                                   \
            if (A->Aj[i] + k < A->cols) sum += Ax[i * bs + k] * x[A->Aj[i] + k];            \
    return sum;                                                                             \
}                                                                                           \
void ora_csr_spmv_##SUF(const ora_csr *A, const DT *x, DT *y)                               \
{                                                                                           \
    for (uint64_t row = 0; row < A->rows; ++row) y[row] = ora_csr_row_##SUF(A, x, row);     \
}                                                                                           \
void ora_csr_defect_##SUF(const ora_csr *A, const DT *rhs, const DT *x, DT *r)              \
{                                                                                           \
    for (uint64_t row = 0; row < A->rows; ++row) r[row] = rhs[row] - ora_csr_row_##SUF(A, x, row); \
}
ORA_CSR(f64, double)
ORA_CSR(f32, float)

/* DotProduct<tags::CPU> -- honei/la/dot_product.hh:72-88: sequential, left to right.
 * Norm<vnt_l_two, false> == DotProduct(x, x) (honei/la/norm.hh:290-306). */
#define ORA_DOT(SUF, DT)                                                                    \
DT ora_dot_##SUF(uint64_t n, const DT *x, const DT *y)                                      \
{                                                                                           \
    DT result = 0;                                                                          \
    for (uint64_t i = 0; i < n; ++i) result += x[i] * y[i];                                 \
    return result;                                                                          \
}
ORA_DOT(f64, double)
ORA_DOT(f32, float)

/* ScaledSum -- honei/la/scaled_sum.hh:73-110: x[i] += b * y[i];  r[i] = b * y[i] + x[i]. */
void ora_scaled_sum_f64(uint64_t n, double *x, const double *y, double b)
{ for (uint64_t i = 0; i < n; ++i) x[i] += b * y[i]; }
void ora_scaled_sum_f32(uint64_t n, float *x, const float *y, float b)
{ for (uint64_t i = 0; i < n; ++i) x[i] += b * y[i]; }
void ora_scaled_sum3_f64(uint64_t n, double *r, const double *x, const double *y, double b)
{ for (uint64_t i = 0; i < n; ++i) r[i] = b * y[i] + x[i]; }
/* Scale -- honei/la/scale.hh:77 (x *= a); Sum -- honei/la/sum.hh:98 (x += y);
 * Difference (r = x - y); ElementProduct -- honei/la/element_product.hh:76-140 (r = x * y). */
void ora_scale_f64(uint64_t n, double *x, double a)
{ for (uint64_t i = 0; i < n; ++i) x[i] *= a; }
void ora_sum_f64(uint64_t n, double *x, const double *y)
{ for (uint64_t i = 0; i < n; ++i) x[i] += y[i]; }
void ora_difference_f64(uint64_t n, double *r, const double *x, const double *y)
{ for (uint64_t i = 0; i < n; ++i) r[i] = x[i] - y[i]; }
void ora_element_product_f64(uint64_t n, double *r, const double *x, const double *y)
{ for (uint64_t i = 0; i < n; ++i) r[i] = x[i] * y[i]; }

/* ---------------------------------------------------------------------------------------
 * CGSolver<Tag, methods::NONE> -- honei/math/cg.hh:63-133.
 *   r = b - A x; p = r; alpha = r.r; d0 = sqrt(alpha)
 *   loop: v = A p; temp = v.p; lambda = alpha / (|temp| > eps_mach ? temp : eps_mach)
 *         x += lambda p; r += (-lambda) v; alpha_old = alpha; alpha = r.r
 *         beta = alpha / (|alpha_old| > eps_mach ? alpha_old : eps_mach); p *= beta; p += r
 *         stop if sqrt(alpha) < eps * d0 or sqrt(alpha) < eps (used_iters set only on stop
 *         or when max_iters is reached).
 * ------------------------------------------------------------------------------------- */
#define ORA_CG(SUF, DT, EPSM, SQRT, FABS)                                                   \
int ora_cg_##SUF(const ora_ell *A, const DT *b, DT *x, uint64_t max_iters, DT eps,          \
                 uint64_t *used, DT *hist)                                                  \
{                                                                                           \
    const uint64_t n = A->rows;                                                             \
    DT *p = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    DT *r = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    DT *v = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    if (!p || !r || !v) { free(p); free(r); free(v); return 1; }                            \
    ora_defect_##SUF(A, b, x, r);                                                           \
    memcpy(p, r, sizeof(DT) * n);                                                           \
    DT alpha = ora_dot_##SUF(n, r, r), alpha_old, lambda, temp;                             \
    DT initial_defect = SQRT(alpha), current_defect = 0;                                    \
    if (hist) hist[0] = initial_defect;                                                     \
    uint64_t it = 0;                                                                        \
    while (it < max_iters) {                                                                \
        ora_spmv_##SUF(A, p, v);                                                            \
        temp = ora_dot_##SUF(n, v, p);                                                      \
        lambda = alpha / (FABS(temp) > EPSM ? temp : EPSM);                                 \
        for (uint64_t i = 0; i < n; ++i) x[i] += lambda * p[i];                             \
        DT mlambda = -lambda;                                                               \
        for (uint64_t i = 0; i < n; ++i) r[i] += mlambda * v[i];                            \
        alpha_old = alpha;                                                                  \
        alpha = ora_dot_##SUF(n, r, r);                                                     \
        DT talpha = alpha / (FABS(alpha_old) > EPSM ? alpha_old : EPSM);                    \
        for (uint64_t i = 0; i < n; ++i) p[i] *= talpha;                                    \
        for (uint64_t i = 0; i < n; ++i) p[i] += r[i];                                      \
        ++it;                                                                               \
        current_defect = SQRT(alpha);                                                       \
        if (hist) hist[it] = current_defect;                                                \
        if (current_defect < eps * initial_defect) { *used = it; break; }                   \
        if (current_defect < eps) { *used = it; break; }                                    \
        if (it == max_iters) *used = it;                                                    \
    }                                                                                       \
    free(p); free(r); free(v);                                                              \
    return 0;                                                                               \
}
ORA_CG(f64, double, DBL_EPSILON, sqrt, fabs)
ORA_CG(f32, float, FLT_EPSILON, sqrtf, fabsf)

/* ---------------------------------------------------------------------------------------
 * CGSolver<Tag, methods::VAR> -- honei/math/cg.hh:140-219.  Product(z, P, r) is the element
 * product for a vector P (Product(DV, DV, DV), honei/la/product.hh:1198-1204) and the ELL
 * product for a matrix P.  Norm<l2, true> = sqrt(r.r); divisions guarded by
 * |t| > eps_mach ? t : eps_mach * (t / |t|) (cg.hh:172, 206).
 * ------------------------------------------------------------------------------------- */
#define ORA_CG_VAR(SUF, DT, EPSM, SQRT, FABS)                                               \
static void precon_##SUF(const DT *Pd, const ora_ell *Pm, uint64_t n, const DT *r, DT *z)    \
{                                                                                           \
    if (Pm) ora_spmv_##SUF(Pm, r, z);                                                       \
    else for (uint64_t i = 0; i < n; ++i) z[i] = Pd[i] * r[i];                              \
}                                                                                           \
int ora_cg_var_##SUF(const ora_ell *A, const DT *Pd, const ora_ell *Pm, const DT *b, DT *x,  \
                     uint64_t max_iters, DT eps, uint64_t *used)                            \
{                                                                                           \
    const uint64_t n = A->rows;                                                             \
    DT *p = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    DT *r = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    DT *v = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    DT *z = (DT *)malloc(sizeof(DT) * (n ? n : 1));                                         \
    if (!p || !r || !v || !z) { free(p); free(r); free(v); free(z); return 1; }             \
    ora_defect_##SUF(A, b, x, r);                                                           \
    precon_##SUF(Pd, Pm, n, r, p);                                                          \
    const DT initial_defect = SQRT(ora_dot_##SUF(n, r, r));                                 \
    DT alpha_new = ora_dot_##SUF(n, r, p), alpha, temp, lambda;                             \
    uint64_t it = 0;                                                                        \
    while (it < max_iters) {                                                                \
        ora_spmv_##SUF(A, p, v);                                                            \
        temp = ora_dot_##SUF(n, v, p);                                                      \
        lambda = alpha_new / (FABS(temp) > EPSM ? temp : EPSM * (temp / FABS(temp)));       \
        ++it;                                                                               \
        for (uint64_t i = 0; i < n; ++i) x[i] += p[i] * lambda;                             \
        DT mlambda = -lambda;                                                               \
        for (uint64_t i = 0; i < n; ++i) r[i] += v[i] * mlambda;                            \
        DT current_defect = SQRT(ora_dot_##SUF(n, r, r));                                   \
        if (current_defect < eps * initial_defect) { *used = it; break; }                   \
        if (current_defect < eps) { *used = it; break; }                                    \
        if (it == max_iters) { *used = it; break; }                                         \
        precon_##SUF(Pd, Pm, n, r, z);                                                      \
        alpha = alpha_new;                                                                  \
        alpha_new = ora_dot_##SUF(n, r, z);                                                 \
        DT talpha = alpha_new / (FABS(alpha) > EPSM ? alpha : EPSM * (alpha / FABS(alpha))); \
        for (uint64_t i = 0; i < n; ++i) p[i] *= talpha;                                    \
        for (uint64_t i = 0; i < n; ++i) p[i] += z[i];                                      \
    }                                                                                       \
    free(p); free(r); free(v); free(z);                                                     \
    return 0;                                                                               \
}
ORA_CG_VAR(f64, double, DBL_EPSILON, sqrt, fabs)
ORA_CG_VAR(f32, float, FLT_EPSILON, sqrtf, fabsf)

/* ---------------------------------------------------------------------------------------
 * Multigrid V-cycle -- honei/math/mg.hh:567-662 (MGCycleCreation<V::STATIC>) and
 * honei/math/mg.hh:1093-1127 (MGSolver), with
 *   smoother RISmoother -- honei/math/ri.hh:97-133: n x { t0 = b - A x; t1 = P * t0; x += t1 }
 *   P = damping / diag(A)  -- PreconFill "jac", honei/math/mg.hh:255-286
 *   restriction  d_{l-1} = Res_l store_l  -- honei/math/restriction.hh:175-185
 *   prolongation store_l = Prol_l c_{l-1}; x_l += store_l -- honei/math/prolongation.hh:142-155
 *   coarse solve CGSolver<NONE>(A_1, b_1, x_1, max_iters_coarse, eps) at min_level = 1.
 * Top level works on (x, b); every lower level on (c, d), c zero-filled before recursion.
 * ------------------------------------------------------------------------------------- */
#define ORA_MG(SUF, DT, SQRT)                                                               \
typedef struct {                                                                            \
    const ora_mg *mg;                                                                       \
    DT **P, **d, **c, **store, **t0, **t1;                                                  \
    DT eps;                                                                                 \
    uint64_t used_coarse;                                                                   \
} mgws_##SUF;                                                                               \
/* A(row, row) as SparseMatrixELL::operator() finds it (sparse_matrix_ell-impl.hh:326-338) */ \
static DT ora_diag_##SUF(const ora_ell *A, uint64_t row)                                    \
{                                                                                           \
    const DT *ax = (const DT *)A->Ax;                                                       \
    uint64_t j = row * A->threads;                                                          \
    for (uint64_t col = 0; col < A->Arl[row] && A->Aj[j] <= row; ++col, j += A->stride)     \
        for (uint64_t t = 0; t < A->threads; ++t)                                           \
            if (A->Aj[j + t] == row) return ax[j + t];                                      \
    return 0;                                                                               \
}                                                                                           \
static void ora_smooth_##SUF(mgws_##SUF *w, int l, const DT *b, DT *x, uint64_t n_sweeps)   \
{                                                                                           \
    const ora_ell *A = &w->mg->A[l];                                                        \
    for (uint64_t s = 0; s < n_sweeps; ++s) {                                               \
        ora_defect_##SUF(A, b, x, w->t0[l]);                                                \
        for (uint64_t i = 0; i < A->rows; ++i) w->t1[l][i] = w->P[l][i] * w->t0[l][i];      \
        for (uint64_t i = 0; i < A->rows; ++i) x[i] += w->t1[l][i];                         \
    }                                                                                       \
}                                                                                           \
static void ora_vcycle_##SUF(mgws_##SUF *w, int l, DT *x, const DT *b)                      \
{                                                                                           \
    const ora_mg *mg = w->mg;                                                               \
    if (l == 0) {                                                                           \
        uint64_t u = w->used_coarse;                                                        \
        ora_cg_##SUF(&mg->A[0], b, x, mg->max_iters_coarse, w->eps, &u, NULL);              \
        w->used_coarse = u;                                                                 \
        return;                                                                             \
    }                                                                                       \
    ora_smooth_##SUF(w, l, b, x, mg->n_pre);                                                \
    ora_defect_##SUF(&mg->A[l], b, x, w->store[l]);                                         \
    ora_spmv_##SUF(&mg->res[l - 1], w->store[l], w->d[l - 1]);                              \
    memset(w->c[l - 1], 0, sizeof(DT) * mg->A[l - 1].rows);                                 \
    ora_vcycle_##SUF(w, l - 1, w->c[l - 1], w->d[l - 1]);                                   \
    ora_spmv_##SUF(&mg->prol[l - 1], w->c[l - 1], w->store[l]);                             \
    for (uint64_t i = 0; i < mg->A[l].rows; ++i) x[i] += w->store[l][i];                    \
    ora_smooth_##SUF(w, l, b, x, mg->n_post);                                               \
}                                                                                           \
int ora_mg_##SUF(const ora_mg *mg, DT damping, const DT *b, DT *x, DT eps, uint64_t *used,  \
                 DT *rnorm_hist)                                                            \
{                                                                                           \
    const int L = mg->nlevels;                                                              \
    mgws_##SUF w;                                                                           \
    w.mg = mg; w.eps = eps; w.used_coarse = 0;                                              \
    DT ***arrs[] = { &w.P, &w.d, &w.c, &w.store, &w.t0, &w.t1 };                            \
    for (int a = 0; a < 6; ++a) {                                                           \
        *arrs[a] = (DT **)calloc(L, sizeof(DT *));                                          \
        for (int l = 0; l < L; ++l)                                                         \
            (*arrs[a])[l] = (DT *)calloc(mg->A[l].rows ? mg->A[l].rows : 1, sizeof(DT));    \
    }                                                                                       \
    for (int l = 0; l < L; ++l)                                                             \
        for (uint64_t i = 0; i < mg->A[l].rows; ++i) {                                      \
            DT p = damping;                                                                 \
            p /= ora_diag_##SUF(&mg->A[l], i);                                              \
            w.P[l][i] = p;                                                                  \
        }                                                                                   \
    const uint64_t n = mg->A[L - 1].rows;                                                   \
    DT *r = (DT *)calloc(n ? n : 1, sizeof(DT));                                            \
    ora_defect_##SUF(&mg->A[L - 1], b, x, r);                                               \
    DT rnorm_initial = SQRT(ora_dot_##SUF(n, r, r));                                        \
    DT rnorm_current = (DT)1e16;                                                            \
    if (rnorm_hist) rnorm_hist[0] = rnorm_initial;                                          \
    for (uint64_t i = 0; i < mg->max_iters; ++i) {                                          \
        ora_vcycle_##SUF(&w, L - 1, x, b);                                                  \
        ora_defect_##SUF(&mg->A[L - 1], b, x, r);                                           \
        rnorm_current = SQRT(ora_dot_##SUF(n, r, r));                                       \
        if (rnorm_hist) rnorm_hist[i + 1] = rnorm_current;                                  \
        *used = i + 1;                                                                      \
        if (rnorm_current < eps * rnorm_initial) break;                                     \
    }                                                                                       \
    free(r);                                                                                \
    for (int a = 0; a < 6; ++a) {                                                           \
        for (int l = 0; l < L; ++l) free((*arrs[a])[l]);                                    \
        free(*arrs[a]);                                                                     \
    }                                                                                       \
    return 0;                                                                               \
}
ORA_MG(f64, double, sqrt)
ORA_MG(f32, float, sqrtf)

/* ---------------------------------------------------------------------------------------
 * IRSolver<Outer=double, Inner=float> -- honei/math/ir.hh:30-78.
 *   for i < max_iters: r = b - A x (FP64); i == 0 ? rnorm0 = |r| : (used = i; stop if
 *   |r| < eps * rnorm0); b_inner = (float) r; inner MG; c = (double) x_inner; x += c.
 * The reference leaves x_inner as it was (warm start, warm_start != 0).  warm_start == 0 is
 * the scaled mode: the defect is normalised to unit norm before the cast, the inner solve starts
 * from zero and the correction is scaled back (x += |r| * c), so the inner eps is relative.
 * ------------------------------------------------------------------------------------- */
int ora_ir_mg(const ora_ell *A64, const ora_mg *mg32, float damping, const double *b, double *x,
              double eps, float inner_eps, uint64_t max_iters, int warm_start, uint64_t *used,
              double *rnorm_hist)
{
    const uint64_t n = A64->rows;
    double *r = (double *)calloc(n ? n : 1, sizeof(double));
    float *bi = (float *)calloc(n ? n : 1, sizeof(float));
    float *xi = (float *)calloc(n ? n : 1, sizeof(float));
    double rnorm_initial = 1e16, rnorm_current = 1e16;
    for (uint64_t i = 0; i < max_iters; ++i) {
        ora_defect_f64(A64, b, x, r);
        if (i == 0) {
            rnorm_initial = sqrt(ora_dot_f64(n, r, r));
            if (rnorm_hist) rnorm_hist[0] = rnorm_initial;
        } else {
            rnorm_current = sqrt(ora_dot_f64(n, r, r));
            if (rnorm_hist) rnorm_hist[i] = rnorm_current;
            *used = i;
            if (rnorm_current < eps * rnorm_initial) break;
        }
        if (warm_start) {
            for (uint64_t k = 0; k < n; ++k) bi[k] = (float)r[k];
        } else {
            /* scaled mode: normalised defect, inner solve from zero, correction scaled back */
            const double s = 1.0 / (i == 0 ? rnorm_initial : rnorm_current);
            for (uint64_t k = 0; k < n; ++k) bi[k] = (float)(r[k] * s);
            memset(xi, 0, sizeof(float) * n);
        }
        uint64_t inner_used = 0;
        ora_mg_f32(mg32, damping, bi, xi, inner_eps, &inner_used, NULL);
        if (warm_start) {
            for (uint64_t k = 0; k < n; ++k) x[k] += (double)xi[k];
        } else {
            const double nr = (i == 0 ? rnorm_initial : rnorm_current);
            for (uint64_t k = 0; k < n; ++k) x[k] += nr * (double)xi[k];
        }
    }
    free(r); free(bi); free(xi);
    return 0;
}

int ora_ir_cg(const ora_ell *A64, const ora_ell *A32, const double *b, double *x, double eps,
              float inner_eps, uint64_t inner_max_iters, uint64_t max_iters, uint64_t *used,
              uint64_t *inner_total, double *rnorm_hist)
{
    const uint64_t n = A64->rows;
    double *r = (double *)calloc(n ? n : 1, sizeof(double));
    float *bi = (float *)calloc(n ? n : 1, sizeof(float));
    float *xi = (float *)calloc(n ? n : 1, sizeof(float));
    double rnorm_initial = 1e16, rnorm_current = 1e16;
    uint64_t total = 0;
    for (uint64_t i = 0; i < max_iters; ++i) {
        ora_defect_f64(A64, b, x, r);
        if (i == 0) {
            rnorm_initial = sqrt(ora_dot_f64(n, r, r));
            if (rnorm_hist) rnorm_hist[0] = rnorm_initial;
        } else {
            rnorm_current = sqrt(ora_dot_f64(n, r, r));
            if (rnorm_hist) rnorm_hist[i] = rnorm_current;
            *used = i;
            if (rnorm_current < eps * rnorm_initial) break;
        }
        /* normalised defect, so the inner CG's absolute test (cg.hh:118) cannot stop it early */
        const double nr = (i == 0 ? rnorm_initial : rnorm_current), s = 1.0 / nr;
        for (uint64_t k = 0; k < n; ++k) bi[k] = (float)(r[k] * s);
        memset(xi, 0, sizeof(float) * n);
        uint64_t inner_used = 0;
        ora_cg_f32(A32, bi, xi, inner_max_iters, inner_eps, &inner_used, NULL);
        total += inner_used;
        for (uint64_t k = 0; k < n; ++k) x[k] += nr * (double)xi[k];
    }
    if (inner_total) *inner_total = total;
    free(r); free(bi); free(xi);
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * IR around an FP32 CG preconditioned by one V-cycle (the served mixed-precision solve of
 * hb_q1_solve; no reference counterpart).  Outer loop as ora_ir_mg's scaled mode; inner PCG
 * from x = 0 on the normalised defect until |r| < inner_eps |r0|:
 *   z = M(r); p = z; rz = r.z; loop { v = A p; a = rz / p.v; x += a p; r -= a v;
 *   stop if |r| < eps |r0|; z = M(r); beta = r.z_new / rz; p = beta p + z }
 * M = one V-cycle of ora_vcycle_f32 from z = 0.
 * ------------------------------------------------------------------------------------- */
static int ora_pcg_f32(mgws_f32 *w, const float *b, float *x, float eps, uint64_t max_iters, uint64_t *used)
{
    const ora_mg *mg = w->mg;
    const int top = mg->nlevels - 1;
    const ora_ell *A = &mg->A[top];
    const uint64_t n = A->rows;
    float *r = (float *)calloc(n ? n : 1, 4), *z = (float *)calloc(n ? n : 1, 4);
    float *p = (float *)calloc(n ? n : 1, 4), *v = (float *)calloc(n ? n : 1, 4);
    memset(x, 0, sizeof(float) * n);
    memcpy(r, b, sizeof(float) * n);
    const float r0 = sqrtf(ora_dot_f32(n, r, r));
    uint64_t it = 0;
    if (r0 > 0.f && max_iters > 0) {
        memset(z, 0, sizeof(float) * n);
        ora_vcycle_f32(w, top, z, r);
        memcpy(p, z, sizeof(float) * n);
        float rz = ora_dot_f32(n, r, z);
        while (it < max_iters) {
            ora_spmv_f32(A, p, v);
            const float pv = ora_dot_f32(n, p, v);
            if (!(pv > 0.f)) break;
            const float a = rz / pv;
            for (uint64_t i = 0; i < n; ++i) x[i] += a * p[i];
            const float ma = -a;
            for (uint64_t i = 0; i < n; ++i) r[i] += ma * v[i];
            ++it;
            if (sqrtf(ora_dot_f32(n, r, r)) < eps * r0) break;
            memset(z, 0, sizeof(float) * n);
            ora_vcycle_f32(w, top, z, r);
            const float rz_new = ora_dot_f32(n, r, z);
            const float beta = rz_new / rz;
            rz = rz_new;
            for (uint64_t i = 0; i < n; ++i) p[i] = beta * p[i] + z[i];
        }
    }
    *used = it;
    free(r); free(z); free(p); free(v);
    return 0;
}

int ora_ir_pcg(const ora_ell *A64, const ora_mg *mg32, float damping, const double *b, double *x, double eps,
               float inner_eps, uint64_t max_outer, uint64_t max_inner, uint64_t *outer_out, uint64_t *inner_total,
               double *rnorm_hist)
{
    const int L = mg32->nlevels;
    mgws_f32 w;
    w.mg = mg32; w.eps = (float)1e-6; w.used_coarse = 0;
    float ***arrs[] = { &w.P, &w.d, &w.c, &w.store, &w.t0, &w.t1 };
    for (int a = 0; a < 6; ++a) {
        *arrs[a] = (float **)calloc(L, sizeof(float *));
        for (int l = 0; l < L; ++l)
            (*arrs[a])[l] = (float *)calloc(mg32->A[l].rows ? mg32->A[l].rows : 1, sizeof(float));
    }
    for (int l = 0; l < L; ++l)
        for (uint64_t i = 0; i < mg32->A[l].rows; ++i) {
            float pv = damping;
            pv /= ora_diag_f32(&mg32->A[l], i);
            w.P[l][i] = pv;
        }
    const uint64_t n = A64->rows;
    double *r = (double *)calloc(n ? n : 1, 8);
    float *bi = (float *)calloc(n ? n : 1, 4), *xi = (float *)calloc(n ? n : 1, 4);
    double nrm0 = 0.0, nrm = 0.0;
    uint64_t outer = 0, total = 0;
    for (;;) {
        ora_defect_f64(A64, b, x, r);
        nrm = sqrt(ora_dot_f64(n, r, r));
        if (rnorm_hist) rnorm_hist[outer] = nrm;
        if (outer == 0) nrm0 = nrm;
        else if (nrm < eps * nrm0) break;
        if (nrm == 0.0 || outer >= max_outer) break;
        const double s = 1.0 / nrm;
        for (uint64_t k = 0; k < n; ++k) bi[k] = (float)(r[k] * s);
        uint64_t used = 0;
        ora_pcg_f32(&w, bi, xi, inner_eps, max_inner, &used);
        total += used;
        for (uint64_t k = 0; k < n; ++k) x[k] += nrm * (double)xi[k];
        ++outer;
    }
    *outer_out = outer;
    if (inner_total) *inner_total = total;
    free(r); free(bi); free(xi);
    for (int a = 0; a < 6; ++a) {
        for (int l = 0; l < L; ++l) free((*arrs[a])[l]);
        free(*arrs[a]);
    }
    return 0;
}

/* ---- BandedMatrixQx<Q1Type> ------------------------------------------------------------
 * Product<tags::CPU>::value(result, BandedMatrixQx, x) (honei/la/product.hh:371-404): the
 * diagonal product first, then the eight off-diagonal bands in the order LL, LD, LU, DL, DU,
 * UL, UD, UU, each only where its column index lies in [0, n) (a bound on the linear index,
 * not on the grid line). */
#define ORA_Q1BAND_ROW(T, i)                                                                  \
    do {                                                                                      \
        const long r_ = (long)root, n_ = (long)n, k_ = (long)(i);                             \
        T s_ = band[4][k_] * x[k_];                                                           \
        if (k_ - r_ - 1 >= 0) s_ += band[0][k_] * x[k_ - r_ - 1];                             \
        if (k_ - r_ >= 0)     s_ += band[1][k_] * x[k_ - r_];                                 \
        if (k_ - r_ + 1 >= 0) s_ += band[2][k_] * x[k_ - r_ + 1];                             \
        if (k_ - 1 >= 0)      s_ += band[3][k_] * x[k_ - 1];                                  \
        if (k_ + 1 < n_)      s_ += band[5][k_] * x[k_ + 1];                                  \
        if (k_ + r_ - 1 < n_) s_ += band[6][k_] * x[k_ + r_ - 1];                             \
        if (k_ + r_ < n_)     s_ += band[7][k_] * x[k_ + r_];                                 \
        if (k_ + r_ + 1 < n_) s_ += band[8][k_] * x[k_ + r_ + 1];                             \
        out_ = s_;                                                                            \
    } while (0)

static uint64_t q1band_root(uint64_t n) { return (uint64_t)sqrt((double)n); }

void ora_q1band_spmv_f64(uint64_t n, const double *const *band, const double *x, double *y)
{
    const uint64_t root = q1band_root(n);
    for (uint64_t i = 0; i < n; ++i) { double out_; ORA_Q1BAND_ROW(double, i); y[i] = out_; }
}

void ora_q1band_spmv_f32(uint64_t n, const float *const *band, const float *x, float *y)
{
    const uint64_t root = q1band_root(n);
    for (uint64_t i = 0; i < n; ++i) { float out_; ORA_Q1BAND_ROW(float, i); y[i] = out_; }
}

void ora_q1band_defect_f64(uint64_t n, const double *const *band, const double *b, const double *x, double *r)
{
    const uint64_t root = q1band_root(n);
    for (uint64_t i = 0; i < n; ++i) { double out_; ORA_Q1BAND_ROW(double, i); r[i] = b[i] - out_; }
}

void ora_q1band_defect_f32(uint64_t n, const float *const *band, const float *b, const float *x, float *r)
{
    const uint64_t root = q1band_root(n);
    for (uint64_t i = 0; i < n; ++i) { float out_; ORA_Q1BAND_ROW(float, i); r[i] = b[i] - out_; }
}

/* FillMatrix<Tag, POISSON, DIRICHLET_0> on BandedMatrixQx (honei/math/fill_matrix.hh:41-77):
 * with 1-based i, rows i <= M, i > N - M, i % M == 1 or i % M == 0 are unit rows; the others
 * hold 8/3 on the diagonal and -1/3 on all eight off-diagonal bands. */
void ora_q1band_poisson_f64(uint64_t n, double *const *band)
{
    const uint64_t M = q1band_root(n);
    for (uint64_t i = 1; i <= n; ++i) {
        const int unit = i <= M || i > n - M || (i % M) == 1 || (i % M) == 0;
        for (int k = 0; k < 9; ++k) band[k][i - 1] = unit ? 0.0 : -1.0 / 3.0;
        band[4][i - 1] = unit ? 1.0 : 8.0 / 3.0;
    }
}

/* ---- Geometric transfers ------------------------------------------------------------------
 * A literal restatement of the reference loops (prolongation.hh:46-139, restriction.hh:45-170,
 * apply_dirichlet_boundaries.hh): same visiting order, every += evaluated in double (the
 * literals 0.5 / 0.25 are double) and stored back as DT. */
#define ORA_DIRICHLET(SUF, DT)                                                                  \
static void dirichlet_##SUF(uint64_t N, DT *g, const uint64_t *mask)                            \
{                                                                                               \
    const uint64_t M = (uint64_t)sqrt((double)N);                                               \
    if (mask[0] == 2) g[0] = 0;                                                                 \
    if (mask[1] == 2) g[M - 1] = 0;                                                             \
    if (mask[2] == 2) g[N - 1] = 0;                                                             \
    if (mask[3] == 2) g[N - M] = 0;                                                             \
    if (mask[4] == 2) for (uint64_t i = 1; i < M - 1; ++i) g[i] = 0;                            \
    if (mask[5] == 2) for (uint64_t i = 2 * M - 1; i < N - M; i += M) g[i] = 0;                 \
    if (mask[6] == 2) for (uint64_t i = N - M + 1; i < N - 1; ++i) g[i] = 0;                    \
    if (mask[7] == 2) for (uint64_t i = M; i < N - M; i += M) g[i] = 0;                         \
}
ORA_DIRICHLET(f64, double)
ORA_DIRICHLET(f32, float)

#define ORA_TRANSFER(SUF, DT)                                                                   \
void ora_prolongate_##SUF(uint64_t n_fine, DT *fine, const DT *coarse, const uint64_t *mask)   \
{                                                                                               \
    const uint64_t nxf = (uint64_t)sqrt((double)n_fine) - 1, nxc = nxf / 2, nyf = nxf + 1,     \
                   nyc = nxc + 1, istep = 2 * nyf;                                              \
    for (uint64_t i = 0; i < n_fine; ++i) fine[i] = 0;                                          \
    for (uint64_t i = 1; i <= nyc; ++i)                                                         \
        for (uint64_t j = 0, k = 0; j < nyc; ++j, k += 2)                                       \
            fine[istep * (i - 1) + k] = coarse[i + nxc * (i - 1) - 1 + j];                      \
    for (uint64_t i = 1; i <= nxc; ++i) {                                                       \
        uint64_t a = 2 * i;                                                                     \
        for (uint64_t j = 0; j < nyc; ++j) {                                                    \
            fine[a - 1 + j * istep] = (DT)((double)fine[a - 1 + j * istep] + (double)coarse[i - 1 + j * nyc] * 0.5); \
            fine[a - 1 + j * istep] = (DT)((double)fine[a - 1 + j * istep] + (double)coarse[i + j * nyc] * 0.5);     \
        }                                                                                       \
        a = nyf + 1 + (i - 1) * istep;                                                          \
        for (uint64_t j = 0; j < nyc; ++j) {                                                    \
            fine[a - 1 + j * 2] = (DT)((double)fine[a - 1 + j * 2] + (double)fine[a - nyf - 1 + j * 2] * 0.5);     \
            fine[a - 1 + j * 2] = (DT)((double)fine[a - 1 + j * 2] + (double)fine[a + nyf - 1 + j * 2] * 0.5);     \
        }                                                                                       \
    }                                                                                           \
    for (uint64_t i = 1; i <= nxc; ++i) {                                                       \
        const uint64_t a = nxf + 3 + (i - 1) * istep;                                           \
        for (uint64_t j = 0; j < nxc; ++j) {                                                    \
            DT *f = &fine[a - 1 + j * 2];                                                       \
            *f = (DT)((double)*f + (double)fine[a - nxf - 3 + j * 2] * 0.25);                   \
            *f = (DT)((double)*f + (double)fine[a - nxf - 1 + j * 2] * 0.25);                   \
            *f = (DT)((double)*f + (double)fine[a + nxf - 1 + j * 2] * 0.25);                   \
            *f = (DT)((double)*f + (double)fine[a + nxf + 1 + j * 2] * 0.25);                   \
        }                                                                                       \
    }                                                                                           \
    dirichlet_##SUF(n_fine, fine, mask);                                                        \
}                                                                                               \
void ora_restrict_##SUF(uint64_t n_fine, DT *coarse, const DT *fine, const uint64_t *mask)     \
{                                                                                               \
    const uint64_t nxf = (uint64_t)sqrt((double)n_fine) - 1, nxc = nxf / 2, nyf = nxf + 1,     \
                   nyc = nxc + 1, istep = 2 * nyf;                                              \
    for (uint64_t i = 1; i <= nyc; ++i)                                                         \
        for (uint64_t j = 0, k = 0; j < nyc; ++j, k += 2)                                       \
            coarse[1 + nyc * (i - 1) - 1 + j] = fine[2 * nyf * (i - 1) + k];                    \
    for (uint64_t i = 1; i <= nxc; ++i) {                                                       \
        uint64_t ia = 1 + nyf + 2 * nyf * (i - 1), ia1 = 1 + nyc * i;                           \
        for (uint64_t j = 0; j < nyc; ++j)                                                      \
            coarse[ia1 - 1 + j] = (DT)((double)coarse[ia1 - 1 + j] + 0.5 * (double)fine[ia - 1 + j * 2]);          \
        ia1 -= nyc;                                                                             \
        for (uint64_t j = 0; j < nyc; ++j)                                                      \
            coarse[ia1 - 1 + j] = (DT)((double)coarse[ia1 - 1 + j] + 0.5 * (double)fine[ia - 1 + j * 2]);          \
        for (uint64_t j = 0; j < nyc; ++j)                                                      \
            coarse[i - 1 + j * nyc] = (DT)((double)coarse[i - 1 + j * nyc] + 0.5 * (double)fine[2 * i - 1 + j * istep]); \
        for (uint64_t j = 0; j < nyc; ++j)                                                      \
            coarse[i + j * nyc] = (DT)((double)coarse[i + j * nyc] + 0.5 * (double)fine[2 * i - 1 + j * istep]);   \
        ++ia;                                                                                   \
        for (uint64_t j = 0; j < nxc; ++j)                                                      \
            coarse[ia1 - 1 + j] = (DT)((double)coarse[ia1 - 1 + j] + 0.25 * (double)fine[ia - 1 + j * 2]);         \
        for (uint64_t j = 0; j < nxc; ++j)                                                      \
            coarse[ia1 + j] = (DT)((double)coarse[ia1 + j] + 0.25 * (double)fine[ia - 1 + j * 2]);                 \
        for (uint64_t j = 0; j < nxc; ++j)                                                      \
            coarse[nyc * i + j] = (DT)((double)coarse[nyc * i + j] + 0.25 * (double)fine[ia - 1 + j * 2]);         \
        for (uint64_t j = 0; j < nxc; ++j)                                                      \
            coarse[1 + nyc * i + j] = (DT)((double)coarse[1 + nyc * i + j] + 0.25 * (double)fine[ia - 1 + j * 2]); \
    }                                                                                           \
    dirichlet_##SUF(nyc * nyc, coarse, mask);                                                   \
}
ORA_TRANSFER(f64, double)
ORA_TRANSFER(f32, float)

/* ---- SPAI2 (honei/math/spai2.hh:129-260) ---- */
#define ORA_CAT2(a, b) a##b
#define ORA_CAT(a, b) ORA_CAT2(a, b)
#define DT double
#define SUF f64
#include "ora_spai2.inc"
#undef DT
#undef SUF
#define DT float
#define SUF f32
#include "ora_spai2.inc"
#undef DT
#undef SUF
