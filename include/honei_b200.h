/* honei_b200.h -- C ABI of the B200 (sm_100a) backend for HONEI's sparse iterative-solver path.
 *
 * Everything here is plain C: opaque handles, plain pointers, sizes and an int status.  No
 * CUDA or torch types appear in the signatures (streams are passed as void* = cudaStream_t).
 * Vectors and matrix arrays are DEVICE pointers unless a parameter says "host".
 *
 * Each entry point names the reference interface it replaces (paths within the HONEI tree).
 * The reference's own GPU ABI is honei/backends/cuda/operations.hh:27-128 (e.g.
 * cuda_product_smell_dv_double) behind the tag-dispatched operators Product<tags::GPU::CUDA>,
 * Defect<...>, DotProduct<...>, Norm<...>, ScaledSum<...> and the solver templates CGSolver,
 * RISmoother, MGSolver and IRSolver.  Results are bit-compatible with tags::CPU wherever the
 * operation is elementwise or per-row (SpMV, defect, axpy family); reductions use a fixed
 * tree order (deterministic, run to run and alone vs. batched).
 *
 * Errors: every function returns HB_OK (0) or an hb_status code.  HB_ERR_SIZE corresponds to
 * the reference's VectorSizeDoesNotMatch / MatrixRowsDoNotMatch, raised before any launch.
 */
#ifndef HONEI_B200_H
#define HONEI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum {
    HB_OK = 0,
    HB_ERR_INVALID = 1,      /* null pointer, bad enum, misaligned device pointer         */
    HB_ERR_SIZE = 2,         /* vector / matrix sizes do not match (VectorSizeDoesNotMatch) */
    HB_ERR_CUDA = 3,         /* a CUDA runtime call failed                                  */
    HB_ERR_ALLOC = 4,        /* device or pinned allocation failed                          */
    HB_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up                          */
    HB_ERR_UNSUPPORTED = 6,  /* shape outside what the kernels support (e.g. > 2^31 rows)   */
    HB_ERR_CAPACITY = 7,     /* admission refused: over the HBM budget or slot count        */
    HB_ERR_NOT_FOUND = 8,    /* unknown request id                                          */
    HB_ERR_NONFINITE = 9     /* NaN or Inf found in an input that must be finite            */
} hb_status;

typedef enum { HB_F64 = 0, HB_F32 = 1 } hb_dtype;

/* ------------------------------------------------------------------------------------------
 * Context: device, stream, reduction scratch and pinned scalar slots (the role of the
 * reference's GPUPool + MemoryBackend<tags::GPU::CUDA>, honei/backends/cuda/gpu_pool.hh:53-88,
 * honei/util/memory_backend.hh:131-165).  One context per host thread / stream.
 * ---------------------------------------------------------------------------------------- */
typedef struct hb_context hb_context;

int  hb_create(hb_context **ctx, int device);
int  hb_destroy(hb_context *ctx);
int  hb_set_stream(hb_context *ctx, void *stream);      /* cudaStream_t; NULL = legacy stream */
int  hb_synchronize(hb_context *ctx);
const char *hb_status_string(int status);
/* Text of the last CUDA error seen by this context (empty if none). */
const char *hb_last_error(hb_context *ctx);
/* Number of kernels this library launched through ctx since creation (instrumentation). */
uint64_t hb_launch_count(hb_context *ctx);
/* Pre-size the context workspace for vectors of n entries, so later calls (and stream
 * captures) need no allocation. */
int  hb_reserve(hb_context *ctx, int64_t n);

/* ------------------------------------------------------------------------------------------
 * Device ELL matrix.  Replaces the device copies of SparseMatrixELL's Aj/Ax/Arl arrays
 * (honei/la/sparse_matrix_ell.hh:44-129) that the reference's MemoryBackend uploads.
 *
 * Layout: K slots per row (K = ncpr * threads of the reference), column-major with leading
 * dimension ld (a multiple of 64): slot k of row r is at k*ld + r.  Slot order within a row
 * is the reference's summation order.  Padding slots hold Aj = -1 and Ax = 0.  Column indices
 * are 32-bit.  Aj and Ax must be 16-byte aligned (cudaMalloc / torch allocations are).
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    int64_t rows, cols;
    int64_t K;        /* slots per row                                         */
    int64_t ld;       /* leading dimension, multiple of 64, >= rows            */
    int32_t *Aj;      /* device int32[K*ld]                                    */
    void *Ax;         /* device double[K*ld] or float[K*ld]                    */
    int32_t dtype;    /* hb_dtype                                              */
    int32_t pad_;
} hb_ell;

/* Device layout for a reference ELL matrix with `rows` rows, `ncpr` columns per row and
 * `threads` lanes: *K = ncpr*threads, *ld = rows rounded up to 64. */
int hb_ell_layout(int64_t rows, int64_t ncpr, int64_t threads, int64_t *K, int64_t *ld);

/* Import a reference SparseMatrixELL whose arrays (u64 Aj, Ax, u64 Arl, reference layout
 * (k%T) + r*T + (k/T)*stride) are already on the device, into the hb_ell layout in `out`
 * (out->Aj / out->Ax preallocated, out->rows/cols/K/ld set, e.g. from hb_ell_layout).
 * Replaces the upload half of MemoryBackend<tags::GPU::CUDA>::upload for matrices
 * (honei/backends/cuda/memory_backend.cc) plus the narrowing of the 64-bit indices. */
int hb_ell_import_f64(hb_context *ctx, int64_t rows, int64_t cols, int64_t stride, int64_t ncpr,
                      int64_t threads, const uint64_t *Aj_ref, const double *Ax_ref,
                      const uint64_t *Arl_ref, hb_ell *out);
int hb_ell_import_f32(hb_context *ctx, int64_t rows, int64_t cols, int64_t stride, int64_t ncpr,
                      int64_t threads, const uint64_t *Aj_ref, const float *Ax_ref,
                      const uint64_t *Arl_ref, hb_ell *out);
/* Debug check of a device ELL matrix (no reference counterpart: the reference's kernels trust
 * their indices): *bad_slots receives the number of slots whose column is neither the padding
 * mark -1 nor inside [0, cols).  The product kernels assume 0 (hb_ell_import and the
 * assemblers guarantee it); run this once on a matrix built by hand before using it.
 * Synchronises ctx's stream. */
int hb_ell_validate(hb_context *ctx, const hb_ell *A, int64_t *bad_slots);
/* Same pattern, values cast to float (for the FP32 inner solves of mixed precision). */
int hb_ell_cast_f64_f32(hb_context *ctx, const hb_ell *src, hb_ell *dst);

/* Locality order of a square device ELL matrix.  No reference counterpart: the reference
 * multiplies in the row order the matrix has (Product<Tag> on SparseMatrixELL,
 * honei/la/product.hh:148-204).  A Cuthill-McKee breadth-first order of the matrix graph (row ->
 * its columns): from the row with the fewest off-diagonal entries (lowest index on ties), each
 * level's newly reached rows in the order of the first row reaching them, then by slot; rows
 * never reached follow in ascending order.  order: device int32[rows], order[k] = the row at
 * position k; pos: device int32[rows] or NULL, pos[order[k]] = k.  info (host int64[3], may be
 * NULL): levels, rows reached, start row.  Uses the context workspace (8 bytes per row, 12
 * without pos, plus 8 bytes per block of the grid-wide form) and synchronises the stream.
 * Deterministic: from 4096 rows on the whole GPU computes it (one cooperative launch, three
 * bounded grid-wide exchanges per level; HB_ERR_TIMEOUT if one gives up), the same order as the
 * one-block form below that size. */
int hb_ell_cm_order(hb_context *ctx, const hb_ell *A, int32_t *order, int32_t *pos, int64_t *info);
/* max |pos[c] - pos[r]| over A's stored entries (r, c); pos NULL = A's own numbering.
 * Synchronises the stream. */
int hb_ell_bandwidth(hb_context *ctx, const hb_ell *A, const int32_t *pos, int64_t *bandwidth);
/* B = A's rows in `order` (B row k = A row order[k], its slots in their order): with pos NULL
 * the columns stay A's; with pos the columns are renumbered (B = P A P^T, square A).  B has A's
 * K and ld and its own arrays (caller-allocated). */
int hb_ell_permute(hb_context *ctx, const hb_ell *A, const int32_t *order, const int32_t *pos, hb_ell *B);
/* Product through a row-reordered copy B (hb_ell_permute): y[order[k]] = sum over B's row k of
 * B(k, j) x[j].  With B's columns A's own (pos NULL above), x is A's x and y = A x bit for bit
 * (each row's sum is the same as Product<tags::CPU>'s).  With renumbered columns, x must be
 * gathered first (hb_gather: xw[k] = x[order[k]]); y is then again A x, bit for bit.  order
 * must be 16-byte aligned.  Asynchronous. */
int hb_spmv_rows_f64(hb_context *ctx, const hb_ell *B, const int32_t *order, const double *x, double *y);
int hb_spmv_rows_f32(hb_context *ctx, const hb_ell *B, const int32_t *order, const float *x, float *y);
/* The copy whose gathers are local: B row k = A row order[k] with its columns renumbered through
 * pos (B = P A P^T, square A) and its stored slots sorted by the new column, so the slots of
 * neighbouring rows point at neighbouring entries of the permuted x.  ranks (device uint64[rows])
 * records, 4 bits per stored slot, that slot's place in A's row -- the reference's summation
 * order -- so the product can still add in that order.  K <= 16 (HB_ERR_UNSUPPORTED above).
 * B has A's K and ld and its own arrays (caller-allocated).  Asynchronous. */
int hb_ell_permute_sorted(hb_context *ctx, const hb_ell *A, const int32_t *order, const int32_t *pos, hb_ell *B,
                          uint64_t *ranks);
/* The product through such a sorted copy: y[order[k]] = B's row k summed in the ranks' order,
 * with x already permuted (hb_gather: xw[k] = x[order[k]]); y = A x bit for bit (one row per
 * thread; each row's products wait in shared memory for their turn).  Asynchronous. */
int hb_spmv_ranked_f64(hb_context *ctx, const hb_ell *B, const int32_t *order, const uint64_t *ranks, const double *x,
                       double *y);
int hb_spmv_ranked_f32(hb_context *ctx, const hb_ell *B, const int32_t *order, const uint64_t *ranks, const float *x,
                       float *y);
/* xw[k] = x[order[k]], k < n.  Asynchronous. */
int hb_gather_f64(hb_context *ctx, int64_t n, const int32_t *order, const double *x, double *xw);
int hb_gather_f32(hb_context *ctx, int64_t n, const int32_t *order, const float *x, float *xw);
/* The packed form of a renumbered copy (hb_ell_permute with pos; no reference counterpart, it
 * only shrinks the index traffic of the product): Bd (device int16[K * ld]) = each stored column
 * as its offset from the row, INT16_MIN for padding.  K <= 9; HB_ERR_UNSUPPORTED when an offset
 * is outside +-32767 (the copy's bandwidth is too large; use the ranked product).  Synchronises
 * the stream. */
int hb_ell_pack_offsets(hb_context *ctx, const hb_ell *B, int16_t *Bd);
/* The product through the packed form: y[order[k]] = B's row k, x already permuted (hb_gather);
 * B supplies rows, K, ld and the values (its Aj is not read).  Each row sums its slots in their
 * order, which the renumbered copy keeps: y = A x bit for bit.  Asynchronous. */
int hb_spmv_packed_f64(hb_context *ctx, const hb_ell *B, const int16_t *Bd, const int32_t *order, const double *x,
                       double *y);
int hb_spmv_packed_f32(hb_context *ctx, const hb_ell *B, const int16_t *Bd, const int32_t *order, const float *x,
                       float *y);

/* SPAI2<tags::GPU::CUDA>::value(M, A) (honei/math/spai2.hh:294-298; wrapper
 * honei/math/spai2-cuda.cc:180-228): the sparse approximate inverse of the square matrix A with
 * A's pattern, bit-identical to SPAI2<tags::CPU::SSE> (honei/math/spai2.hh:129-260): for every
 * column the normal equations of the least-squares problem on the rows A's pattern reaches,
 * solved by LU without pivoting.  M is caller-allocated with A's rows, cols, K and ld (M->Aj
 * may be A->Aj; M->Ax must not be A->Ax); it receives A's pattern and the SPAI values, the
 * columns whose system is empty keeping A's values (M = A.copy() first, as the reference).
 * Entries are the slots whose value is not 0.  HB_ERR_UNSUPPORTED when one column's system
 * does not fit in shared memory (columns of more than about 150 entries in FP64, 220 in FP32)
 * or a column holds more than 256 entries.  Uses the context workspace (about 8 * (K + 2) bytes
 * per row) and synchronizes the stream once. */
int hb_spai2_f64(hb_context *ctx, const hb_ell *A, hb_ell *M);
int hb_spai2_f32(hb_context *ctx, const hb_ell *A, hb_ell *M);

/* ------------------------------------------------------------------------------------------
 * Device CSR matrix.  Replaces the device copies of SparseMatrixCSR's Ar/Aj/Ax arrays
 * (honei/la/sparse_matrix_csr.hh) that the reference uploads for its CSR product kernel
 * (cuda_product_csr_dv_{float,double}, honei/backends/cuda/operations.hh, product.cu:257-296).
 *
 * Layout: Ar int64[rows + 1] block offsets (Ar[0] = 0, non-decreasing, Ar[rows] = nblocks);
 * Aj int32[nblocks] the first column of each block (csr::blocksize values per block); Ax
 * dtype[nblocks * blocksize].  Block columns at or beyond cols are stored as cols: every lane of
 * such a block lies outside the matrix, as in the reference, whose product skips lanes whose
 * column is not below cols.
 * ---------------------------------------------------------------------------------------- */
typedef struct hb_csr {
    int64_t rows, cols;
    int64_t blocksize;   /* csr::blocksize */
    int64_t nblocks;
    int64_t *Ar;         /* device */
    int32_t *Aj;         /* device */
    void *Ax;            /* device */
    int32_t dtype;       /* HB_F64 / HB_F32 */
    int32_t pad_;
} hb_csr;

/* Import a reference SparseMatrixCSR whose arrays (uint64 Ar[rows + 1], uint64 Aj[nblocks],
 * values Ax[nblocks * blocksize]) are already on the device into out (out->Ar/Aj/Ax
 * preallocated; out->rows, cols, blocksize, nblocks set).  Replaces the matrix half of
 * MemoryBackend<tags::GPU::CUDA>::upload for SparseMatrixCSR plus the narrowing of the 64-bit
 * indices.  HB_ERR_INVALID when Ar is not a valid offset array (checked on the device; the
 * call synchronises ctx's stream); HB_ERR_UNSUPPORTED for cols or rows beyond 2^31 - 2. */
int hb_csr_import_f64(hb_context *ctx, const uint64_t *Ar_ref, const uint64_t *Aj_ref, const double *Ax_ref,
                      hb_csr *out);
int hb_csr_import_f32(hb_context *ctx, const uint64_t *Ar_ref, const uint64_t *Aj_ref, const float *Ax_ref,
                      hb_csr *out);

/* Q1 Poisson assembly on the device (the FillMatrix<POISSON, DIRICHLET_0> stencil,
 * honei/math/fill_matrix.hh:37-77, built straight into hb_ell layout, K = 9): M x M nodes,
 * Dirichlet rows identity; coef = NULL (unit) or device double[(M-1)^2] cell coefficients
 * (bilinear element matrix k/6 [[4,-1,-2,-1],...]).  symmetric = 0 keeps the interior rows'
 * couplings to boundary nodes, as FillMatrix does (non-symmetric); symmetric = 1 drops them
 * (Dirichlet values eliminated into the right-hand side), which makes the matrix SPD.
 * out->Aj/Ax preallocated with K=9, ld from hb_ell_layout(M*M, 9, 1).  Identical to the host
 * generator (honei_b200/problems.py) bit for bit. */
int hb_q1_assemble_f64(hb_context *ctx, int64_t M, const double *coef, int symmetric, hb_ell *out);

/* HONEI's binary ELL files (MatrixIO<io_formats::ELL>, honei/math/matrix_io.hh:433-582): five
 * uint64 {size, rows, columns, stride, num_cols_per_row}, uint64 Aj[size], double Ax[size].
 * hb_ell_file_info fills info[5] with that header.  hb_ell_read_file_* streams the file into
 * the caller's hb_ell (Aj/Ax allocated for hb_ell_layout(rows, num_cols_per_row, 1)), keeping
 * each row's slots up to its first zero value as the reference's raw-array constructor does
 * (honei/la/sparse_matrix_ell-impl.hh:184-206); _f32 rounds the values as read_matrix's
 * convert does.  hb_ell_write_file writes an FP64 hb_ell in the reference's one-lane layout
 * (zero values dropped, num_cols_per_row = longest row, stride = rows rounded up to 32).
 * HB_ERR_NOT_FOUND: the file cannot be opened; HB_ERR_INVALID: a short or inconsistent file, or
 * a column index out of range. */
int hb_ell_file_info(const char *path, int64_t *info);
int hb_ell_read_file_f64(hb_context *ctx, const char *path, hb_ell *out);
int hb_ell_read_file_f32(hb_context *ctx, const char *path, hb_ell *out);
int hb_ell_write_file(hb_context *ctx, const hb_ell *A, const char *path);

/* ------------------------------------------------------------------------------------------
 * Operators (the static value() functions of the tag-dispatched API).
 * ---------------------------------------------------------------------------------------- */
/* y = A x.  Product<tags::GPU::CUDA>::value(DenseVector&, const SparseMatrixELL&, const
 * DenseVector&), honei/la/product.hh:1758-1760; replaces cuda_product_smell_dv_{float,double}
 * (honei/backends/cuda/operations.hh, honei/backends/cuda/product.cu:356-401).
 * Per-row sum in the reference order, one rounding per multiply and per add: bit-identical to
 * Product<tags::CPU> (honei/la/product.hh:148-204). */
int hb_spmv_f64(hb_context *ctx, const hb_ell *A, const double *x, double *y);
int hb_spmv_f32(hb_context *ctx, const hb_ell *A, const float *x, float *y);

/* r = b - A x.  Defect<tags::GPU::CUDA>::value, honei/math/defect.hh:660-670; replaces
 * cuda_defect_smell_dv_{float,double} (honei/backends/cuda/defect.cu:367-416).
 * Bit-identical to Defect<tags::CPU> (honei/math/defect.hh:357-383). */
int hb_defect_f64(hb_context *ctx, const hb_ell *A, const double *b, const double *x, double *r);
/* RISmoother<tags::GPU::CUDA>::value(A, P, b, x, temp_vecs, sweeps) (honei/math/ri.hh:97-133)
 * with a vector P: `sweeps` times x = x + P (b - A x), each sweep one fused kernel rounding as
 * Defect, Product(P, .) and Sum do (bit-identical to tags::CPU).  tmp: a device vector of rows
 * entries other than x (the sweep reads x while it writes).  Asynchronous. */
int hb_jacobi_sweeps_f64(hb_context *ctx, const hb_ell *A, const double *P, const double *b, double *x, double *tmp,
                         int64_t sweeps);
int hb_jacobi_sweeps_f32(hb_context *ctx, const hb_ell *A, const float *P, const float *b, float *x, float *tmp,
                         int64_t sweeps);
int hb_defect_f32(hb_context *ctx, const hb_ell *A, const float *b, const float *x, float *r);

/* BandedMatrixQx<Q1Type, DT> (honei/la/banded_matrix_qx.hh:44-129): the nine-band matrix of a
 * square Q1 grid, one device array of n values per band, in the Q1BandIndex order LL, LD, LU,
 * DL, DD, DU, UL, UD, UU (honei/la/band_type.hh); band k of row i multiplies x at i + offset_k,
 * offsets -root-1, -root, -root+1, -1, 0, 1, root-1, root, root+1, root = floor(sqrt(n)). */
typedef struct {
    int64_t n;          /* rows = columns */
    int64_t root;       /* floor(sqrt(n)); set by hb_q1band_fill_poisson / hb_q1band_from_ell */
    void *band[9];      /* device pointers, n values each (16-byte aligned for vector loads) */
    int32_t dtype;      /* hb_dtype */
    int32_t pad_;
} hb_q1band;
int64_t hb_q1band_root(int64_t n);
/* y = A x.  Product<tags::GPU::CUDA>::value(DenseVector&, const BandedMatrixQx<Q1Type>&, const
 * DenseVectorContinuousBase&), honei/la/product.hh:1750-1756; replaces
 * cuda_product_bmdv_q1_{float,double} (honei/backends/cuda/product.cu:30-145).  Bit-identical
 * to Product<tags::CPU> (honei/la/product.hh:371-404): DD x[i] first, then the eight other
 * bands in index order, each only where its column lies in [0, n). */
int hb_q1band_spmv_f64(hb_context *ctx, const hb_q1band *A, const double *x, double *y);
int hb_q1band_spmv_f32(hb_context *ctx, const hb_q1band *A, const float *x, float *y);
/* r = b - A x.  Defect<tags::GPU::CUDA>::value on BandedMatrixQx, honei/math/defect.hh:
 * 645-658; bit-identical to Defect<tags::CPU> (honei/math/defect.hh:194-199). */
int hb_q1band_defect_f64(hb_context *ctx, const hb_q1band *A, const double *b, const double *x, double *r);
int hb_q1band_defect_f32(hb_context *ctx, const hb_q1band *A, const float *b, const float *x, float *r);
/* FillMatrix<Tag, POISSON, DIRICHLET_0>::value(BandedMatrixQx&), honei/math/fill_matrix.hh:
 * 41-77, on an M x M grid (A->n = M^2, A->dtype and A->band[] set by the caller). */
int hb_q1band_fill_poisson(hb_context *ctx, int64_t M, hb_q1band *A);
/* BandedMatrixQx(SparseMatrixELL&), honei/la/banded_matrix_qx-impl.hh:111-167: band k of row
 * i = A(i, i + offset_k) where that column exists, 0 elsewhere.  n must be a square and every
 * non-zero entry of E must lie on one of the nine bands (HB_ERR_UNSUPPORTED otherwise: the
 * conversion would drop it); E->dtype == A->dtype. */
int hb_q1band_from_ell(hb_context *ctx, const hb_ell *E, hb_q1band *A);

/* Matrix-free geometric transfers of (2^k + 1)^2 grids: Prolongation<Tag, methods::NONE>
 * ::value(fine, coarse, mask, prolmat) (honei/math/prolongation.hh:42-139) and
 * Restriction<Tag, methods::NONE>::value(coarse, fine, mask, resmat) (honei/math/
 * restriction.hh:41-170), each followed by ApplyDirichletBoundaries with the host array
 * mask[8] (corners bottom-left, bottom-right, top-right, top-left, edges bottom, right, top,
 * left; 2 = zero those nodes).  n_fine = Mf^2 with Mf odd (HB_ERR_UNSUPPORTED otherwise); the
 * coarse vector has ((Mf - 1) / 2 + 1)^2 entries.  Bit-identical to tags::CPU: every node
 * replays the reference's sequence of += updates, evaluated in double and stored as T. */
int hb_prolongate_f64(hb_context *ctx, int64_t n_fine, double *fine, const double *coarse, const uint64_t *mask);
int hb_prolongate_f32(hb_context *ctx, int64_t n_fine, float *fine, const float *coarse, const uint64_t *mask);
int hb_restrict_f64(hb_context *ctx, int64_t n_fine, double *coarse, const double *fine, const uint64_t *mask);
int hb_restrict_f32(hb_context *ctx, int64_t n_fine, float *coarse, const float *fine, const uint64_t *mask);

/* Host scalar results (synchronous, like the reference's value-returning operators).
 * DotProduct<tags::GPU::CUDA>::value, honei/la/dot_product.hh:358-360 (replaces
 * cuda_dot_product_two_{float,double}, honei/backends/cuda/dot_product.cu:77-155);
 * Norm<vnt_l_two, root, tags::GPU::CUDA>::value, honei/la/norm.hh:551-574 (root = 0 returns
 * the squared norm, as Norm<vnt_l_two, false> does). */
int hb_dot_f64(hb_context *ctx, int64_t n, const double *x, const double *y, double *result_host);
int hb_dot_f32(hb_context *ctx, int64_t n, const float *x, const float *y, float *result_host);
int hb_norm_l2_f64(hb_context *ctx, int64_t n, const double *x, int root, double *result_host);
int hb_norm_l2_f32(hb_context *ctx, int64_t n, const float *x, int root, float *result_host);

/* x += b*y  (ScaledSum(x, y, b), honei/la/scaled_sum.hh:461-466)
 * r = x + b*y (ScaledSum(r, x, y, b), honei/la/scaled_sum.hh:467-471) */
int hb_scaled_sum_f64(hb_context *ctx, int64_t n, double *x, const double *y, double b);
int hb_scaled_sum_f32(hb_context *ctx, int64_t n, float *x, const float *y, float b);
int hb_scaled_sum3_f64(hb_context *ctx, int64_t n, double *r, const double *x, const double *y, double b);
int hb_scaled_sum3_f32(hb_context *ctx, int64_t n, float *r, const float *x, const float *y, float b);
/* x *= a (Scale, honei/la/scale.hh:263); x += y (Sum, honei/la/sum.hh:684);
 * r = x - y (Difference); r = x * y elementwise (ElementProduct; also the Jacobi apply
 * Product(DV, DV, DV), honei/la/product.hh:1198-1204). */
int hb_scale_f64(hb_context *ctx, int64_t n, double *x, double a);
int hb_scale_f32(hb_context *ctx, int64_t n, float *x, float a);
int hb_sum_f64(hb_context *ctx, int64_t n, double *x, const double *y);
int hb_sum_f32(hb_context *ctx, int64_t n, float *x, const float *y);
int hb_difference_f64(hb_context *ctx, int64_t n, double *r, const double *x, const double *y);
int hb_difference_f32(hb_context *ctx, int64_t n, float *r, const float *x, const float *y);
int hb_element_product_f64(hb_context *ctx, int64_t n, double *r, const double *x, const double *y);
int hb_element_product_f32(hb_context *ctx, int64_t n, float *r, const float *x, const float *y);
/* copy / fill / precision conversion: copy<Tag>, fill<Tag>, convert<Tag>
 * (honei/la/algorithm.hh:50-86,163-198; MemoryBackend copy/fill/convert_float_double/
 * convert_double_float, honei/backends/cuda/transfer.cu:28-46,153-159). */
int hb_copy(hb_context *ctx, void *dst, const void *src, int64_t bytes);
int hb_fill_f64(hb_context *ctx, int64_t n, double *x, double value);
int hb_fill_f32(hb_context *ctx, int64_t n, float *x, float value);
int hb_convert_f64_f32(hb_context *ctx, int64_t n, float *dst, const double *src);
int hb_convert_f32_f64(hb_context *ctx, int64_t n, double *dst, const float *src);

/* y = A x on SparseMatrixCSR: Product<tags::GPU::CUDA>::value(DV, SparseMatrixCSR, DV)
 * (honei/la/product.hh:1762-1764) with the tags::CPU arithmetic (honei/la/product.hh:209-242):
 * per row, its blocks and their lanes in order, lanes whose column is not below cols skipped;
 * bit-identical to tags::CPU.  r = rhs - A x: Defect<tags::GPU::CUDA>::value(DV, DV,
 * SparseMatrixCSR, DV) (honei/math/defect.hh:673-676; tags::CPU honei/math/defect.hh:386-419).
 * x has cols entries, y / rhs / r rows; asynchronous on ctx's stream. */
int hb_csr_spmv_f64(hb_context *ctx, const hb_csr *A, const double *x, double *y);
int hb_csr_spmv_f32(hb_context *ctx, const hb_csr *A, const float *x, float *y);
int hb_csr_defect_f64(hb_context *ctx, const hb_csr *A, const double *rhs, const double *x, double *r);
int hb_csr_defect_f32(hb_context *ctx, const hb_csr *A, const float *rhs, const float *x, float *r);

/* ------------------------------------------------------------------------------------------
 * Solvers.
 * ---------------------------------------------------------------------------------------- */
/* Plain CG, CGSolver<Tag, methods::NONE>::value(A, P, b, x, max_iters, used_iters, eps),
 * honei/math/cg.hh:63-133: same update formulas, the same guarded divisions and the same dual
 * stopping rule (sqrt(alpha) < eps*sqrt(alpha0) or sqrt(alpha) < eps).  The whole loop runs
 * in ONE persistent cooperative kernel (2 grid-wide reductions per iteration, scalars on the
 * device); x holds x0 on entry and the solution on exit.  *used_iters (host) receives the
 * iteration count, *final_defect (host, may be NULL) sqrt(alpha) at exit.  Systems whose rows
 * fit the shared memory of one block per SM run in the resident-operator kernel (matrix rows
 * and vector windows kept on chip for the whole solve); larger ones stream the matrix each
 * iteration.  Returns HB_ERR_TIMEOUT if a bounded device-side wait gave up. */
int hb_cg_f64(hb_context *ctx, const hb_ell *A, const double *b, double *x, int64_t max_iters,
              double eps, int64_t *used_iters, double *final_defect);
int hb_cg_f32(hb_context *ctx, const hb_ell *A, const float *b, float *x, int64_t max_iters,
              float eps, int64_t *used_iters, float *final_defect);

/* Selects whether hb_cg_f64 / hb_cg_f32 and hb_cg_var_diag_f64 / _f32 on this context use the
 * resident-operator kernels where they apply (enable != 0, the default) or always the
 * streaming kernels.  Both give
 * results within rounding of each other (their dot products use different summation trees);
 * each is deterministic.  Returns the previous setting. */
int hb_cg_set_resident(hb_context *ctx, int enable);
/* Selects the streaming CG kernel's layout on this context: rows_per_thread 4 (groups of four
 * rows per thread, 16-byte loads; the default) or 1 (one row per thread, every slot of the row in
 * flight, more threads per SM).  Same formulas and per-row sums; the dot products' partial sums
 * group the rows differently, so the iterates agree to rounding.  Returns the previous setting,
 * or -1 for an invalid argument. */
int hb_cg_set_layout(hb_context *ctx, int rows_per_thread);
/* Threads per block of a kernel family on this context, the knob HONEI's honeirc keys set for
 * its CUDA kernels (honei/honeirc: cuda::product_smell_dv_*, cuda::product_bmdv_q1_*,
 * cuda::scaled_sum_two_* and the other vector keys; read at honei/la/product-cuda.cc:594-625,
 * honei/la/scaled_sum-cuda.cc:210-236, honei/la/difference-cuda.cc:184-210):
 *   HB_BLOCK_ELL     the ELL product / defect / Jacobi-sweep kernel (4 rows per thread): 32..256
 *   HB_BLOCK_Q1BAND  the banded Q1 kernels: 32..256
 *   HB_BLOCK_VECTOR  the elementwise vector kernels (scaled sums, scale, sum, difference,
 *                    element product, fill): 32..1024
 * in multiples of 32; 0 restores the library's default (256).  Results do not depend on it (each
 * output element is computed by one thread in a fixed order).  The dot-product and norm kernels
 * keep their fixed reduction tree (and so their bits) and have no such knob.  Returns the
 * previous setting (0 = default), or -1 for an invalid family or size. */
enum { HB_BLOCK_ELL = 0, HB_BLOCK_Q1BAND = 1, HB_BLOCK_VECTOR = 2 };
int hb_set_block_size(hb_context *ctx, int family, int threads);

/* Preconditioned CG, CGSolver<Tag, methods::VAR>::value(A, P, b, x, max_iters, used_iters,
 * eps), honei/math/cg.hh:140-219, with the preconditioner container P either a vector (the
 * _diag entry points: z = P r elementwise, e.g. Jacobi P = damping / diag(A)) or an ELL matrix
 * of A's size (the _ell entry points: z = P r, e.g. SPAI / SAINV approximate inverses).  Same
 * update order, sign-keeping division guards and stopping tests (||r|| < eps ||r0||,
 * ||r|| < eps, max_iters) as the reference; one persistent kernel per solve.  *final_defect
 * (may be NULL) = ||r|| at exit. */
int hb_cg_var_diag_f64(hb_context *ctx, const hb_ell *A, const double *P, const double *b, double *x,
                       int64_t max_iters, double eps, int64_t *used_iters, double *final_defect);
int hb_cg_var_diag_f32(hb_context *ctx, const hb_ell *A, const float *P, const float *b, float *x,
                       int64_t max_iters, float eps, int64_t *used_iters, float *final_defect);
int hb_cg_var_ell_f64(hb_context *ctx, const hb_ell *A, const hb_ell *P, const double *b, double *x,
                      int64_t max_iters, double eps, int64_t *used_iters, double *final_defect);
int hb_cg_var_ell_f32(hb_context *ctx, const hb_ell *A, const hb_ell *P, const float *b, float *x,
                      int64_t max_iters, float eps, int64_t *used_iters, float *final_defect);

/* Self-test of the bounded device waits (no reference counterpart): one block waits for an
 * arrival that never comes, first at a grid barrier, then at an arrival-counter exchange (the
 * CG kernels' reductions); each wait gives up after its limit (2 s), records the timeout in the
 * context's status word and the kernel returns.  Returns HB_ERR_TIMEOUT when both happened as
 * designed; the context stays usable. */
int hb_selftest_wait_timeout(hb_context *ctx);

/* Allocation-free variant of hb_cg_f64.  This entry point has no counterpart in the reference.
 * It is for callers that cannot allocate device memory when they solve: real-time or embedded
 * hosts that forbid allocation after start-up (an allocation may block for an unbounded
 * time), and processes whose device memory is held entirely by another framework's caching
 * allocator (a cudaMalloc there fails although that memory is idle).  It needs no hb_context:
 * its work vectors, reduction partials, barrier words and result record live in one static
 * __device__ array of about 5.3 MB, which every GPU that loads this library in a process keeps
 * until the process exits.
 * Limit: A->rows <= 131072 (FP64; e.g. the 257 x 257 Q1 grid); larger systems return
 * HB_ERR_UNSUPPORTED without launching.  The caller passes A, b, x (device) and the stream
 * (cudaStream_t, NULL = legacy stream); `stream` must belong to the current device
 * (HB_ERR_INVALID otherwise).  Results as for hb_cg_f64: the call copies its result record to
 * the host and synchronises `stream` before it returns.  It calls no cudaMalloc, cudaFree or
 * other allocating routine.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; a lookup that fails is retried by the next
 * call.  The array is per process and per device: all calls in one process on one device share
 * it, so such calls that overlap on the GPU (different streams or host threads at once) race
 * and must be serialised by the caller.  The barrier words are re-zeroed by every call. */
int hb_cg_f64_noalloc(const hb_ell *A, const double *b, double *x, int64_t max_iters, double eps,
                      int64_t *used_iters, double *final_defect, void *stream);

/* Multigrid (MGData + MGCycleCreation<V::STATIC, CGSolver<NONE>, RISmoother, Restriction
 * <PROLMAT>, Prolongation<PROLMAT>> + MGSolver<Norm<l2, true>>, honei/math/mg.hh:57-243,
 * 567-662, 1093-1127; RISmoother honei/math/ri.hh:97-133 with the "jac" preconditioner
 * damping/diag(A), honei/math/mg.hh:255-286).  Levels are given coarsest first (HONEI level
 * 1 first); prol[l] maps level l to l+1, res[l] = prol[l]^T.  All matrices share one dtype.
 * The hierarchy object owns its per-level work vectors. */
typedef struct hb_mg hb_mg;
typedef struct {
    int64_t max_iters;         /* V-cycles                                        */
    int64_t max_iters_coarse;  /* CG iterations on level 1                        */
    int64_t n_pre, n_post;     /* smoothing sweeps                                */
    double damping;            /* Jacobi damping (0.7 in the north-star configs)  */
    double eps;                /* relative stop on ||r||_2; also the coarse CG eps */
} hb_mg_params;

int hb_mg_create(hb_context *ctx, int nlevels, const hb_ell *A, const hb_ell *prol,
                 const hb_ell *res, const hb_mg_params *params, hb_mg **out);
/* The same multigrid on square Q1 grids with banded level matrices B[l] (hb_q1band; coarse side
 * = finer side / 2 + 1, the 2:1 coarsening for (2^k + 1) sides) and matrix-free bilinear
 * transfers with Dirichlet fine rows zero (the PROLMAT matrices, never stored).  Levels >= 1 smooth and take
 * defects with B[l]; level 0 keeps A[0] for its coarse CG; A[l] also gives the Jacobi diagonals.
 * Every operation rounds as the ELL cycle on the same matrices (bit-identical iterates); per fine
 * row the cycle reads no column indices and no transfer matrix. */
int hb_mg_create_banded(hb_context *ctx, int nlevels, const hb_ell *A, const hb_q1band *B, const hb_mg_params *params,
                        hb_mg **out);
int hb_mg_destroy(hb_mg *mg);
int hb_mg_set_params(hb_mg *mg, const hb_mg_params *params);
/* Solve on the finest level: x holds x0 on entry.  *used_cycles (host) and
 * rnorm_host[2] = {initial, final} defect norms (may be NULL). */
int hb_mg_solve_f64(hb_mg *mg, const double *b, double *x, int64_t *used_cycles, double *rnorm_host);
int hb_mg_solve_f32(hb_mg *mg, const float *b, float *x, int64_t *used_cycles, float *rnorm_host);
/* One V-cycle on the finest level, x updated in place: what one OperatorList::value() call of
 * the cycle MGCycleCreation<Tag, V::STATIC, CGSolver<NONE>, RISmoother, Restriction<PROLMAT>,
 * Prolongation<PROLMAT>> builds does (honei/math/mg.hh:567-662).  Asynchronous. */
int hb_mg_cycle_f64(hb_mg *mg, const double *b, double *x);
int hb_mg_cycle_f32(hb_mg *mg, const float *b, float *x);
/* The smoother vector of one level (0 = coarsest) taken from the caller (device, rows entries,
 * the hierarchy's dtype), in place of damping / diag(A): MGData's P[l] as PreconFill built it
 * (honei/math/mg.hh:255-286).  A later hb_mg_set_params that changes the damping recomputes
 * damping / diag(A). */
int hb_mg_set_smoother(hb_mg *mg, int level, const void *P);

/* Mixed precision iterative refinement, IRSolver<Outer=double, Inner=float>,
 * honei/math/ir.hh:30-78: FP64 defect b - A x, convergence norm and solution update on the
 * device; FP32 inner MG (mg32, eps and cycle count from its params) on the cast defect.
 * warm_start != 0 is the reference's loop: the cast defect is the inner right-hand side and
 * the inner x is kept between outer steps (ir.hh:69-73).  warm_start = 0 is the scaled mode:
 * the defect is normalised to unit norm before the cast, the inner solve starts from zero and
 * x += |r| * c, so the inner eps is relative to each step's defect.
 * *used_outer (host) gets the outer step count; rnorm_host[2] = {initial, final}. */
int hb_ir_mg_solve(hb_context *ctx, const hb_ell *A64, hb_mg *mg32, const double *b, double *x,
                   double eps, int64_t max_iters, int warm_start, int64_t *used_outer,
                   double *rnorm_host);
/* The same outer loop, scaled mode, with an FP32 CG inner solver (A32 = A64 cast) from zero:
 * the normalised defect keeps CGSolver's absolute stopping test (cg.hh:118) from ending the
 * inner solve early, so inner_eps is relative.  *inner_total = summed inner CG iterations. */
int hb_ir_cg_solve(hb_context *ctx, const hb_ell *A64, const hb_ell *A32, const double *b, double *x,
                   double eps, float inner_eps, int64_t inner_max_iters, int64_t max_iters,
                   int64_t *used_outer, int64_t *inner_total, double *rnorm_host);

/* ------------------------------------------------------------------------------------------
 * Batched solves (no reference counterpart: HONEI solves one system per CGSolver call).
 * Many independent systems of uneven size in ONE persistent launch: each system is solved by
 * one thread-block cluster (hardware cluster barriers, DSMEM reductions), clusters pull
 * systems largest-first from a device work counter.  A system's result depends only on the
 * system and the launch shape, never on what else is in the batch (same answer alone and in
 * the mix, bit for bit).
 *   HB_BATCH_CG64: plain FP64 CG with CGSolver<NONE>'s update formulas and dual stopping rule.
 *   HB_BATCH_IR32: FP64 outer refinement (defect, norm, update in FP64) around FP32 CG with
 *                  FP32 accumulation on the normalised defect to inner_eps per outer step,
 *                  until ||b - A x|| < eps ||b - A x0||.
 * A64 is always required (FP64 values); A32 (same pattern, FP32 values) for HB_BATCH_IR32.
 * ---------------------------------------------------------------------------------------- */
enum { HB_BATCH_CG64 = 0, HB_BATCH_IR32 = 1 };

typedef struct {
    hb_ell A64;                /* device matrix, FP64 values                              */
    hb_ell A32;                /* same pattern, FP32 values (HB_BATCH_IR32), else zeroed   */
    const double *b;           /* device, n entries                                       */
    double *x;                 /* device, n entries: x0 in, solution out                  */
    int32_t mode;              /* HB_BATCH_CG64 / HB_BATCH_IR32                           */
    int32_t pad_;
    int64_t max_iters;         /* CG iterations (CG64) / inner CG iterations per step (IR) */
    int64_t max_outer;         /* outer refinement steps (IR)                             */
    double eps;                /* CG64: CGSolver eps; IR: target relative FP64 residual   */
    double inner_eps;          /* IR: inner relative eps (FP32 CG)                        */
} hb_batch_system;

typedef struct {
    int64_t iterations;        /* CG iterations (IR: summed inner iterations)             */
    int64_t outer;             /* outer steps (IR), 0 for CG64                            */
    double defect0;            /* initial defect norm (CG64: sqrt(alpha0))                 */
    double defect;             /* final defect norm (CG64: sqrt(alpha), IR: true FP64)     */
    double true_relres;        /* ||b - A x|| / ||b|| in FP64 after the solve             */
    int32_t status;            /* hb_status                                               */
    int32_t pad_;
} hb_batch_result;

typedef struct {
    int32_t cluster;           /* CTAs per system: 1, 2, 4, 8 or 16                        */
    int32_t threads;           /* threads per CTA: 256 or 512                              */
    int32_t max_clusters;      /* cap on resident clusters (0 = all that fit): leaves SMs
                                  to concurrent work on other streams                      */
    int32_t rows_per_thread;   /* CG rows per thread: 4 (a group of four rows, 16-byte
                                  loads; 0 means 4) or 1 (one row, every slot in flight)   */
} hb_batch_config;

/* Device workspace bytes for these systems (work vectors, descriptors, results, counter). */
int hb_batch_workspace_bytes(const hb_batch_system *sys, int64_t count, size_t *bytes);
/* Solve all systems in one launch (workspace: device, hb_batch_workspace_bytes long, 256-byte
 * aligned).  results_host receives one record per system.  cfg = NULL picks the default
 * (cluster 4, 512 threads).  Synchronous. */
int hb_batch_solve(hb_context *ctx, const hb_batch_system *sys, int64_t count, void *workspace,
                   const hb_batch_config *cfg, hb_batch_result *results_host);
/* Two-step form for CUDA graphs: prepare writes the device descriptors into the workspace
 * (synchronous, once per batch); run only resets the work counter and launches, so it can be
 * captured into a graph and replayed.  Results land in the workspace; hb_batch_results copies
 * them to the host. */
int hb_batch_prepare(hb_context *ctx, const hb_batch_system *sys, int64_t count, void *workspace);
int hb_batch_run(hb_context *ctx, int64_t count, void *workspace, const hb_batch_config *cfg);
int hb_batch_results(hb_context *ctx, int64_t count, void *workspace, hb_batch_result *results_host);
/* Autotuner core: times every (rows per thread, cluster, threads) candidate on this batch (each
 * run once after a warm-up) and returns the fastest in *best; times_ms (may be NULL, else 20
 * entries) receives one time per candidate in the order rows per thread {4,1} x cluster
 * {1,2,4,8,16} x threads {256,512} (-1 = shape not launchable).  Every run starts from x = 0 (the
 * systems' x are zeroed and overwritten). */
int hb_batch_tune(hb_context *ctx, const hb_batch_system *sys, int64_t count, void *workspace,
                  hb_batch_config *best, double *times_ms);

/* ------------------------------------------------------------------------------------------
 * Served Q1 systems: device-built multigrid for grids of ANY side (no reference counterpart;
 * the reference's MG needs pre-built files per level, honei/math/mg.hh:442-547).
 * Coarsening keeps the even-indexed fine nodes plus the last one (coarse side Mf/2 + 1);
 * transfers are Prolongation<methods::NONE>'s bilinear interpolation with fine Dirichlet rows
 * zeroed (honei/math/prolongation.hh:42-139) and its transpose; coarse operators are Galerkin
 * R A P (robust for jumping coefficients), coarse nodes without fine support get identity rows.
 * ---------------------------------------------------------------------------------------- */
/* Coarse side of an Mf x Mf grid. */
int hb_q1_coarse_side(int64_t Mf);
/* P (Nf x Nc, K = 4) and R = P^T (Nc x Nf, K = 9) for an Mf grid, FP64 or FP32 (P->dtype),
 * preallocated with hb_ell_layout. */
int hb_q1_transfers(hb_context *ctx, int64_t Mf, hb_ell *P, hb_ell *R);
/* Galerkin coarse operator Ac = R Af P (FP64, K = 9) of a Q1-structured fine matrix. */
int hb_q1_galerkin(hb_context *ctx, int64_t Mf, const hb_ell *Af, hb_ell *Ac);

typedef struct hb_q1 hb_q1;
/* Builds the SPD Q1 system of an M x M grid (coef: device (M-1)^2 cell coefficients or NULL)
 * with its FP32 MG hierarchy, all device-resident (stream-ordered memory on ctx's stream). */
int hb_q1_create(hb_context *ctx, int64_t M, const double *coef, hb_q1 **out);
int hb_q1_destroy(hb_q1 *q);
int hb_q1_levels(const hb_q1 *q, int *nlevels, int64_t *sides);
/* Level matrices (level 0 = coarsest): FP64 A, FP32 A (shares A64's index array), and the
 * FP32 transfers from this level to the next finer one (levels below the finest only). */
int hb_q1_level(const hb_q1 *q, int level, hb_ell *A64, hb_ell *A32, hb_ell *P32, hb_ell *R32);
/* Mixed-precision solve: FP64 defect, norm and update around FP32 CG preconditioned by one
 * V(2,2) cycle (damped Jacobi 0.7, coarse CG), on the normalised defect to inner_eps, until
 * ||b - A x|| < eps ||b - A x0||.  info: iterations = summed inner PCG iterations, outer,
 * defect0/defect = FP64 defect norms, true_relres = ||b - A x|| / ||b||. */
int hb_q1_solve(hb_q1 *q, const double *b, double *x, double eps, double inner_eps, int64_t max_outer,
                int64_t max_inner, hb_batch_result *info);

/* Runs the coarse levels of the served solve's cycle -- those of at most max_rows rows -- as one
 * single-cluster launch: the same arithmetic as the per-level kernels, so the same iterates, in
 * one launch instead of about eight per level.  max_rows = 0 (the default) runs every level with
 * its own kernels, which measured faster for single solves on B200. */
int hb_q1_set_fused_tail(hb_q1 *q, int64_t max_rows);

/* Batched served solves (no reference counterpart): count distinct hb_q1 systems, each with its
 * own b[i] and x[i] (device, x holds x0), solved in one persistent launch with the algorithm of
 * hb_q1_solve; one thread-block cluster (cfg->cluster CTAs of cfg->threads threads; NULL = 8 x
 * 256) solves one system at a time, largest first, with cluster barriers between phases and
 * DSMEM reductions.  The systems must be ready on ctx's stream (created on it, or synchronised).
 * A system's result does not depend on the rest of the batch.  results[i] as hb_q1_solve's info. */
int hb_q1_batch_solve(hb_context *ctx, hb_q1 *const *systems, const double *const *b, double *const *x, int64_t count,
                      double eps, double inner_eps, int64_t max_outer, int64_t max_inner, const hb_batch_config *cfg,
                      hb_batch_result *results);

/* ------------------------------------------------------------------------------------------
 * Serving (no reference counterpart): a request loop that admits Q1 solve requests by an HBM
 * budget, keeps each admitted request's matrix, hierarchy and Krylov state on the device, and
 * serves them concurrently -- small grids in batched cluster launches (HB_BATCH_IR32), mid-size
 * grids in batched MG-preconditioned cluster launches (hb_q1_batch_solve), large grids on
 * MG-preconditioned mixed-precision workers (hb_q1_solve), each on its own stream --
 * while new requests keep arriving (continuous batching).  A request's result does not depend
 * on what it was served with.  Two baselines run on the same queue: HB_SERVE_PLAIN_CG64, one
 * request at a time, plain FP64 CG (hb_cg_f64) on the whole GPU; and HB_SERVE_PLAIN_CG64_BATCHED,
 * plain FP64 CG with the mixed server's concurrency -- grids up to mid_max_side in batched
 * cluster launches (HB_BATCH_CG64), larger grids on large_workers concurrent hb_cg_f64 streams.
 * ---------------------------------------------------------------------------------------- */
enum { HB_SERVE_MIXED = 0, HB_SERVE_PLAIN_CG64 = 1, HB_SERVE_PLAIN_CG64_BATCHED = 2 };
enum { HB_PATH_BATCH = 0, HB_PATH_MGPCG = 1, HB_PATH_CG64 = 2, HB_PATH_MGBATCH = 3, HB_PATH_BATCH_CG64 = 4 };

typedef struct {
    int32_t mode;               /* HB_SERVE_MIXED, HB_SERVE_PLAIN_CG64 or _PLAIN_CG64_BATCHED  */
    int32_t device;
    int64_t hbm_budget_bytes;   /* admission limit for resident request state                  */
    int32_t large_workers;      /* concurrent MG-PCG solves (one stream each)                  */
    int32_t small_workers;      /* concurrent batched launches (one stream each)               */
    int64_t small_max_side;     /* grid sides <= this take the batched path                    */
    int32_t max_batch;          /* systems per batched launch                                  */
    int32_t pad_;
    hb_batch_config batch_cfg;  /* cluster shape of the batched launches                       */
    double eps;                 /* target relative FP64 residual ||b - A x|| / ||b||           */
    double inner_eps;           /* FP32 inner tolerance per refinement step                    */
    int64_t mid_max_side;       /* sides in (small_max_side, mid_max_side] take the batched
                                   MG-PCG path (hb_q1_batch_solve); 0 = no such path           */
    int32_t mid_workers;        /* concurrent batched MG-PCG launches (one stream each)        */
    int32_t pad2_;
    hb_batch_config mid_cfg;    /* cluster shape of the batched MG-PCG launches                */
    int32_t pad3_;
} hb_server_params;

typedef struct {
    int64_t M;                  /* grid side: an M x M node Q1 system (SPD form)              */
    const double *coef;         /* host, (M-1)^2 cell coefficients, or NULL for 1              */
    const double *b;            /* host, M^2 right-hand side, or NULL: b = A x_true            */
    const double *x_true;       /* host, M^2, used when b == NULL                              */
    double *x;                  /* host, M^2: receives the solution (kept alive by the caller) */
    uint64_t tag;               /* returned in the completion                                  */
} hb_request;

typedef struct {
    uint64_t tag;
    int32_t status;             /* hb_status                                                   */
    int32_t path;               /* HB_PATH_*                                                   */
    int64_t iterations;         /* CG / inner PCG iterations                                   */
    int64_t outer;              /* refinement steps                                            */
    double true_relres;         /* ||b - A x|| / ||b|| in FP64                                  */
    double t_submit, t_admit, t_done;   /* seconds on the server clock                       */
    int64_t bytes;              /* HBM charged to the request while resident                   */
} hb_completion;

typedef struct hb_server hb_server;
int hb_server_create(const hb_server_params *params, hb_server **out);
/* Queues a request (non-blocking); the host arrays must stay valid until its completion. */
int hb_server_submit(hb_server *s, const hb_request *req);
/* Up to max completions (oldest first) into out; waits up to wait_ms for at least one. */
int hb_server_poll(hb_server *s, hb_completion *out, int max, int *n, int wait_ms);
/* Blocks until every submitted request has completed. */
int hb_server_drain(hb_server *s);
/* Seconds since the server started (the clock of the completion records). */
double hb_server_clock(hb_server *s);
/* in_use / peak resident bytes, requests submitted / completed. */
int hb_server_stats(hb_server *s, int64_t *bytes_in_use, int64_t *bytes_peak, int64_t *submitted, int64_t *completed);
/* What the device's stream-ordered memory pool (which holds every request's device memory)
 * actually used and reserved at its highest since the server started, against the admission
 * charges above.  Counts every stream-ordered allocation of the process on that device. */
int hb_server_pool_stats(hb_server *s, int64_t *used_high, int64_t *reserved_high);
int hb_server_destroy(hb_server *s);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* HONEI_B200_H */
