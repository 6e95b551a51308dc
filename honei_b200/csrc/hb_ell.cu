// hb_ell.cu -- device ELL layout, import from the reference layout, Q1 assembly, SpMV, defect.
//
// Data layout in HBM (see include/honei_b200.h): K slots per row, column-major with leading
// dimension ld (multiple of 64), int32 column indices, padding slots Aj = -1 / Ax = 0.  One
// thread owns 4 consecutive rows, so every slot is one 16-byte load of Aj (int4) and one or
// two 16-byte loads of Ax (float4 / 2 x double2), coalesced across the warp; the x gathers go
// through L1/L2 (x is the reusable part of the working set, the matrix is streamed with
// evict-first loads).  Per row the sum runs over the slots in the reference order with one
// rounding per multiply and add, so y is bit-identical to Product<tags::CPU>
// (honei/la/product.hh:148-204).
#include "hb_spmv_core.cuh"

namespace {

constexpr int SPMV_THREADS = 256;

// ---------------------------------------------------------------------------------------
// Import: reference layout (u64 Aj, Ax, u64 Arl; entry k of row r at (k%T) + r*T + (k/T)*stride)
// -> hb_ell layout.  Slot k = g*T + t keeps the reference order (g outer, t inner).
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void ell_import_kernel(int64_t rows, int64_t cols, int64_t stride, int64_t T_,
                                  int64_t K, int64_t ld, const uint64_t *__restrict__ Aj_ref,
                                  const T *__restrict__ Ax_ref, const uint64_t *__restrict__ Arl,
                                  int32_t *__restrict__ Aj, T *__restrict__ Ax, int *bad)
{
    const int64_t total = K * ld;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx / ld, r = idx - k * ld;
        int32_t j = -1;
        T a = T(0);
        if (r < rows) {
            const int64_t g = k / T_, t = k - g * T_;
            if ((uint64_t)g < Arl[r]) {
                const int64_t src = t + r * T_ + g * stride;
                const uint64_t c = Aj_ref[src];
                if (c >= (uint64_t)cols) {
                    atomicExch(bad, 1);
                } else {
                    j = (int32_t)c;
                    a = Ax_ref[src];
                }
            }
        }
        Aj[idx] = j;
        Ax[idx] = a;
    }
}

__global__ void ell_cast_kernel(int64_t total, const double *__restrict__ src, float *__restrict__ dst)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// ---------------------------------------------------------------------------------------
// Q1 Poisson assembly, one thread per row (FillMatrix<POISSON, DIRICHLET_0> stencil, or the
// bilinear element matrix k/6 [[4,-1,-2,-1],...] summed per node for a cell coefficient).
// ---------------------------------------------------------------------------------------
__global__ void q1_assemble_kernel(int64_t M, const double *__restrict__ coef, int64_t ld, int symmetric,
                                   int32_t *__restrict__ Aj, double *__restrict__ Ax)
{
    const int64_t N = M * M;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < ld;
         r += (int64_t)gridDim.x * blockDim.x) {
        int32_t jj[9];
        double vv[9];
#pragma unroll
        for (int s = 0; s < 9; ++s) { jj[s] = -1; vv[s] = 0.0; }
        if (r < N) {
            const int64_t i = r / M, j = r - i * M;
            if (i == 0 || i == M - 1 || j == 0 || j == M - 1) {
                jj[0] = (int32_t)r;
                vv[0] = 1.0;
            } else {
                double knw = 1.0, kne = 1.0, ksw = 1.0, kse = 1.0;
                if (coef) {
                    const int64_t C = M - 1;
                    knw = coef[(i - 1) * C + (j - 1)];
                    kne = coef[(i - 1) * C + j];
                    ksw = coef[i * C + (j - 1)];
                    kse = coef[i * C + j];
                }
                using hbd::add; using hbd::mul;
                const double six = 6.0;
                vv[0] = -__ddiv_rn(mul(2.0, knw), six);
                vv[1] = -__ddiv_rn(add(knw, kne), six);
                vv[2] = -__ddiv_rn(mul(2.0, kne), six);
                vv[3] = -__ddiv_rn(add(knw, ksw), six);
                vv[4] = __ddiv_rn(mul(4.0, add(add(add(knw, kne), ksw), kse)), six);
                vv[5] = -__ddiv_rn(add(kne, kse), six);
                vv[6] = -__ddiv_rn(mul(2.0, ksw), six);
                vv[7] = -__ddiv_rn(add(ksw, kse), six);
                vv[8] = -__ddiv_rn(mul(2.0, kse), six);
                const int64_t offs[9] = {-M - 1, -M, -M + 1, -1, 0, 1, M - 1, M, M + 1};
#pragma unroll
                for (int s = 0; s < 9; ++s) jj[s] = (int32_t)(r + offs[s]);
                if (symmetric) {
                    // drop couplings to boundary nodes, keep the slot order compact
                    int k = 0;
#pragma unroll
                    for (int s = 0; s < 9; ++s) {
                        const int64_t c = r + offs[s];
                        const int64_t ci = c / M, cj = c - ci * M;
                        const bool cb = ci == 0 || ci == M - 1 || cj == 0 || cj == M - 1;
                        const int32_t jv = jj[s];
                        const double av = vv[s];
                        jj[s] = -1;
                        vv[s] = 0.0;
                        if (!cb) { jj[k] = jv; vv[k] = av; ++k; }
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 9; ++s) {
            Aj[s * ld + r] = jj[s];
            Ax[s * ld + r] = vv[s];
        }
    }
}

// ---------------------------------------------------------------------------------------
// SpMV family, one kernel template per output mode:
//   SPMV    y = A x                                   (Product)
//   DEFECT  y = b - A x                               (Defect: temp = A x; r = b - temp)
//   ADD     y = y + A x                               (Prolongation<PROLMAT> + Sum: store = P c; x += store)
//   JACOBI  y = x + P * (b - A x)                     (one RISmoother sweep: t0 = b - A x; t1 = P t0; x += t1)
// Each rounds exactly as the reference's operator sequence does, so the results are
// bit-identical to tags::CPU.  x is read-only for the whole launch (gathered through L1).
// ---------------------------------------------------------------------------------------
template <typename T, int KT, int MODE>
__global__ void __launch_bounds__(SPMV_THREADS)
ell_spmv_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj,
                const T *__restrict__ Ax, const T *__restrict__ x, const T *__restrict__ b,
                const T *__restrict__ P, T *__restrict__ y, int vec_io)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r0 = g * 4;
    if (r0 >= rows) return;
    T sum[4];
    hbd::ell_rows4<T, KT>(Aj, Ax, ld, K, r0, [&](int32_t j) { return __ldg(x + j); }, sum);
    T out[4];
    if (vec_io && r0 + 3 < rows) {
        T bb[4], xx[4], pp[4], yy[4];
        if (MODE == HB_MODE_DEFECT || MODE == HB_MODE_JACOBI) hbd::ld4(b + r0, bb);
        if (MODE == HB_MODE_JACOBI) { hbd::ld4(x + r0, xx); hbd::ld4(P + r0, pp); }
        if (MODE == HB_MODE_ADD) hbd::ld4(y + r0, yy);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (MODE == HB_MODE_SPMV) out[i] = sum[i];
            if (MODE == HB_MODE_DEFECT) out[i] = sub(bb[i], sum[i]);
            if (MODE == HB_MODE_ADD) out[i] = add(yy[i], sum[i]);
            if (MODE == HB_MODE_JACOBI) out[i] = add(xx[i], mul(pp[i], sub(bb[i], sum[i])));
        }
        hbd::st4(y + r0, out);
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t r = r0 + i;
            if (r >= rows) break;
            T o = sum[i];
            if (MODE == HB_MODE_DEFECT) o = sub(b[r], sum[i]);
            if (MODE == HB_MODE_ADD) o = add(y[r], sum[i]);
            if (MODE == HB_MODE_JACOBI) o = add(x[r], mul(P[r], sub(b[r], sum[i])));
            y[r] = o;
        }
    }
}

// P[i] = damping / A(i, i), A(i, i) = the first slot of row i holding column i
// (SparseMatrixELL::operator(), honei/la/sparse_matrix_ell-impl.hh:326-338; PreconFill "jac",
// honei/math/mg.hh:255-286).
template <typename T>
__global__ void jacobi_diag_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj,
                                   const T *__restrict__ Ax, T damping, T *__restrict__ P)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows;
         r += (int64_t)gridDim.x * blockDim.x) {
        T d = T(0);
        for (int k = 0; k < K; ++k) {
            if (Aj[k * ld + r] == (int32_t)r) { d = Ax[k * ld + r]; break; }
        }
        P[r] = damping / d;
    }
}

}  // namespace

template <typename T>
int hb_launch_spmv_mode(hb_context *ctx, const hb_ell *A, int mode, const T *x, const T *b, const T *P, T *y)
{
    if (!ctx || !A) return HB_ERR_INVALID;
    if (A->rows == 0) return HB_OK;
    if (!x || !y) return HB_ERR_INVALID;
    if ((mode == HB_MODE_DEFECT || mode == HB_MODE_JACOBI) && !b) return HB_ERR_INVALID;
    if (mode == HB_MODE_JACOBI && !P) return HB_ERR_INVALID;
    const int64_t groups = (A->rows + 3) / 4;
    const int threads = ctx->block[HB_BLOCK_ELL] ? ctx->block[HB_BLOCK_ELL] : SPMV_THREADS;
    const int64_t blocks = (groups + threads - 1) / threads;
    const int vec = (((uintptr_t)y | (uintptr_t)b | (uintptr_t)P |
                      (mode == HB_MODE_JACOBI ? (uintptr_t)x : 0)) % 16) == 0;
    const int K = (int)A->K;
    const int32_t *Aj = A->Aj;
    const T *Ax = (const T *)A->Ax;
#define HB_SPMV_CASE(KC, MD)                                                                    \
    ell_spmv_kernel<T, KC, MD><<<(unsigned)blocks, threads, 0, ctx->stream>>>(                   \
        A->rows, A->ld, K, Aj, Ax, x, b, P, y, vec)
#define HB_SPMV_K(MD)                                                                           \
    switch (K) {                                                                                \
        case 4: HB_SPMV_CASE(4, MD); break;                                                     \
        case 9: HB_SPMV_CASE(9, MD); break;                                                     \
        default: HB_SPMV_CASE(0, MD); break;                                                    \
    }
    switch (mode) {
        case HB_MODE_SPMV: HB_SPMV_K(HB_MODE_SPMV); break;
        case HB_MODE_DEFECT: HB_SPMV_K(HB_MODE_DEFECT); break;
        case HB_MODE_ADD: HB_SPMV_K(HB_MODE_ADD); break;
        case HB_MODE_JACOBI: HB_SPMV_K(HB_MODE_JACOBI); break;
        default: return HB_ERR_INVALID;
    }
#undef HB_SPMV_K
#undef HB_SPMV_CASE
    return hb_check_launch(ctx, "ell_spmv_kernel");
}
template int hb_launch_spmv_mode<double>(hb_context *, const hb_ell *, int, const double *, const double *,
                                         const double *, double *);
template int hb_launch_spmv_mode<float>(hb_context *, const hb_ell *, int, const float *, const float *,
                                        const float *, float *);

template <typename T>
int hb_launch_jacobi_diag(hb_context *ctx, const hb_ell *A, T damping, T *P)
{
    if (A->rows == 0) return HB_OK;
    const unsigned blocks = (unsigned)std::min<int64_t>((A->rows + 255) / 256, (int64_t)ctx->num_sms * 16);
    jacobi_diag_kernel<T><<<blocks, 256, 0, ctx->stream>>>(A->rows, A->ld, (int)A->K, A->Aj, (const T *)A->Ax,
                                                           damping, P);
    return hb_check_launch(ctx, "jacobi_diag_kernel");
}
template int hb_launch_jacobi_diag<double>(hb_context *, const hb_ell *, double, double *);
template int hb_launch_jacobi_diag<float>(hb_context *, const hb_ell *, float, float *);

int hb_check_ell(const hb_ell *A, int dtype)
{
    if (!A || !A->Aj || !A->Ax) return HB_ERR_INVALID;
    if (A->dtype != dtype) return HB_ERR_INVALID;
    if (A->rows < 0 || A->cols < 0 || A->K < 1 || A->ld < A->rows || A->ld % 64) return HB_ERR_INVALID;
    if (A->rows > INT32_MAX || A->cols > INT32_MAX) return HB_ERR_UNSUPPORTED;
    if (((uintptr_t)A->Aj | (uintptr_t)A->Ax) % 16) return HB_ERR_INVALID;
    return HB_OK;
}

namespace {

// Counts the slots whose column is neither the padding mark (-1) nor inside [0, cols).
__global__ void ell_validate_kernel(int64_t total, int64_t cols, const int32_t *__restrict__ Aj,
                                    unsigned long long *bad)
{
    unsigned long long n = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t j = Aj[i];
        if (j < -1 || (int64_t)j >= cols) ++n;
    }
    if (n) atomicAdd(bad, n);
}

template <typename T>
int import_impl(hb_context *ctx, int64_t rows, int64_t cols, int64_t stride, int64_t ncpr,
                int64_t threads, const uint64_t *Aj_ref, const T *Ax_ref, const uint64_t *Arl,
                hb_ell *out, int dtype)
{
    if (!ctx || !out || threads < 1 || ncpr < 1) return HB_ERR_INVALID;
    if (rows > 0 && (!Aj_ref || !Ax_ref || !Arl)) return HB_ERR_INVALID;
    if (stride < rows * threads) return HB_ERR_SIZE;
    out->rows = rows;
    out->cols = cols;
    out->dtype = dtype;
    int64_t K, ld;
    hb_ell_layout(rows, ncpr, threads, &K, &ld);
    if (out->K != K || out->ld != ld) return HB_ERR_SIZE;
    int st = hb_check_ell(out, dtype);
    if (st) return st;
    int *bad = (int *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
    const int64_t total = K * ld;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32);
    ell_import_kernel<T><<<blocks, 256, 0, ctx->stream>>>(rows, cols, stride, threads, K, ld, Aj_ref,
                                                          Ax_ref, Arl, out->Aj, (T *)out->Ax, bad);
    st = hb_check_launch(ctx, "ell_import_kernel");
    if (st) return st;
    int *h = (int *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return *h ? HB_ERR_INVALID : HB_OK;
}

}  // namespace

template <typename T>
static int jacobi_sweeps(hb_context *ctx, const hb_ell *A, int dtype, const T *P, const T *b, T *x, T *tmp,
                         int64_t sweeps)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = hb_check_ell(A, dtype);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    if (sweeps < 0) return HB_ERR_INVALID;
    if (sweeps == 0 || A->rows == 0) return HB_OK;
    if (!P || !b || !x || !tmp || tmp == x) return HB_ERR_INVALID;
    // x' = x + P (b - A x) reads every x it gathers while it writes: ping-pong through tmp
    T *cur = x, *other = tmp;
    for (int64_t k = 0; k < sweeps; ++k) {
        st = hb_launch_spmv_mode<T>(ctx, A, HB_MODE_JACOBI, cur, b, P, other);
        if (st) return st;
        T *t = cur; cur = other; other = t;
    }
    if (cur != x)
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(x, cur, sizeof(T) * A->rows, cudaMemcpyDeviceToDevice, ctx->stream));
    return HB_OK;
}

extern "C" {

int hb_ell_validate(hb_context *ctx, const hb_ell *A, int64_t *bad_slots)
{
    HB_RANGE("hb_ell_validate");
    if (!ctx || !bad_slots || !A || !A->Aj) return HB_ERR_INVALID;
    if (A->rows < 0 || A->cols < 0 || A->K < 1 || A->ld < A->rows) return HB_ERR_INVALID;
    unsigned long long *bad = (unsigned long long *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(*bad), ctx->stream));
    const int64_t total = A->K * A->ld;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32));
    ell_validate_kernel<<<blocks, 256, 0, ctx->stream>>>(total, A->cols, A->Aj, bad);
    int st = hb_check_launch(ctx, "ell_validate_kernel");
    if (st) return st;
    unsigned long long *h = (unsigned long long *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, bad, sizeof(*h), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *bad_slots = (int64_t)*h;
    return HB_OK;
}

int hb_ell_layout(int64_t rows, int64_t ncpr, int64_t threads, int64_t *K, int64_t *ld)
{
    if (!K || !ld || rows < 0 || ncpr < 1 || threads < 1) return HB_ERR_INVALID;
    *K = ncpr * threads;
    *ld = hb_round_up(rows > 0 ? rows : 1, 64);
    return HB_OK;
}

int hb_ell_import_f64(hb_context *ctx, int64_t rows, int64_t cols, int64_t stride, int64_t ncpr,
                      int64_t threads, const uint64_t *Aj_ref, const double *Ax_ref,
                      const uint64_t *Arl_ref, hb_ell *out)
{
    HB_RANGE("hb_ell_import_f64");
    return import_impl<double>(ctx, rows, cols, stride, ncpr, threads, Aj_ref, Ax_ref, Arl_ref, out, HB_F64);
}

int hb_ell_import_f32(hb_context *ctx, int64_t rows, int64_t cols, int64_t stride, int64_t ncpr,
                      int64_t threads, const uint64_t *Aj_ref, const float *Ax_ref,
                      const uint64_t *Arl_ref, hb_ell *out)
{
    HB_RANGE("hb_ell_import_f32");
    return import_impl<float>(ctx, rows, cols, stride, ncpr, threads, Aj_ref, Ax_ref, Arl_ref, out, HB_F32);
}

int hb_ell_cast_f64_f32(hb_context *ctx, const hb_ell *src, hb_ell *dst)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = hb_check_ell(src, HB_F64);
    if (st) return st;
    if (!dst || dst->K != src->K || dst->ld != src->ld) return HB_ERR_SIZE;
    dst->rows = src->rows;
    dst->cols = src->cols;
    dst->dtype = HB_F32;
    st = hb_check_ell(dst, HB_F32);
    if (st) return st;
    const int64_t total = src->K * src->ld;
    if (dst->Aj != src->Aj)   // the FP32 copy may share the index array
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(dst->Aj, src->Aj, total * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                         ctx->stream));
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32);
    ell_cast_kernel<<<blocks, 256, 0, ctx->stream>>>(total, (const double *)src->Ax, (float *)dst->Ax);
    return hb_check_launch(ctx, "ell_cast_kernel");
}

int hb_q1_assemble_f64(hb_context *ctx, int64_t M, const double *coef, int symmetric, hb_ell *out)
{
    if (!ctx || !out || M < 1) return HB_ERR_INVALID;
    const int64_t N = M * M;
    int64_t K, ld;
    hb_ell_layout(N, 9, 1, &K, &ld);
    if (out->K != K || out->ld != ld) return HB_ERR_SIZE;
    out->rows = N;
    out->cols = N;
    out->dtype = HB_F64;
    int st = hb_check_ell(out, HB_F64);
    if (st) return st;
    const unsigned blocks = (unsigned)std::min<int64_t>((ld + 255) / 256, (int64_t)ctx->num_sms * 32);
    q1_assemble_kernel<<<blocks, 256, 0, ctx->stream>>>(M, coef, ld, symmetric, out->Aj, (double *)out->Ax);
    return hb_check_launch(ctx, "q1_assemble_kernel");
}

int hb_spmv_f64(hb_context *ctx, const hb_ell *A, const double *x, double *y)
{
    HB_RANGE("hb_spmv_f64");
    int st = hb_check_ell(A, HB_F64);
    if (st) return st;
    return hb_launch_spmv_mode<double>(ctx, A, HB_MODE_SPMV, x, nullptr, nullptr, y);
}

int hb_spmv_f32(hb_context *ctx, const hb_ell *A, const float *x, float *y)
{
    HB_RANGE("hb_spmv_f32");
    int st = hb_check_ell(A, HB_F32);
    if (st) return st;
    return hb_launch_spmv_mode<float>(ctx, A, HB_MODE_SPMV, x, nullptr, nullptr, y);
}

int hb_jacobi_sweeps_f64(hb_context *ctx, const hb_ell *A, const double *P, const double *b, double *x, double *tmp,
                         int64_t sweeps)
{
    HB_RANGE("hb_jacobi_sweeps_f64");
    return jacobi_sweeps<double>(ctx, A, HB_F64, P, b, x, tmp, sweeps);
}

int hb_jacobi_sweeps_f32(hb_context *ctx, const hb_ell *A, const float *P, const float *b, float *x, float *tmp,
                         int64_t sweeps)
{
    HB_RANGE("hb_jacobi_sweeps_f32");
    return jacobi_sweeps<float>(ctx, A, HB_F32, P, b, x, tmp, sweeps);
}

int hb_defect_f64(hb_context *ctx, const hb_ell *A, const double *b, const double *x, double *r)
{
    HB_RANGE("hb_defect_f64");
    int st = hb_check_ell(A, HB_F64);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    return hb_launch_spmv_mode<double>(ctx, A, HB_MODE_DEFECT, x, b, nullptr, r);
}

int hb_defect_f32(hb_context *ctx, const hb_ell *A, const float *b, const float *x, float *r)
{
    HB_RANGE("hb_defect_f32");
    int st = hb_check_ell(A, HB_F32);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    return hb_launch_spmv_mode<float>(ctx, A, HB_MODE_DEFECT, x, b, nullptr, r);
}

}  // extern "C"
