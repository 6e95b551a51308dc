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
#include "hb_internal.cuh"

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
__global__ void q1_assemble_kernel(int64_t M, const double *__restrict__ coef, int64_t ld,
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
// SpMV / defect.  KT > 0: K known at compile time (all slot loads issued up front);
// KT == 0: runtime K in chunks of 4 slots.
// ---------------------------------------------------------------------------------------
template <typename T, int KT, bool DEFECT>
__global__ void __launch_bounds__(SPMV_THREADS)
ell_spmv_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj,
                const T *__restrict__ Ax, const T *__restrict__ x, const T *__restrict__ b,
                T *__restrict__ y, int vec_io)
{
    using hbd::add; using hbd::mul;
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r0 = g * 4;
    if (r0 >= rows) return;
    T sum[4] = {T(0), T(0), T(0), T(0)};
    if (KT > 0) {
        int32_t j[KT > 0 ? KT : 1][4];
        T a[KT > 0 ? KT : 1][4];
#pragma unroll
        for (int k = 0; k < KT; ++k) {
            hbd::ld4_stream(Aj + k * ld + r0, j[k]);
            hbd::ld4_stream(Ax + k * ld + r0, a[k]);
        }
#pragma unroll
        for (int k = 0; k < KT; ++k)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (j[k][i] >= 0) sum[i] = add(sum[i], mul(a[k][i], __ldg(x + j[k][i])));
    } else {
        for (int k0 = 0; k0 < K; k0 += 4) {
            int32_t j[4][4];
            T a[4][4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (k0 + c < K) {
                    hbd::ld4_stream(Aj + (k0 + c) * ld + r0, j[c]);
                    hbd::ld4_stream(Ax + (k0 + c) * ld + r0, a[c]);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i) { j[c][i] = -1; a[c][i] = T(0); }
                }
            }
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (j[c][i] >= 0) sum[i] = add(sum[i], mul(a[c][i], __ldg(x + j[c][i])));
        }
    }
    if (vec_io && r0 + 3 < rows) {
        if (DEFECT) {
            T bb[4];
            hbd::ld4(b + r0, bb);
#pragma unroll
            for (int i = 0; i < 4; ++i) sum[i] = hbd::sub(bb[i], sum[i]);
        }
        hbd::st4(y + r0, sum);
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (r0 + i < rows) y[r0 + i] = DEFECT ? hbd::sub(b[r0 + i], sum[i]) : sum[i];
    }
}

template <typename T, bool DEFECT>
int launch_spmv(hb_context *ctx, const hb_ell *A, const T *x, const T *b, T *y)
{
    if (!ctx || !A) return HB_ERR_INVALID;
    if (A->rows == 0) return HB_OK;
    if (!x || !y || (DEFECT && !b)) return HB_ERR_INVALID;
    const int64_t groups = (A->rows + 3) / 4;
    const int64_t blocks = (groups + SPMV_THREADS - 1) / SPMV_THREADS;
    const int vec = (((uintptr_t)y | (DEFECT ? (uintptr_t)b : 0)) % 16) == 0;
    const int K = (int)A->K;
    const int32_t *Aj = A->Aj;
    const T *Ax = (const T *)A->Ax;
#define HB_SPMV_CASE(KC)                                                                       \
    ell_spmv_kernel<T, KC, DEFECT><<<(unsigned)blocks, SPMV_THREADS, 0, ctx->stream>>>(         \
        A->rows, A->ld, K, Aj, Ax, x, b, y, vec)
    switch (K) {
        case 1: HB_SPMV_CASE(1); break;
        case 4: HB_SPMV_CASE(4); break;
        case 9: HB_SPMV_CASE(9); break;
        default: HB_SPMV_CASE(0); break;
    }
#undef HB_SPMV_CASE
    return hb_check_launch(ctx, DEFECT ? "ell_defect_kernel" : "ell_spmv_kernel");
}

int check_ell(const hb_ell *A, int dtype)
{
    if (!A || !A->Aj || !A->Ax) return HB_ERR_INVALID;
    if (A->dtype != dtype) return HB_ERR_INVALID;
    if (A->rows < 0 || A->cols < 0 || A->K < 1 || A->ld < A->rows || A->ld % 64) return HB_ERR_INVALID;
    if (A->rows > INT32_MAX || A->cols > INT32_MAX) return HB_ERR_UNSUPPORTED;
    if (((uintptr_t)A->Aj | (uintptr_t)A->Ax) % 16) return HB_ERR_INVALID;
    return HB_OK;
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
    int st = check_ell(out, dtype);
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

extern "C" {

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
    return import_impl<double>(ctx, rows, cols, stride, ncpr, threads, Aj_ref, Ax_ref, Arl_ref, out, HB_F64);
}

int hb_ell_import_f32(hb_context *ctx, int64_t rows, int64_t cols, int64_t stride, int64_t ncpr,
                      int64_t threads, const uint64_t *Aj_ref, const float *Ax_ref,
                      const uint64_t *Arl_ref, hb_ell *out)
{
    return import_impl<float>(ctx, rows, cols, stride, ncpr, threads, Aj_ref, Ax_ref, Arl_ref, out, HB_F32);
}

int hb_ell_cast_f64_f32(hb_context *ctx, const hb_ell *src, hb_ell *dst)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = check_ell(src, HB_F64);
    if (st) return st;
    if (!dst || dst->K != src->K || dst->ld != src->ld) return HB_ERR_SIZE;
    dst->rows = src->rows;
    dst->cols = src->cols;
    dst->dtype = HB_F32;
    st = check_ell(dst, HB_F32);
    if (st) return st;
    const int64_t total = src->K * src->ld;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(dst->Aj, src->Aj, total * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                     ctx->stream));
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32);
    ell_cast_kernel<<<blocks, 256, 0, ctx->stream>>>(total, (const double *)src->Ax, (float *)dst->Ax);
    return hb_check_launch(ctx, "ell_cast_kernel");
}

int hb_q1_assemble_f64(hb_context *ctx, int64_t M, const double *coef, hb_ell *out)
{
    if (!ctx || !out || M < 1) return HB_ERR_INVALID;
    const int64_t N = M * M;
    int64_t K, ld;
    hb_ell_layout(N, 9, 1, &K, &ld);
    if (out->K != K || out->ld != ld) return HB_ERR_SIZE;
    out->rows = N;
    out->cols = N;
    out->dtype = HB_F64;
    int st = check_ell(out, HB_F64);
    if (st) return st;
    const unsigned blocks = (unsigned)std::min<int64_t>((ld + 255) / 256, (int64_t)ctx->num_sms * 32);
    q1_assemble_kernel<<<blocks, 256, 0, ctx->stream>>>(M, coef, ld, out->Aj, (double *)out->Ax);
    return hb_check_launch(ctx, "q1_assemble_kernel");
}

int hb_spmv_f64(hb_context *ctx, const hb_ell *A, const double *x, double *y)
{
    int st = check_ell(A, HB_F64);
    if (st) return st;
    return launch_spmv<double, false>(ctx, A, x, nullptr, y);
}

int hb_spmv_f32(hb_context *ctx, const hb_ell *A, const float *x, float *y)
{
    int st = check_ell(A, HB_F32);
    if (st) return st;
    return launch_spmv<float, false>(ctx, A, x, nullptr, y);
}

int hb_defect_f64(hb_context *ctx, const hb_ell *A, const double *b, const double *x, double *r)
{
    int st = check_ell(A, HB_F64);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    return launch_spmv<double, true>(ctx, A, x, b, r);
}

int hb_defect_f32(hb_context *ctx, const hb_ell *A, const float *b, const float *x, float *r)
{
    int st = check_ell(A, HB_F32);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    return launch_spmv<float, true>(ctx, A, x, b, r);
}

}  // extern "C"
