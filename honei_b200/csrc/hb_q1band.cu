// hb_q1band.cu -- Product and Defect on BandedMatrixQx<Q1Type> (the nine-band Q1 matrix of a
// square grid), its Poisson fill and its conversion from ELL.
//
// Reference: Product<tags::CPU>::value(result, BandedMatrixQx<Q1Type>, x)
// (honei/la/product.hh:371-404): y[i] = DD[i] x[i], then += LL, LD, LU, DL, DU, UL, UD, UU
// times x at column i - root - 1, i - root, i - root + 1, i - 1, i + 1, i + root - 1, i + root,
// i + root + 1, each term only where its column lies in [0, n) (a bound on the linear index,
// not on the grid line); root = floor(sqrt(n)).  Defect<tags::CPU> (honei/math/defect.hh:
// 194-199) is that product followed by Difference: r = b - y.
//
// Per row the kernel reads the nine band values once (16-byte streaming loads when every band
// is 16-byte aligned) and three windows of x (L1/L2-resident), with no column index array: 11
// values of traffic per row against 9 values + 9 indices + 2 values for the ELL product of the
// same matrix.  Every sum rounds in the reference's order (no FMA contraction).
#include "hb_internal.cuh"

#include <cmath>

namespace {

template <typename T> struct Bands {
    const T *p[9];
};

__host__ __device__ __forceinline__ int64_t q1band_root(int64_t n)
{
    int64_t r = (int64_t)sqrt((double)n);
    while (r > 0 && r * r > n) --r;
    while ((r + 1) * (r + 1) <= n) ++r;
    return r;
}

// R consecutive rows per thread, R = 16 / sizeof(T): each band is one 16-byte load.
template <typename T> struct Rows;
template <> struct Rows<double> { static constexpr int R = 2; };
template <> struct Rows<float> { static constexpr int R = 4; };

template <typename T, int R> __device__ __forceinline__ void ld_vec(const T *p, T (&v)[R]);
template <> __device__ __forceinline__ void ld_vec<double, 2>(const double *p, double (&v)[2])
{
    const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
    v[0] = t.x; v[1] = t.y;
}
template <> __device__ __forceinline__ void ld_vec<float, 4>(const float *p, float (&v)[4])
{
    const float4 t = __ldcs(reinterpret_cast<const float4 *>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
template <typename T, int R> __device__ __forceinline__ void st_vec(T *p, const T (&v)[R]);
template <> __device__ __forceinline__ void st_vec<double, 2>(double *p, const double (&v)[2])
{
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
}
template <> __device__ __forceinline__ void st_vec<float, 4>(float *p, const float (&v)[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// MODE 0: y = A x;  MODE 1: y = b - A x;  MODE 2: y = x + P (b - A x) (damped Jacobi sweep).
// VEC: every band, b, P and y 16-byte aligned.  ELL: sum the bands in ascending column order
// (LL, LD, LU, DL, DD, DU, UL, UD, UU: the order of the same matrix's ELL row) instead of the
// reference's banded order (DD first).
template <typename T, int MODE, bool VEC, bool ELL = false>
__global__ void __launch_bounds__(256) q1band_kernel(int64_t n, int64_t root, Bands<T> B, const T *__restrict__ x,
                                                     const T *__restrict__ b, T *__restrict__ y,
                                                     const T *__restrict__ P = nullptr)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    constexpr int R = Rows<T>::R;
    const int64_t groups = (n + R - 1) / R;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < groups;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r0 = R * g;
        const bool full = r0 + R <= n;
        T a[9][R];
        if (VEC && full) {
#pragma unroll
            for (int k = 0; k < 9; ++k) ld_vec<T, R>(B.p[k] + r0, a[k]);
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k)
#pragma unroll
                for (int i = 0; i < R; ++i) a[k][i] = (r0 + i < n) ? __ldcs(B.p[k] + r0 + i) : T(0);
        }
        // x windows around the three band groups: lo[t] = x[r0 - root - 1 + t],
        // mid[t] = x[r0 - 1 + t], hi[t] = x[r0 + root - 1 + t]
        T lo[R + 2], mid[R + 2], hi[R + 2];
#pragma unroll
        for (int t = 0; t < R + 2; ++t) {
            const int64_t jl = r0 - root - 1 + t, jm = r0 - 1 + t, jh = r0 + root - 1 + t;
            lo[t] = (jl >= 0 && jl < n) ? __ldg(x + jl) : T(0);
            mid[t] = (jm >= 0 && jm < n) ? __ldg(x + jm) : T(0);
            hi[t] = (jh >= 0 && jh < n) ? __ldg(x + jh) : T(0);
        }
        T out[R];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int64_t r = r0 + i;
            T s;
            if (ELL) {
                s = T(0);
                if (r - root - 1 >= 0) s = add(s, mul(a[0][i], lo[i]));
                if (r - root >= 0) s = add(s, mul(a[1][i], lo[i + 1]));
                if (r - root + 1 >= 0) s = add(s, mul(a[2][i], lo[i + 2]));
                if (r - 1 >= 0) s = add(s, mul(a[3][i], mid[i]));
                s = add(s, mul(a[4][i], mid[i + 1]));
            } else {
                s = mul(a[4][i], mid[i + 1]);
                if (r - root - 1 >= 0) s = add(s, mul(a[0][i], lo[i]));
                if (r - root >= 0) s = add(s, mul(a[1][i], lo[i + 1]));
                if (r - root + 1 >= 0) s = add(s, mul(a[2][i], lo[i + 2]));
                if (r - 1 >= 0) s = add(s, mul(a[3][i], mid[i]));
            }
            if (r + 1 < n) s = add(s, mul(a[5][i], mid[i + 2]));
            if (r + root - 1 < n) s = add(s, mul(a[6][i], hi[i]));
            if (r + root < n) s = add(s, mul(a[7][i], hi[i + 1]));
            if (r + root + 1 < n) s = add(s, mul(a[8][i], hi[i + 2]));
            out[i] = s;
        }
        if (MODE >= 1) {
            T bv[R];
            if (VEC && full) {
                ld_vec<T, R>(b + r0, bv);
            } else {
#pragma unroll
                for (int i = 0; i < R; ++i) bv[i] = (r0 + i < n) ? __ldcs(b + r0 + i) : T(0);
            }
            if (MODE == 1) {
#pragma unroll
                for (int i = 0; i < R; ++i) out[i] = sub(bv[i], out[i]);
            } else {
                // x + P (b - s); the own x values are mid[1..R]
                T pv[R];
                if (VEC && full) {
                    ld_vec<T, R>(P + r0, pv);
                } else {
#pragma unroll
                    for (int i = 0; i < R; ++i) pv[i] = (r0 + i < n) ? __ldcs(P + r0 + i) : T(0);
                }
#pragma unroll
                for (int i = 0; i < R; ++i) out[i] = add(mid[i + 1], mul(pv[i], sub(bv[i], out[i])));
            }
        }
        if (VEC && full) {
            st_vec<T, R>(y + r0, out);
        } else {
#pragma unroll
            for (int i = 0; i < R; ++i)
                if (r0 + i < n) y[r0 + i] = out[i];
        }
    }
}

// FillMatrix<Tag, POISSON, DIRICHLET_0> on BandedMatrixQx (honei/math/fill_matrix.hh:41-77):
// 1-based row i is a unit row when i <= M, i > N - M, i % M == 1 or i % M == 0; otherwise 8/3
// on the diagonal and -1/3 on all eight off-diagonal bands (double constants rounded to T).
template <typename T>
__global__ void q1band_poisson_kernel(int64_t N, int64_t M, Bands<T> B)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = r + 1;
        const bool unit = i <= M || i > N - M || (i % M) == 1 || (i % M) == 0;
#pragma unroll
        for (int k = 0; k < 9; ++k) const_cast<T *>(B.p[k])[r] = unit ? T(0.0) : (T)(-1.0 / 3.0);
        const_cast<T *>(B.p[4])[r] = unit ? T(1.0) : (T)(8.0 / 3.0);
    }
}

// BandedMatrixQx(SparseMatrixELL &) (honei/la/banded_matrix_qx-impl.hh:111-167): band k of
// row r holds A(r, r + offset_k) where that column exists; entries the conversion never sets
// are 0 here.
template <typename T>
__global__ void q1band_from_ell_kernel(int64_t n, int64_t root, int64_t ld, int K, const int32_t *__restrict__ Aj,
                                       const T *__restrict__ Ax, Bands<T> B, int *off_band)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t off[9] = {-root - 1, -root, -root + 1, -1, 0, 1, root - 1, root, root + 1};
        T v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = T(0);
        for (int s = 0; s < K; ++s) {
            const int32_t j = Aj[(int64_t)s * ld + r];
            if (j < 0) continue;
            const int64_t d = (int64_t)j - r;
            bool hit = false;
#pragma unroll
            for (int k = 0; k < 9; ++k)
                if (d == off[k]) { v[k] = Ax[(int64_t)s * ld + r]; hit = true; }
            if (!hit && Ax[(int64_t)s * ld + r] != T(0)) atomicExch(off_band, 1);   // not a Q1 band
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) const_cast<T *>(B.p[k])[r] = v[k];
    }
}

template <typename T> Bands<T> bands_of(const hb_q1band *A)
{
    Bands<T> B;
    for (int k = 0; k < 9; ++k) B.p[k] = (const T *)A->band[k];
    return B;
}

int check_q1band(const hb_q1band *A, int dtype)
{
    if (!A || A->n < 0 || A->dtype != dtype) return HB_ERR_INVALID;
    if (A->n == 0) return HB_OK;
    for (int k = 0; k < 9; ++k)
        if (!A->band[k]) return HB_ERR_INVALID;
    if (A->root != q1band_root(A->n)) return HB_ERR_INVALID;
    return HB_OK;
}

inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// threads per block of the banded kernels on this context (hb_set_block_size), and their grid
int band_threads(hb_context *ctx) { return ctx->block[HB_BLOCK_Q1BAND] ? ctx->block[HB_BLOCK_Q1BAND] : 256; }

int grid_for(hb_context *ctx, int64_t work)
{
    const int th = band_threads(ctx);
    const int64_t blocks = (work + th - 1) / th;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)ctx->num_sms * 64 * (256 / th)));
}

template <typename T>
int q1band_apply(hb_context *ctx, const hb_q1band *A, const T *b, const T *x, T *y, int mode, int dtype)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = check_q1band(A, dtype);
    if (st) return st;
    const int64_t n = A->n;
    if (n == 0) return HB_OK;
    if (!x || !y || (mode == 1 && !b)) return HB_ERR_INVALID;
    bool vec = aligned16(y) && (mode == 0 || aligned16(b));
    for (int k = 0; k < 9; ++k) vec = vec && aligned16(A->band[k]);
    const Bands<T> B = bands_of<T>(A);
    const int grid = grid_for(ctx, (n + Rows<T>::R - 1) / Rows<T>::R);
    if (mode == 0) {
        if (vec) q1band_kernel<T, 0, true><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, B, x, b, y);
        else q1band_kernel<T, 0, false><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, B, x, b, y);
    } else {
        if (vec) q1band_kernel<T, 1, true><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, B, x, b, y);
        else q1band_kernel<T, 1, false><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, B, x, b, y);
    }
    return hb_check_launch(ctx, "q1band_kernel");
}

}  // namespace

template <typename T>
int hb_launch_band_mode(hb_context *ctx, const hb_q1band *A, int mode, const T *x, const T *b, const T *P, T *y)
{
    const int64_t n = A->n;
    if (n == 0) return HB_OK;
    bool vec = aligned16(y) && (mode == HB_MODE_SPMV || aligned16(b)) && (mode != HB_MODE_JACOBI || aligned16(P));
    for (int k = 0; k < 9; ++k) vec = vec && aligned16(A->band[k]);
    const Bands<T> B = bands_of<T>(A);
    const int grid = grid_for(ctx, (n + Rows<T>::R - 1) / Rows<T>::R);
#define HB_BAND_LAUNCH(MD)                                                                                     \
    if (vec) q1band_kernel<T, MD, true, true><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, B, x, b, y, P);       \
    else q1band_kernel<T, MD, false, true><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, B, x, b, y, P)
    switch (mode) {
        case HB_MODE_SPMV: HB_BAND_LAUNCH(0); break;
        case HB_MODE_DEFECT: HB_BAND_LAUNCH(1); break;
        case HB_MODE_JACOBI: HB_BAND_LAUNCH(2); break;
        default: return HB_ERR_INVALID;
    }
#undef HB_BAND_LAUNCH
    return hb_check_launch(ctx, "q1band_kernel (ELL order)");
}
template int hb_launch_band_mode<double>(hb_context *, const hb_q1band *, int, const double *, const double *,
                                         const double *, double *);
template int hb_launch_band_mode<float>(hb_context *, const hb_q1band *, int, const float *, const float *,
                                        const float *, float *);

extern "C" {

int64_t hb_q1band_root(int64_t n) { return n > 0 ? q1band_root(n) : 0; }

int hb_q1band_spmv_f64(hb_context *ctx, const hb_q1band *A, const double *x, double *y)
{
    HB_RANGE("hb_q1band_spmv_f64");
    return q1band_apply<double>(ctx, A, nullptr, x, y, 0, HB_F64);
}

int hb_q1band_spmv_f32(hb_context *ctx, const hb_q1band *A, const float *x, float *y)
{
    HB_RANGE("hb_q1band_spmv_f32");
    return q1band_apply<float>(ctx, A, nullptr, x, y, 0, HB_F32);
}

int hb_q1band_defect_f64(hb_context *ctx, const hb_q1band *A, const double *b, const double *x, double *r)
{
    HB_RANGE("hb_q1band_defect_f64");
    return q1band_apply<double>(ctx, A, b, x, r, 1, HB_F64);
}

int hb_q1band_defect_f32(hb_context *ctx, const hb_q1band *A, const float *b, const float *x, float *r)
{
    HB_RANGE("hb_q1band_defect_f32");
    return q1band_apply<float>(ctx, A, b, x, r, 1, HB_F32);
}

int hb_q1band_fill_poisson(hb_context *ctx, int64_t M, hb_q1band *A)
{
    if (!ctx || !A || M < 0 || A->n != M * M) return HB_ERR_INVALID;
    if (A->dtype != HB_F64 && A->dtype != HB_F32) return HB_ERR_INVALID;
    A->root = M;
    if (A->n == 0) return HB_OK;
    for (int k = 0; k < 9; ++k)
        if (!A->band[k]) return HB_ERR_INVALID;
    const int grid = grid_for(ctx, A->n);
    if (A->dtype == HB_F64)
        q1band_poisson_kernel<double><<<grid, band_threads(ctx), 0, ctx->stream>>>(A->n, M, bands_of<double>(A));
    else
        q1band_poisson_kernel<float><<<grid, band_threads(ctx), 0, ctx->stream>>>(A->n, M, bands_of<float>(A));
    return hb_check_launch(ctx, "q1band_poisson_kernel");
}

int hb_q1band_from_ell(hb_context *ctx, const hb_ell *E, hb_q1band *A)
{
    if (!ctx || !E || !A || E->rows != E->cols || A->n != E->rows || A->dtype != E->dtype) return HB_ERR_INVALID;
    const int64_t n = E->rows;
    A->root = n > 0 ? q1band_root(n) : 0;
    if (n == 0) return HB_OK;
    if (A->root * A->root != n) return HB_ERR_UNSUPPORTED;
    for (int k = 0; k < 9; ++k)
        if (!A->band[k]) return HB_ERR_INVALID;
    if (!E->Aj || !E->Ax) return HB_ERR_INVALID;
    const int grid = grid_for(ctx, n);
    int *flag = (int *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
    if (A->dtype == HB_F64)
        q1band_from_ell_kernel<double><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, E->ld, (int)E->K, E->Aj,
                                                                      (const double *)E->Ax, bands_of<double>(A), flag);
    else
        q1band_from_ell_kernel<float><<<grid, band_threads(ctx), 0, ctx->stream>>>(n, A->root, E->ld, (int)E->K, E->Aj,
                                                                     (const float *)E->Ax, bands_of<float>(A), flag);
    int st = hb_check_launch(ctx, "q1band_from_ell_kernel");
    if (st) return st;
    int *h = (int *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return *h ? HB_ERR_UNSUPPORTED : HB_OK;
}

}  // extern "C"
