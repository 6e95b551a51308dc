// hb_blas1.cu -- dot / norm reductions and the elementwise vector operators.
//
// Reductions: one launch, grid size a function of n only; each block reduces its contiguous
// slice in a fixed order (per-thread strided sums, then a warp/block shuffle tree), writes one
// partial, and the last block to finish (atomic ticket) sums the partials in a fixed tree and
// resets the ticket.  Results are deterministic run to run.  The reference instead copies
// grid*block partials to the host and sums them there, with a cudaMalloc/cudaFree per call
// (honei/backends/cuda/dot_product.cu:77-155, honei/backends/cuda/norm.cu:77-155).
//
// Elementwise operators are single-rounding per element and therefore bit-identical to the
// tags::CPU loops they replace (honei/la/scaled_sum.hh:73-110, scale.hh:77, sum.hh:98,
// element_product.hh:76-140).
#include "hb_internal.cuh"

#include <cmath>

namespace {

constexpr int RED_THREADS = 512;

inline int red_blocks(hb_context *ctx, int64_t n)
{
    // ~8 elements per thread minimum, at most 2 blocks per SM: fixed for a given n.
    int64_t b = (n + RED_THREADS * 8 - 1) / (RED_THREADS * 8);
    b = std::max<int64_t>(1, std::min<int64_t>(b, 2 * (int64_t)ctx->num_sms));
    return (int)b;
}

template <typename T, bool SQUARE>
__global__ void __launch_bounds__(RED_THREADS)
dot_kernel(int64_t n, const T *__restrict__ x, const T *__restrict__ y, double *partials,
           unsigned *ticket, T *out)
{
    using hbd::add; using hbd::mul;
    __shared__ T smem[32];
    __shared__ int s_last;
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = blockIdx.x * per, hi = min(n, lo + per);
    T acc = T(0);
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
        acc = add(acc, SQUARE ? mul(x[i], x[i]) : mul(x[i], y[i]));
    acc = hbd::block_sum(acc, smem);
    T *tp = reinterpret_cast<T *>(partials);
    if (threadIdx.x == 0) {
        tp[blockIdx.x] = acc;
        __threadfence();
        s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    T v = T(0);
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
        v = add(v, ((volatile T *)tp)[i]);
    v = hbd::block_sum(v, smem);
    if (threadIdx.x == 0) {
        *out = v;
        *ticket = 0;
    }
}

template <typename T, bool SQUARE>
int dot_launch(hb_context *ctx, int64_t n, const T *x, const T *y, T *out)
{
    const int blocks = red_blocks(ctx, n);
    unsigned *ticket = hb_bar(ctx) + 8;
    dot_kernel<T, SQUARE><<<blocks, RED_THREADS, 0, ctx->stream>>>(n, x, y, hb_partials(ctx), ticket, out);
    return hb_check_launch(ctx, "dot_kernel");
}

template <typename T, bool SQUARE>
int dot_impl(hb_context *ctx, int64_t n, const T *x, const T *y, T *result_host)
{
    if (!ctx || !result_host || n < 0) return HB_ERR_INVALID;
    if (n == 0) { *result_host = T(0); return HB_OK; }
    if (!x || (!SQUARE && !y)) return HB_ERR_INVALID;
    T *out = reinterpret_cast<T *>(hb_scalars(ctx) + 8);
    int st = dot_launch<T, SQUARE>(ctx, n, x, y, out);
    if (st) return st;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, out, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *result_host = *reinterpret_cast<T *>(ctx->pinned);
    return HB_OK;
}

// ---------------------------------------------------------------------------------------
// Elementwise operators
// ---------------------------------------------------------------------------------------
enum Op { OP_AXPY, OP_AXPY3, OP_SCALE, OP_SUM, OP_DIFF, OP_EPROD, OP_FILL };

template <typename T, int OP>
__device__ __forceinline__ T apply(T xv, T yv, T a)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    switch (OP) {
        case OP_AXPY: return add(xv, mul(a, yv));    // x += b*y
        case OP_AXPY3: return add(mul(a, yv), xv);   // r = b*y + x
        case OP_SCALE: return mul(xv, a);            // x *= a
        case OP_SUM: return add(xv, yv);             // x += y
        case OP_DIFF: return sub(xv, yv);            // r = x - y
        case OP_EPROD: return mul(xv, yv);           // r = x * y
        default: return a;                           // fill
    }
}

template <typename T, int OP>
__global__ void ew_kernel(int64_t n, T *__restrict__ r, const T *__restrict__ x, const T *__restrict__ y, T a)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T xv = (OP == OP_FILL) ? T(0) : x[i];
        const T yv = (OP == OP_AXPY || OP == OP_AXPY3 || OP == OP_SUM || OP == OP_DIFF || OP == OP_EPROD) ? y[i] : T(0);
        r[i] = apply<T, OP>(xv, yv, a);
    }
}

template <typename T, int OP>
int ew_launch(hb_context *ctx, int64_t n, T *r, const T *x, const T *y, T a)
{
    if (!ctx || n < 0 || !r) return HB_ERR_INVALID;
    if (n == 0) return HB_OK;
    const int th = ctx->block[HB_BLOCK_VECTOR] ? ctx->block[HB_BLOCK_VECTOR] : 256;
    const int64_t blocks = std::min<int64_t>((n + th - 1) / th, (int64_t)ctx->num_sms * 16 * (256 / th > 0 ? 256 / th : 1));
    ew_kernel<T, OP><<<(unsigned)blocks, th, 0, ctx->stream>>>(n, r, x, y, a);
    return hb_check_launch(ctx, "ew_kernel");
}

template <typename S, typename D>
__global__ void convert_kernel(int64_t n, D *__restrict__ dst, const S *__restrict__ src)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (D)src[i];
}

template <typename S, typename D>
int convert_impl(hb_context *ctx, int64_t n, D *dst, const S *src)
{
    if (!ctx || n < 0 || !dst || !src) return HB_ERR_INVALID;
    if (n == 0) return HB_OK;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 16);
    convert_kernel<S, D><<<(unsigned)blocks, 256, 0, ctx->stream>>>(n, dst, src);
    return hb_check_launch(ctx, "convert_kernel");
}

}  // namespace

template <typename T> int hb_launch_dot(hb_context *ctx, int64_t n, const T *x, const T *y, T *out_dev)
{
    if (n == 0) {
        HB_CUDA_TRY(ctx, cudaMemsetAsync(out_dev, 0, sizeof(T), ctx->stream));
        return HB_OK;
    }
    return (x == y) ? dot_launch<T, true>(ctx, n, x, x, out_dev) : dot_launch<T, false>(ctx, n, x, y, out_dev);
}
template int hb_launch_dot<double>(hb_context *, int64_t, const double *, const double *, double *);
template int hb_launch_dot<float>(hb_context *, int64_t, const float *, const float *, float *);

extern "C" {

int hb_dot_f64(hb_context *ctx, int64_t n, const double *x, const double *y, double *res)
{ HB_RANGE("hb_dot_f64"); return dot_impl<double, false>(ctx, n, x, y, res); }
int hb_dot_f32(hb_context *ctx, int64_t n, const float *x, const float *y, float *res)
{ HB_RANGE("hb_dot_f32"); return dot_impl<float, false>(ctx, n, x, y, res); }

int hb_norm_l2_f64(hb_context *ctx, int64_t n, const double *x, int root, double *res)
{
    HB_RANGE("hb_norm_l2_f64");
    int st = dot_impl<double, true>(ctx, n, x, nullptr, res);
    if (!st && root) *res = std::sqrt(*res);
    return st;
}
int hb_norm_l2_f32(hb_context *ctx, int64_t n, const float *x, int root, float *res)
{
    HB_RANGE("hb_norm_l2_f32");
    int st = dot_impl<float, true>(ctx, n, x, nullptr, res);
    if (!st && root) *res = std::sqrt(*res);
    return st;
}

int hb_scaled_sum_f64(hb_context *c, int64_t n, double *x, const double *y, double b)
{ HB_RANGE("hb_scaled_sum_f64"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<double, OP_AXPY>(c, n, x, x, y, b); }
int hb_scaled_sum_f32(hb_context *c, int64_t n, float *x, const float *y, float b)
{ HB_RANGE("hb_scaled_sum_f32"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<float, OP_AXPY>(c, n, x, x, y, b); }
int hb_scaled_sum3_f64(hb_context *c, int64_t n, double *r, const double *x, const double *y, double b)
{ HB_RANGE("hb_scaled_sum3_f64"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<double, OP_AXPY3>(c, n, r, x, y, b); }
int hb_scaled_sum3_f32(hb_context *c, int64_t n, float *r, const float *x, const float *y, float b)
{ HB_RANGE("hb_scaled_sum3_f32"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<float, OP_AXPY3>(c, n, r, x, y, b); }
int hb_scale_f64(hb_context *c, int64_t n, double *x, double a)
{ HB_RANGE("hb_scale_f64"); if (!x) return HB_ERR_INVALID; return ew_launch<double, OP_SCALE>(c, n, x, x, nullptr, a); }
int hb_scale_f32(hb_context *c, int64_t n, float *x, float a)
{ HB_RANGE("hb_scale_f32"); if (!x) return HB_ERR_INVALID; return ew_launch<float, OP_SCALE>(c, n, x, x, nullptr, a); }
int hb_sum_f64(hb_context *c, int64_t n, double *x, const double *y)
{ HB_RANGE("hb_sum_f64"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<double, OP_SUM>(c, n, x, x, y, 0.0); }
int hb_sum_f32(hb_context *c, int64_t n, float *x, const float *y)
{ HB_RANGE("hb_sum_f32"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<float, OP_SUM>(c, n, x, x, y, 0.f); }
int hb_difference_f64(hb_context *c, int64_t n, double *r, const double *x, const double *y)
{ HB_RANGE("hb_difference_f64"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<double, OP_DIFF>(c, n, r, x, y, 0.0); }
int hb_difference_f32(hb_context *c, int64_t n, float *r, const float *x, const float *y)
{ HB_RANGE("hb_difference_f32"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<float, OP_DIFF>(c, n, r, x, y, 0.f); }
int hb_element_product_f64(hb_context *c, int64_t n, double *r, const double *x, const double *y)
{ HB_RANGE("hb_element_product_f64"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<double, OP_EPROD>(c, n, r, x, y, 0.0); }
int hb_element_product_f32(hb_context *c, int64_t n, float *r, const float *x, const float *y)
{ HB_RANGE("hb_element_product_f32"); if (!x || !y) return HB_ERR_INVALID; return ew_launch<float, OP_EPROD>(c, n, r, x, y, 0.f); }
int hb_fill_f64(hb_context *c, int64_t n, double *x, double v)
{ return ew_launch<double, OP_FILL>(c, n, x, nullptr, nullptr, v); }
int hb_fill_f32(hb_context *c, int64_t n, float *x, float v)
{ return ew_launch<float, OP_FILL>(c, n, x, nullptr, nullptr, v); }

int hb_copy(hb_context *ctx, void *dst, const void *src, int64_t bytes)
{
    if (!ctx || !dst || !src || bytes < 0) return HB_ERR_INVALID;
    if (bytes == 0) return HB_OK;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return HB_OK;
}

int hb_convert_f64_f32(hb_context *ctx, int64_t n, float *dst, const double *src)
{ HB_RANGE("hb_convert_f64_f32"); return convert_impl<double, float>(ctx, n, dst, src); }
int hb_convert_f32_f64(hb_context *ctx, int64_t n, double *dst, const float *src)
{ HB_RANGE("hb_convert_f32_f64"); return convert_impl<float, double>(ctx, n, dst, src); }

}  // extern "C"
