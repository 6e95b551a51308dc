// hb_resident.cuh -- pieces shared by the resident-operator solver kernels (cg_res_kernel in
// hb_cg.cu, pcg_res_kernel in hb_pcg.cu).
//
// A resident kernel runs one block per SM (fewer for small systems); block b owns the rows
// [b*rpb, min(rows, (b+1)*rpb)) and keeps, for the whole solve, its ELL rows in shared memory
// (values in slot-major order, columns as offsets into its window) plus vectors on its column
// window: the contiguous range of columns that covers its own rows and every column they reach
// (or, when that range is wider than the window capacity, the capacity centred on the own rows;
// columns outside it are then gathered from global memory).  Grid-wide reductions go through
// hbd::CountExchange; res_partial / res_total_* give the fixed reduction tree that makes every
// block hold the same scalars.
#pragma once
#include "hb_spmv_core.cuh"

#include <climits>

namespace hbr {

constexpr int RES_THREADS = 512;
constexpr int RES_MAX_BLOCKS = 256;

// The block's partial, in thread 0: warp trees, then warp 0 sums the warp results.  One
// __syncthreads; the red[] slots are free again because every caller passes another block-wide
// barrier (the exchange) before the next call.
template <typename T>
__device__ __forceinline__ T res_partial(T v, T *red)
{
    v = hbd::warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) v = hbd::warp_sum((int)threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : T(0));
    return v;
}

// The grid total of one slot array: warp 0 loads the partials (lane l: l, l + 32, ... summed in
// order, then a warp tree) -- the same value in every block -- and broadcasts it through shared
// memory; the other warps' loads (the halo) go out between res_total_load and res_total_sum.
// Reading the partials in one warp per block keeps the L2 lines that hold them from being
// hammered by every warp of the grid at once.
template <typename T>
__device__ __forceinline__ void res_total_load(const T *slots, unsigned G, T (&pv)[RES_MAX_BLOCKS / 32])
{
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
#pragma unroll
        for (int i = 0; i < RES_MAX_BLOCKS / 32; ++i)
            pv[i] = (lane + 32 * i < (int)G) ? __ldcg(slots + lane + 32 * i) : T(0);
    }
}
// Ends in a __syncthreads (which also orders the halo's shared-memory writes before their use).
template <typename T>
__device__ __forceinline__ T res_total_sum(unsigned G, const T (&pv)[RES_MAX_BLOCKS / 32], T *bcast)
{
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        T v = T(0);
#pragma unroll
        for (int i = 0; i < RES_MAX_BLOCKS / 32; ++i)
            if (lane + 32 * i < (int)G) v = hbd::add(v, pv[i]);
        v = hbd::warp_sum(v);
        if (lane == 0) *bcast = v;
    }
    __syncthreads();
    return *bcast;
}

// A block's rows and window: own rows [lo, hi) (nr of them), window [wlo, wlo + W).
struct ResWindow {
    int64_t lo, hi, wlo, W;
    int nr;
    __device__ int64_t own() const { return lo - wlo; }    // window offset of the first own row
};

// Finds the block's window and stages its ELL rows: Ax_s[k * rpb + i] = value, Aj_s[k * rpb + i]
// = window offset of the column, -1 for padding, -(column + 2) for a column outside the window.
// Ends in a __syncthreads.
template <typename T, int KT>
__device__ ResWindow res_stage(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t ld, int K_rt,
                               int64_t rows, int64_t rpb, int64_t wcap, T *Ax_s, int32_t *Aj_s, int *s_min, int *s_max)
{
    const int K = KT > 0 ? KT : K_rt;
    ResWindow w;
    w.lo = (int64_t)blockIdx.x * rpb;
    w.hi = min(rows, w.lo + rpb);
    w.nr = w.hi > w.lo ? (int)(w.hi - w.lo) : 0;
    if (threadIdx.x == 0) { *s_min = INT_MAX; *s_max = -1; }
    __syncthreads();
    {
        int cmin = INT_MAX, cmax = -1;
        for (int64_t q = threadIdx.x; q < (int64_t)K * w.nr; q += blockDim.x) {
            const int k = (int)(q / w.nr), il = (int)(q - (int64_t)k * w.nr);
            const int32_t j = Aj[(int64_t)k * ld + w.lo + il];
            if (j >= 0) { cmin = min(cmin, (int)j); cmax = max(cmax, (int)j); }
        }
        if (w.nr > 0) { cmin = min(cmin, (int)w.lo); cmax = max(cmax, (int)(w.hi - 1)); }
        atomicMin(s_min, cmin);
        atomicMax(s_max, cmax);
    }
    __syncthreads();
    w.wlo = 0;
    w.W = 0;
    if (w.nr > 0) {
        if ((int64_t)*s_max - *s_min + 1 <= wcap) {
            w.wlo = *s_min;
            w.W = (int64_t)*s_max - *s_min + 1;
        } else {
            w.wlo = w.lo - (wcap - w.nr) / 2;
            if (w.wlo < 0) w.wlo = 0;
            w.W = wcap < rows - w.wlo ? wcap : rows - w.wlo;
        }
    }
    for (int64_t q = threadIdx.x; q < (int64_t)K * w.nr; q += blockDim.x) {
        const int k = (int)(q / w.nr), il = (int)(q - (int64_t)k * w.nr);
        const int64_t gi = (int64_t)k * ld + w.lo + il;
        const int32_t j = Aj[gi];
        Ax_s[(int64_t)k * rpb + il] = Ax[gi];
        Aj_s[(int64_t)k * rpb + il] = j < 0 ? -1 : ((j >= w.wlo && j < w.wlo + w.W) ? (int32_t)(j - w.wlo) : -(j + 2));
    }
    __syncthreads();
    return w;
}

// Loads the window's rows other than the block's own (its halo) of the global vector g into the
// window array v_w: two loads in flight per thread.
template <typename T>
__device__ __forceinline__ void res_halo(const T *__restrict__ g, T *v_w, const ResWindow &w)
{
    const int64_t n_left = w.nr > 0 ? w.own() : 0;
    const int64_t n_halo = w.nr > 0 ? w.own() + (w.wlo + w.W - w.hi) : 0;
    for (int64_t q = threadIdx.x; q < n_halo; q += 2 * (int64_t)blockDim.x) {
        const int64_t q2 = q + blockDim.x;
        const int64_t w1 = q < n_left ? q : q - n_left + (w.hi - w.wlo);
        const int64_t w2 = q2 < n_left ? q2 : q2 - n_left + (w.hi - w.wlo);
        const T a = __ldcg(g + w.wlo + w1);
        const T b = q2 < n_halo ? __ldcg(g + w.wlo + w2) : T(0);
        v_w[w1] = a;
        if (q2 < n_halo) v_w[w2] = b;
    }
}

// Decodes a staged column: the global column of code c (c >= 0: window offset; c <= -2: outside).
__device__ __forceinline__ int64_t res_column(int32_t c, int64_t wlo)
{
    return c >= 0 ? (int64_t)c + wlo : -(int64_t)c - 2;
}

// Shared memory of a resident kernel: the ELL rows (values and int32 codes), nwin window arrays
// of wcap entries and nown arrays of rpb entries.
template <typename T> size_t res_smem_bytes(int K, int64_t rpb, int64_t wcap, int nwin, int nown)
{
    return (size_t)((int64_t)K * rpb + nwin * wcap + nown * rpb) * sizeof(T) + (size_t)K * rpb * sizeof(int32_t);
}

struct ResPlan {
    int blocks;
    int64_t rpb, wcap;
    size_t smem;
};

// One block per SM (fewer for small systems, about 128 rows each), the window as large as the
// shared memory left over allows.  False when the rows of a block do not fit.
template <typename T>
bool res_plan(hb_context *ctx, int64_t rows, int K, int nwin, int nown, const void *kernel, ResPlan *out)
{
    int dev = 0, optin = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const size_t avail = (size_t)optin - 1024;    // static shared memory of the kernels
    const int64_t G = std::max<int64_t>(1, std::min<int64_t>(std::min(ctx->num_sms, RES_MAX_BLOCKS), (rows + 127) / 128));
    const int64_t r = (rows + G - 1) / G;
    const size_t fixed = res_smem_bytes<T>(K, r, 0, nwin, nown);
    if (fixed + nwin * (size_t)r * sizeof(T) > avail) return false;
    const int64_t w = std::min<int64_t>(rows, (int64_t)((avail - fixed) / (nwin * sizeof(T))));
    const size_t bytes = res_smem_bytes<T>(K, r, w, nwin, nown);
    // The kernel's dynamic shared memory cap is process-wide: always the largest value, so that
    // plans of concurrent solves (other threads, other contexts) never lower it under each
    // other's launches; each launch passes its own size.
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess ||
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) != cudaSuccess ||
        bytes + fa.sharedSizeBytes > (size_t)optin ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, RES_THREADS, bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if ((int64_t)occ * ctx->num_sms < G) return false;
    out->blocks = (int)G;
    out->rpb = r;
    out->wcap = w;
    out->smem = bytes;
    return true;
}

}  // namespace hbr
