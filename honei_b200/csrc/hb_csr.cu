// hb_csr.cu -- SparseMatrixCSR<DT> (honei/la/sparse_matrix_csr.hh) on the device:
//   Product<tags::GPU::CUDA>::value(DV, SparseMatrixCSR, DV)   honei/la/product.hh:1762-1764
//   Defect<tags::GPU::CUDA>::value(DV, DV, SparseMatrixCSR, DV) honei/math/defect.hh:673-676
// with the tags::CPU arithmetic (honei/la/product.hh:209-242, honei/math/defect.hh:386-419):
// per row, sum = 0, then over the row's blocks and each block's csr::blocksize lanes in order,
// sum += Ax * x[column] for lanes whose column is below cols; the defect is rhs - sum.  Each row
// is summed by one thread in exactly that order, so the results are bit-identical to tags::CPU.
//
// Layout (hb_csr): Ar int64[rows + 1] block offsets, Aj int32[nblocks] first column of each
// block (the reference's 64-bit indices narrowed at import; a column at or beyond cols is
// stored as cols, whose lanes the bounds test skips exactly as it skips the original), Ax
// dtype[nblocks * blocksize].
//
// Kernel: one thread per row, its entries GATHER at a time with their Aj, Ax and x loads in
// flight together, summed in the reference's order.  Consecutive rows' entries are contiguous,
// so a warp's loads of entry j fall on a few lines that its loads of entries j + 1, ... reuse
// from L1: DRAM traffic stays at the algorithmic bytes (the reference's CUDA kernel is also one
// thread per row, product.cu:257-296, but reads x through a texture and 64-bit indices one
// entry at a time).  Robust against any Ar / Aj content: block offsets are clamped to
// [0, nblocks] and every column is tested against [0, cols) before x is read.
#include "hb_internal.cuh"

#include <type_traits>

namespace {

constexpr int CSR_THREADS = 256;
constexpr int GATHER = 8;          // entries of a row whose loads are in flight together

__device__ __forceinline__ int64_t clamp_block(int64_t v, int64_t nblocks)
{
    return v < 0 ? 0 : (v > nblocks ? nblocks : v);
}

// MODE 0: y = A x; MODE 1: y = rhs - A x.  BS > 0: compile-time blocksize, 0: runtime.
// One thread per row; the row's entries (block i, lane k: value Ax[i * bs + k], column
// Aj[i] + k) are taken GATHER at a time -- their Aj, Ax and x loads in flight together -- and
// summed in order, skipping columns outside [0, cols).
template <typename T, int MODE, int BS>
__global__ void __launch_bounds__(CSR_THREADS) csr_kernel(int64_t rows, int64_t cols, int64_t nblocks, int64_t bs_rt,
                                                          const int64_t *__restrict__ Ar,
                                                          const int32_t *__restrict__ Aj,
                                                          const T *__restrict__ Ax, const T *__restrict__ x,
                                                          const T *__restrict__ rhs, T *__restrict__ y)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    const int64_t bs = BS > 0 ? BS : bs_rt;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < rows; row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t lo = clamp_block(Ar[row], nblocks) * bs;
        const int64_t hi = max(lo, clamp_block(Ar[row + 1], nblocks) * bs);
        T sum = T(0);
        // blocksize 1: the column is Aj itself (int32, -1 past the row's end); otherwise block
        // start + lane, in 64 bits
        using Col = typename std::conditional<BS == 1, int32_t, int64_t>::type;
        for (int64_t e = lo; e < hi; e += GATHER) {
            Col c[GATHER];
            T av[GATHER], xv[GATHER];
#pragma unroll
            for (int j = 0; j < GATHER; ++j) {
                const bool in = e + j < hi;
                c[j] = in ? (BS == 1 ? (Col)Aj[e + j] : (Col)((int64_t)Aj[(e + j) / bs] + (e + j) % bs)) : Col(-1);
                av[j] = in ? Ax[e + j] : T(0);
            }
#pragma unroll
            for (int j = 0; j < GATHER; ++j)
                xv[j] = (typename std::make_unsigned<Col>::type)c[j] < (uint64_t)cols ? __ldg(x + c[j]) : T(0);
#pragma unroll
            for (int j = 0; j < GATHER; ++j)
                if ((typename std::make_unsigned<Col>::type)c[j] < (uint64_t)cols) sum = add(sum, mul(av[j], xv[j]));
        }
        y[row] = MODE == 1 ? sub(rhs[row], sum) : sum;
    }
}

template <typename T>
__global__ void csr_import_kernel(int64_t rows, int64_t cols, int64_t nblocks, int64_t bs,
                                  const uint64_t *__restrict__ Ar_ref, const uint64_t *__restrict__ Aj_ref,
                                  const T *__restrict__ Ax_ref, int64_t *__restrict__ Ar,
                                  int32_t *__restrict__ Aj, T *__restrict__ Ax, int *bad)
{
    const int64_t nvals = nblocks * bs;
    const int64_t total = max(rows + 1, nvals);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        if (i <= rows) {
            const uint64_t v = Ar_ref[i];
            Ar[i] = (int64_t)(v < (uint64_t)nblocks ? v : (uint64_t)nblocks);
            const bool ok = v <= (uint64_t)nblocks && (i > 0 || v == 0) && (i < rows || v == (uint64_t)nblocks) &&
                            (i == 0 || Ar_ref[i - 1] <= v);
            if (!ok) atomicOr(bad, 1);
        }
        if (i < nblocks) {
            const uint64_t c = Aj_ref[i];
            Aj[i] = (int32_t)(c >= (uint64_t)cols ? (uint64_t)cols : c);
        }
        if (i < nvals) Ax[i] = Ax_ref[i];
    }
}

int check_csr(const hb_csr *A, int dtype)
{
    if (!A || A->dtype != dtype) return HB_ERR_INVALID;
    if (A->rows < 0 || A->cols < 0 || A->blocksize < 1 || A->nblocks < 0) return HB_ERR_INVALID;
    if (A->cols > INT32_MAX - 1 || A->rows > INT32_MAX) return HB_ERR_UNSUPPORTED;
    if (!A->Ar || (A->nblocks > 0 && (!A->Aj || !A->Ax))) return HB_ERR_INVALID;
    const size_t es = dtype == HB_F64 ? 8 : 4;
    if ((uintptr_t)A->Ar % 8 || (uintptr_t)A->Aj % 4 || (uintptr_t)A->Ax % es) return HB_ERR_INVALID;
    return HB_OK;
}

template <typename T, int MODE>
int launch(hb_context *ctx, const hb_csr *A, const T *x, const T *rhs, T *y, int dtype)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = check_csr(A, dtype);
    if (st) return st;
    if (A->rows == 0) return HB_OK;
    if (!y || (A->cols > 0 && !x) || (MODE == 1 && !rhs)) return HB_ERR_INVALID;
    if (((uintptr_t)x | (uintptr_t)y | (uintptr_t)rhs) % sizeof(T)) return HB_ERR_INVALID;
    const unsigned blocks = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>((A->rows + CSR_THREADS - 1) / CSR_THREADS, (int64_t)ctx->num_sms * 8));
    if (A->blocksize == 1)
        csr_kernel<T, MODE, 1><<<blocks, CSR_THREADS, 0, ctx->stream>>>(A->rows, A->cols, A->nblocks, 1, A->Ar,
                                                                      A->Aj, (const T *)A->Ax, x, rhs, y);
    else
        csr_kernel<T, MODE, 0><<<blocks, CSR_THREADS, 0, ctx->stream>>>(A->rows, A->cols, A->nblocks, A->blocksize,
                                                                      A->Ar, A->Aj, (const T *)A->Ax, x, rhs, y);
    return hb_check_launch(ctx, "csr_kernel");
}

template <typename T>
int import_impl(hb_context *ctx, const uint64_t *Ar_ref, const uint64_t *Aj_ref, const T *Ax_ref, hb_csr *out,
                int dtype)
{
    if (!ctx || !out || !Ar_ref) return HB_ERR_INVALID;
    out->dtype = dtype;
    int st = check_csr(out, dtype);
    if (st) return st;
    if (out->nblocks > 0 && (!Aj_ref || !Ax_ref)) return HB_ERR_INVALID;
    int *bad = (int *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
    const int64_t total = std::max<int64_t>(out->rows + 1, out->nblocks * out->blocksize);
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32));
    csr_import_kernel<T><<<blocks, 256, 0, ctx->stream>>>(out->rows, out->cols, out->nblocks, out->blocksize, Ar_ref,
                                                          Aj_ref, Ax_ref, out->Ar, out->Aj, (T *)out->Ax, bad);
    st = hb_check_launch(ctx, "csr_import_kernel");
    if (st) return st;
    int *h = (int *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return *h ? HB_ERR_INVALID : HB_OK;
}

}  // namespace

extern "C" {

int hb_csr_import_f64(hb_context *ctx, const uint64_t *Ar_ref, const uint64_t *Aj_ref, const double *Ax_ref,
                      hb_csr *out)
{
    HB_RANGE("hb_csr_import_f64");
    return import_impl<double>(ctx, Ar_ref, Aj_ref, Ax_ref, out, HB_F64);
}

int hb_csr_import_f32(hb_context *ctx, const uint64_t *Ar_ref, const uint64_t *Aj_ref, const float *Ax_ref,
                      hb_csr *out)
{
    HB_RANGE("hb_csr_import_f32");
    return import_impl<float>(ctx, Ar_ref, Aj_ref, Ax_ref, out, HB_F32);
}

int hb_csr_spmv_f64(hb_context *ctx, const hb_csr *A, const double *x, double *y)
{
    HB_RANGE("hb_csr_spmv_f64");
    return launch<double, 0>(ctx, A, x, nullptr, y, HB_F64);
}

int hb_csr_spmv_f32(hb_context *ctx, const hb_csr *A, const float *x, float *y)
{
    HB_RANGE("hb_csr_spmv_f32");
    return launch<float, 0>(ctx, A, x, nullptr, y, HB_F32);
}

int hb_csr_defect_f64(hb_context *ctx, const hb_csr *A, const double *rhs, const double *x, double *r)
{
    HB_RANGE("hb_csr_defect_f64");
    return launch<double, 1>(ctx, A, x, rhs, r, HB_F64);
}

int hb_csr_defect_f32(hb_context *ctx, const hb_csr *A, const float *rhs, const float *x, float *r)
{
    HB_RANGE("hb_csr_defect_f32");
    return launch<float, 1>(ctx, A, x, rhs, r, HB_F32);
}

}  // extern "C"
