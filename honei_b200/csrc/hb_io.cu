// hb_io.cu -- HONEI's binary ELL matrix files straight to and from the device layout.
//
// File format (MatrixIO<io_formats::ELL>, honei/math/matrix_io.hh:433-582): five uint64
// {size, rows, columns, stride, num_cols_per_row}, then uint64 Aj[size] and double Ax[size] in
// the one-lane reference layout (entry k of row r at r + k * stride).  The reader keeps, per
// row, the leading slots up to the first zero value -- the row length the reference's raw-array
// constructor derives (honei/la/sparse_matrix_ell-impl.hh:184-206) -- and converts the values
// to the target precision (convert<tags::CPU>, as read_matrix does for float matrices).
//
// Reading streams the file through two pinned staging buffers into device memory (the copy of
// one chunk overlaps the read of the next), then one kernel builds the hb_ell arrays.  Writing
// compacts every row's stored entries (zero values dropped, as SparseMatrixELL(SparseMatrix)
// does, honei/la/sparse_matrix_ell-impl.hh:75-122) into the reference layout with
// num_cols_per_row = the longest row and stride = rows rounded up to 32.
#include "hb_internal.cuh"

#include <cstdio>
#include <vector>

namespace {

constexpr size_t STAGE_BYTES = 8u << 20;

template <typename T>
__global__ void ell_file_kernel(int64_t rows, int64_t cols, int64_t stride, int64_t ncpr, int64_t ld,
                                const uint64_t *__restrict__ Aj_raw, const double *__restrict__ Ax_raw,
                                int32_t *__restrict__ Aj, T *__restrict__ Ax, int *bad)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < ld; r += (int64_t)gridDim.x * blockDim.x) {
        bool live = r < rows;
        for (int64_t k = 0; k < ncpr; ++k) {
            int32_t j = -1;
            T a = T(0);
            if (live) {
                const double v = Ax_raw[r + k * stride];
                if (v == 0.0) {
                    live = false;   // the row ends at its first zero value
                } else {
                    const uint64_t c = Aj_raw[r + k * stride];
                    if (c >= (uint64_t)cols) {
                        atomicExch(bad, 1);
                    } else {
                        j = (int32_t)c;
                        a = (T)v;
                    }
                }
            }
            Aj[k * ld + r] = j;
            Ax[k * ld + r] = a;
        }
    }
}

struct File {
    FILE *f = nullptr;
    explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() { if (f) std::fclose(f); }
};

int read_header(FILE *f, uint64_t h[5])
{
    if (std::fread(h, sizeof(uint64_t), 5, f) != 5) return HB_ERR_INVALID;
    const uint64_t size = h[0], rows = h[1], stride = h[3], ncpr = h[4];
    if (ncpr < 1 || stride < rows || size != ncpr * stride) return HB_ERR_INVALID;
    if (rows > (uint64_t)INT32_MAX || h[2] > (uint64_t)INT32_MAX) return HB_ERR_UNSUPPORTED;
    return HB_OK;
}

// Streams `bytes` of the file into device memory at dst through two pinned buffers.
int stream_to_device(hb_context *ctx, FILE *f, void *dst, size_t bytes)
{
    void *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    int st = HB_OK;
    for (int i = 0; i < 2 && !st; ++i) {
        if (cudaMallocHost(&stage[i], STAGE_BYTES) != cudaSuccess) st = HB_ERR_ALLOC;
        else if (cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming) != cudaSuccess) st = HB_ERR_CUDA;
    }
    size_t off = 0;
    int buf = 0;
    while (!st && off < bytes) {
        const size_t n = std::min(STAGE_BYTES, bytes - off);
        if (cudaEventSynchronize(done[buf]) != cudaSuccess) { st = HB_ERR_CUDA; break; }
        if (std::fread(stage[buf], 1, n, f) != n) { st = HB_ERR_INVALID; break; }
        if (cudaMemcpyAsync((char *)dst + off, stage[buf], n, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
            cudaEventRecord(done[buf], ctx->stream) != cudaSuccess) {
            st = HB_ERR_CUDA;
            break;
        }
        off += n;
        buf ^= 1;
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && !st) st = HB_ERR_CUDA;
    for (int i = 0; i < 2; ++i) {
        if (done[i]) cudaEventDestroy(done[i]);
        if (stage[i]) cudaFreeHost(stage[i]);
    }
    cudaGetLastError();
    return st;
}

template <typename T>
int read_impl(hb_context *ctx, const char *path, hb_ell *out, int dtype)
{
    if (!ctx || !path || !out) return HB_ERR_INVALID;
    File file(path, "rb");
    if (!file.f) return HB_ERR_NOT_FOUND;
    uint64_t h[5];
    int st = read_header(file.f, h);
    if (st) return st;
    const int64_t size = (int64_t)h[0], rows = (int64_t)h[1], cols = (int64_t)h[2], stride = (int64_t)h[3],
                  ncpr = (int64_t)h[4];
    int64_t K, ld;
    hb_ell_layout(rows, ncpr, 1, &K, &ld);
    if (out->K != K || out->ld != ld) return HB_ERR_SIZE;
    out->rows = rows;
    out->cols = cols;
    if ((st = hb_check_ell(out, dtype))) return st;
    if ((st = hb_ensure_work(ctx, (size_t)size * 16))) return st;
    uint64_t *Aj_raw = (uint64_t *)ctx->work;
    double *Ax_raw = (double *)((char *)ctx->work + (size_t)size * 8);
    if ((st = stream_to_device(ctx, file.f, Aj_raw, (size_t)size * 8))) return st;
    if ((st = stream_to_device(ctx, file.f, Ax_raw, (size_t)size * 8))) return st;
    int *bad = (int *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((ld + 255) / 256, (int64_t)ctx->num_sms * 32));
    ell_file_kernel<T><<<blocks, 256, 0, ctx->stream>>>(rows, cols, stride, ncpr, ld, Aj_raw, Ax_raw, out->Aj,
                                                        (T *)out->Ax, bad);
    if ((st = hb_check_launch(ctx, "ell_file_kernel"))) return st;
    int *hb = (int *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(hb, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return *hb ? HB_ERR_INVALID : HB_OK;
}

}  // namespace

extern "C" {

int hb_ell_file_info(const char *path, int64_t *info)
{
    if (!path || !info) return HB_ERR_INVALID;
    File file(path, "rb");
    if (!file.f) return HB_ERR_NOT_FOUND;
    uint64_t h[5];
    int st = read_header(file.f, h);
    if (st) return st;
    for (int i = 0; i < 5; ++i) info[i] = (int64_t)h[i];
    return HB_OK;
}

int hb_ell_read_file_f64(hb_context *ctx, const char *path, hb_ell *out)
{
    HB_RANGE("hb_ell_read_file_f64");
    return read_impl<double>(ctx, path, out, HB_F64);
}

int hb_ell_read_file_f32(hb_context *ctx, const char *path, hb_ell *out)
{
    HB_RANGE("hb_ell_read_file_f32");
    return read_impl<float>(ctx, path, out, HB_F32);
}

int hb_ell_write_file(hb_context *ctx, const hb_ell *A, const char *path)
{
    HB_RANGE("hb_ell_write_file");
    if (!ctx || !A || !path) return HB_ERR_INVALID;
    int st = hb_check_ell(A, HB_F64);
    if (st) return st;
    const int64_t rows = A->rows, K = A->K, ld = A->ld;
    std::vector<int32_t> aj((size_t)(K * ld));
    std::vector<double> ax((size_t)(K * ld));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(aj.data(), A->Aj, aj.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(ax.data(), A->Ax, ax.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    // longest row (stored, non-zero entries), at least 1
    uint64_t ncpr = 1;
    for (int64_t r = 0; r < rows; ++r) {
        uint64_t n = 0;
        for (int64_t k = 0; k < K; ++k)
            if (aj[k * ld + r] >= 0 && ax[k * ld + r] != 0.0) ++n;
        ncpr = std::max(ncpr, n);
    }
    const uint64_t stride = 32 * (((uint64_t)rows + 31) / 32), size = ncpr * stride;
    std::vector<uint64_t> fj(size, 0);
    std::vector<double> fx(size, 0.0);
    for (int64_t r = 0; r < rows; ++r) {
        uint64_t t = 0;
        for (int64_t k = 0; k < K; ++k) {
            const int32_t j = aj[k * ld + r];
            const double v = ax[k * ld + r];
            if (j < 0 || v == 0.0) continue;
            fj[r + t * stride] = (uint64_t)j;
            fx[r + t * stride] = v;
            ++t;
        }
    }
    File file(path, "wb");
    if (!file.f) return HB_ERR_NOT_FOUND;
    const uint64_t h[5] = {size, (uint64_t)rows, (uint64_t)A->cols, stride, ncpr};
    if (std::fwrite(h, sizeof(uint64_t), 5, file.f) != 5 || std::fwrite(fj.data(), sizeof(uint64_t), size, file.f) != size ||
        std::fwrite(fx.data(), sizeof(double), size, file.f) != size)
        return HB_ERR_INVALID;
    return HB_OK;
}

}  // extern "C"
