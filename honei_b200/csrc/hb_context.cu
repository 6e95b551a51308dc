// hb_context.cu -- context lifetime, error text, workspace management.
//
// The context plays the part of the reference's per-device runtime: GPUPool's worker thread
// per device (honei/backends/cuda/gpu_pool.hh:53-88) becomes the caller's thread plus one
// CUDA stream, and MemoryBackend<tags::GPU::CUDA>'s transient cudaMalloc/cudaFree per
// reduction (honei/backends/cuda/dot_product.cu:77-155) becomes one persistent scratch block.
#include "hb_internal.cuh"

#include <cstring>

void hb_note_error(hb_context *ctx, cudaError_t e, const char *what)
{
    // clear the runtime's last error (a failed launch or API call that is not sticky), so the
    // failure is reported once, through the status this library returns, and not again by the
    // caller's next unrelated CUDA call
    cudaGetLastError();
    if (!ctx) return;
    ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
}

int hb_check_launch(hb_context *ctx, const char *what)
{
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        hb_note_error(ctx, e, what);
        return HB_ERR_CUDA;
    }
    return HB_OK;
}

int hb_ensure_work(hb_context *ctx, size_t bytes)
{
    if (bytes <= ctx->work_bytes) return HB_OK;
    if (ctx->work) {
        // the old block may still be in use by queued work on this stream
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaStreamSynchronize"); return HB_ERR_CUDA; }
        cudaFree(ctx->work);
        ctx->work = nullptr;
        ctx->work_bytes = 0;
    }
    size_t want = bytes + bytes / 8;
    if (cudaMalloc(&ctx->work, want) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_ALLOC;
    }
    ctx->work_bytes = want;
    return HB_OK;
}

extern "C" {

int hb_create(hb_context **out, int device)
{
    if (!out) return HB_ERR_INVALID;
    *out = nullptr;
    hb_context *ctx = new hb_context();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete ctx; return HB_ERR_CUDA; }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&ctx->scratch, HB_SCRATCH_BYTES) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return HB_ERR_ALLOC;
    }
    ctx->scratch_bytes = HB_SCRATCH_BYTES;
    if (cudaMemset(ctx->scratch, 0, HB_SCRATCH_BYTES) != cudaSuccess ||
        cudaMallocHost(&ctx->pinned, 4096) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(ctx->scratch);
        delete ctx;
        return HB_ERR_ALLOC;
    }
    std::memset(ctx->pinned, 0, 4096);
    // keep freed stream-ordered allocations in the device pool (no release to the driver
    // between requests)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = ctx;
    return HB_OK;
}

int hb_destroy(hb_context *ctx)
{
    if (!ctx) return HB_ERR_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->work) cudaFree(ctx->work);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
    return HB_OK;
}

int hb_set_stream(hb_context *ctx, void *stream)
{
    if (!ctx) return HB_ERR_INVALID;
    ctx->stream = (cudaStream_t)stream;
    return HB_OK;
}

int hb_synchronize(hb_context *ctx)
{
    if (!ctx) return HB_ERR_INVALID;
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return HB_OK;
}

const char *hb_status_string(int status)
{
    switch (status) {
        case HB_OK: return "ok";
        case HB_ERR_INVALID: return "invalid argument";
        case HB_ERR_SIZE: return "vector or matrix sizes do not match";
        case HB_ERR_CUDA: return "CUDA error";
        case HB_ERR_ALLOC: return "allocation failed";
        case HB_ERR_TIMEOUT: return "bounded device wait timed out";
        case HB_ERR_UNSUPPORTED: return "unsupported shape";
        case HB_ERR_CAPACITY: return "over capacity (HBM budget or slots)";
        case HB_ERR_NOT_FOUND: return "unknown request";
        case HB_ERR_NONFINITE: return "non-finite input";
        default: return "unknown status";
    }
}

const char *hb_last_error(hb_context *ctx)
{
    return ctx ? ctx->last_error.c_str() : "";
}

uint64_t hb_launch_count(hb_context *ctx)
{
    return ctx ? ctx->launches : 0;
}

int hb_cg_set_resident(hb_context *ctx, int enable)
{
    if (!ctx) return HB_ERR_INVALID;
    const int prev = ctx->cg_resident;
    ctx->cg_resident = enable != 0;
    return prev;
}

int hb_cg_set_layout(hb_context *ctx, int rows_per_thread)
{
    if (!ctx || (rows_per_thread != 1 && rows_per_thread != 4)) return -1;
    const int prev = ctx->cg_row_layout ? 1 : 4;
    ctx->cg_row_layout = rows_per_thread == 1;
    return prev;
}

int hb_set_block_size(hb_context *ctx, int family, int threads)
{
    if (!ctx || family < HB_BLOCK_ELL || family > HB_BLOCK_VECTOR) return -1;
    const int max = family == HB_BLOCK_VECTOR ? 1024 : 256;
    if (threads != 0 && (threads < 32 || threads > max || threads % 32)) return -1;
    const int prev = ctx->block[family];
    ctx->block[family] = threads;
    return prev;
}

int hb_reserve(hb_context *ctx, int64_t n)
{
    if (!ctx || n < 0) return HB_ERR_INVALID;
    // CG needs 5 padded vectors of doubles; MG/IR keep their own.
    const int64_t ld = hb_round_up(n > 0 ? n : 1, 64);
    return hb_ensure_work(ctx, (size_t)ld * 8 * 6);
}

}  // extern "C"
