// hb_mg.cu -- multigrid (MGSolver with a V(n_pre, n_post) cycle) and mixed-precision
// iterative refinement (IRSolver) on the device.
//
// Reference: MGData / MGCycleCreation<V::STATIC, CGSolver<NONE>, RISmoother, Restriction
// <PROLMAT>, Prolongation<PROLMAT>> / MGSolver<Norm<l2, true>> (honei/math/mg.hh:57-243,
// 567-662, 1093-1127), RISmoother (honei/math/ri.hh:97-133), IRSolver (honei/math/ir.hh:30-78).
//
// The reference executes its cycle as a list of Operator objects, one tag-dispatched call
// each (honei/math/operator_list.hh:48-90).  Here every level is a short, fixed sequence of
// fused kernels on one stream:
//   n_pre  x  Jacobi sweep   x' = x + P (b - A x)          (defect + ElementProduct + Sum)
//   defect + restriction     d_c = R (b - A x)              (Defect into store, Product)
//   zero c_c, recurse / coarse CG (persistent kernel)
//   prolongation + sum       x += P_l c_c                    (Product into store, Sum)
//   n_post x  Jacobi sweep
// Every fused formula rounds as the reference's operator sequence does; the only
// difference from tags::CPU is the summation order of the norms and of the coarse CG's
// dot products.
#include "hb_internal.cuh"

#include <cmath>
#include <vector>

struct hb_mg {
    hb_context *ctx = nullptr;
    int L = 0;
    int dtype = HB_F64;
    std::vector<hb_ell> A, prol, res;
    hb_mg_params prm{};
    void *mem = nullptr;
    std::vector<void *> P, d, c, store, xt;   // per level
    void *r = nullptr;                          // finest defect (dtype)
    void *cgwork = nullptr;                     // 5 * ld(level 0), dtype
    hb_solve_result *cgres = nullptr;
    void *norm = nullptr;                       // device scalar
    // mixed precision (dtype == F32): FP64 defect, FP32 inner right-hand side and solution
    double *ir_r = nullptr;
    float *ir_b = nullptr, *ir_x = nullptr;
    int64_t used_coarse_total = 0;
    // optional exact coarse solve: dense inverse of A[0] (row-major, dtype), replacing the CG
    void *coarse_inv = nullptr;
    // optional banded levels (hb_mg_create_banded): levels >= 1 smooth and take defects with the
    // banded operator and transfer matrix-free; level 0 keeps its ELL matrix for the coarse CG
    std::vector<hb_q1band> B;
    // fused coarse cycle (FP32 banded hierarchies with a dense coarse solve): levels <= tail_level
    // run as one single-cluster launch; tail_desc is its device descriptor
    int tail_level = -1, tail_top = -1;
    void *tail_desc = nullptr;
    // one cycle of hb_mg_solve_* (V-cycle, finest defect, its squared norm) captured as a CUDA
    // graph for the (x, b) it was captured with; replayed once per cycle
    cudaGraphExec_t cycle_graph = nullptr;
    const void *graph_x = nullptr, *graph_b = nullptr;
    uint64_t graph_kernels = 0;
    bool graph_failed = false;
};

// Drops the captured cycle (its kernels' parameters changed); waits for replays in flight.
static void drop_cycle_graph(hb_mg *mg)
{
    if (!mg->cycle_graph) return;
    cudaStreamSynchronize(mg->ctx->stream);
    cudaGraphExecDestroy(mg->cycle_graph);
    mg->cycle_graph = nullptr;
    mg->graph_x = mg->graph_b = nullptr;
}

namespace {

__global__ void add_f32_to_f64_kernel(int64_t n, double *__restrict__ x, const float *__restrict__ c)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], (double)c[i]);
}

__global__ void f64_to_f32_kernel(int64_t n, float *__restrict__ dst, const double *__restrict__ src)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// Scaled mode: b32 = (float)(r * s) with s = 1/|r|, and x += |r| * (double)c.
__global__ void f64_to_f32_scaled_kernel(int64_t n, float *__restrict__ dst, const double *__restrict__ src, double s)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (float)__dmul_rn(src[i], s);
}

__global__ void add_scaled_f32_to_f64_kernel(int64_t n, double *__restrict__ x, const float *__restrict__ c, double a)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(a, (double)c[i]));
}

inline unsigned ew_blocks(hb_context *ctx, int64_t n)
{
    return (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 16);
}

int launch_add_f32_to_f64(hb_context *ctx, int64_t n, double *x, const float *c)
{
    if (n == 0) return HB_OK;
    add_f32_to_f64_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, x, c);
    return hb_check_launch(ctx, "add_f32_to_f64_kernel");
}

int launch_f64_to_f32(hb_context *ctx, int64_t n, float *dst, const double *src)
{
    if (n == 0) return HB_OK;
    f64_to_f32_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, dst, src);
    return hb_check_launch(ctx, "f64_to_f32_kernel");
}

int launch_f64_to_f32_scaled(hb_context *ctx, int64_t n, float *dst, const double *src, double s)
{
    if (n == 0) return HB_OK;
    f64_to_f32_scaled_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, dst, src, s);
    return hb_check_launch(ctx, "f64_to_f32_scaled_kernel");
}

int launch_add_scaled_f32_to_f64(hb_context *ctx, int64_t n, double *x, const float *c, double a)
{
    if (n == 0) return HB_OK;
    add_scaled_f32_to_f64_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, x, c, a);
    return hb_check_launch(ctx, "add_scaled_f32_to_f64_kernel");
}

#define HB_TRY(expr) do { int s_ = (expr); if (s_) return s_; } while (0)

template <typename T> inline T *tp(void *p) { return static_cast<T *>(p); }

// Device norm: sqrt of the fixed-order sum of squares, read back (one sync).
template <typename T> int norm_host(hb_mg *mg, const T *v, int64_t n, T *out)
{
    hb_context *ctx = mg->ctx;
    HB_TRY(hb_launch_dot<T>(ctx, n, v, v, tp<T>(mg->norm)));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, mg->norm, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *out = std::sqrt(*static_cast<T *>(ctx->pinned));
    return HB_OK;
}

// The level operator in a fused mode: banded levels (l >= 1 of a banded hierarchy) or ELL.
template <typename T> int level_mode(hb_mg *mg, int l, int mode, const T *x, const T *b, const T *P, T *y)
{
    if (!mg->B.empty() && l >= 1) return hb_launch_band_mode<T>(mg->ctx, &mg->B[l], mode, x, b, P, y);
    return hb_launch_spmv_mode<T>(mg->ctx, &mg->A[l], mode, x, b, P, y);
}

template <typename T> int smooth(hb_mg *mg, int l, T *X, const T *B, int64_t sweeps)
{
    hb_context *ctx = mg->ctx;
    T *cur = X, *other = tp<T>(mg->xt[l]);
    for (int64_t s = 0; s < sweeps; ++s) {
        HB_TRY(level_mode<T>(mg, l, HB_MODE_JACOBI, cur, B, tp<T>(mg->P[l]), other));
        T *t = cur; cur = other; other = t;
    }
    if (cur != X)
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(X, cur, sizeof(T) * mg->A[l].rows, cudaMemcpyDeviceToDevice, ctx->stream));
    return HB_OK;
}

// x = Ainv b on the coarsest level (one block, one thread per row, fixed summation order).
template <typename T>
__global__ void dense_solve_kernel(int64_t n, const T *__restrict__ inv, const T *__restrict__ b, T *__restrict__ x)
{
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        T acc = T(0);
        for (int64_t j = 0; j < n; ++j) acc = hbd::add(acc, hbd::mul(inv[i * n + j], b[j]));
        x[i] = acc;
    }
}

// The fused coarse cycle applies to FP32 hierarchies only.
inline bool run_tail(hb_mg *mg, int l, float *X, const float *B, int *st)
{
    if (l != mg->tail_level || !mg->tail_desc) return false;
    *st = hb_tail_launch(mg->ctx, mg->tail_desc, X, B);
    return true;
}
inline bool run_tail(hb_mg *, int, double *, const double *, int *) { return false; }

template <typename T> int vcycle(hb_mg *mg, int l, T *X, const T *B)
{
    hb_context *ctx = mg->ctx;
    int tst = HB_OK;
    if (run_tail(mg, l, X, B, &tst)) return tst;
    if (l == 0 && mg->coarse_inv) {
        dense_solve_kernel<T><<<1, 128, 0, ctx->stream>>>(mg->A[0].rows, tp<T>(mg->coarse_inv), B, X);
        return hb_check_launch(ctx, "dense_solve_kernel");
    }
    if (l == 0)
        return hb_launch_cg<T>(ctx, &mg->A[0], B, X, mg->prm.max_iters_coarse, (T)mg->prm.eps, tp<T>(mg->cgwork),
                               mg->cgres);
    HB_TRY(smooth<T>(mg, l, X, B, mg->prm.n_pre));
    HB_TRY(level_mode<T>(mg, l, HB_MODE_DEFECT, X, B, nullptr, tp<T>(mg->store[l])));
    if (!mg->B.empty())
        HB_TRY(hb_launch_restrict_pt<T>(ctx, mg->B[l].root, tp<T>(mg->d[l - 1]), tp<T>(mg->store[l])));
    else
        HB_TRY(hb_launch_spmv_mode<T>(ctx, &mg->res[l - 1], HB_MODE_SPMV, tp<T>(mg->store[l]), nullptr, nullptr,
                                      tp<T>(mg->d[l - 1])));
    HB_CUDA_TRY(ctx, cudaMemsetAsync(mg->c[l - 1], 0, sizeof(T) * mg->A[l - 1].rows, ctx->stream));
    HB_TRY(vcycle<T>(mg, l - 1, tp<T>(mg->c[l - 1]), tp<T>(mg->d[l - 1])));
    if (!mg->B.empty())
        HB_TRY(hb_launch_prolong_add<T>(ctx, mg->B[l].root, X, tp<T>(mg->c[l - 1])));
    else
        HB_TRY(hb_launch_spmv_mode<T>(ctx, &mg->prol[l - 1], HB_MODE_ADD, tp<T>(mg->c[l - 1]), nullptr, nullptr, X));
    return smooth<T>(mg, l, X, B, mg->prm.n_post);
}

// One cycle of mg_solve as enqueued work: the V-cycle, the finest defect and its squared norm
// into mg->norm.
template <typename T> int solve_cycle(hb_mg *mg, T *x, const T *b)
{
    const int top = mg->L - 1;
    T *r = tp<T>(mg->r);
    HB_TRY(vcycle<T>(mg, top, x, b));
    HB_TRY(level_mode<T>(mg, top, HB_MODE_DEFECT, x, b, nullptr, r));
    return hb_launch_dot<T>(mg->ctx, mg->A[top].rows, r, r, tp<T>(mg->norm));
}

// Captures solve_cycle into mg->cycle_graph on a private stream (the context's stream may be
// the legacy default stream, which cannot be captured).  Only hierarchies whose coarse solve is
// one plain launch qualify (the dense inverse, the fused tail, or the one-block CG).
template <typename T> int capture_cycle(hb_mg *mg, T *x, const T *b)
{
    hb_context *ctx = mg->ctx;
    const bool coarse_plain = mg->coarse_inv || mg->tail_level >= 0 || mg->A[0].ld / 4 <= 256;
    if (!coarse_plain || mg->graph_failed) return HB_ERR_UNSUPPORTED;
    cudaStream_t cs = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (cs) cudaStreamDestroy(cs);
        mg->graph_failed = true;
        return HB_ERR_CUDA;
    }
    cudaEventRecord(ev, ctx->stream);
    cudaStreamWaitEvent(cs, ev, 0);
    cudaStream_t saved = ctx->stream;
    const uint64_t l0 = ctx->launches;
    ctx->stream = cs;
    cudaGraph_t g = nullptr;
    int st = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess ? HB_OK : HB_ERR_CUDA;
    if (!st) st = solve_cycle<T>(mg, x, b);
    const cudaError_t e = cudaStreamEndCapture(cs, &g);
    ctx->stream = saved;
    mg->graph_kernels = ctx->launches - l0;
    ctx->launches = l0;
    if (!st && e != cudaSuccess) st = HB_ERR_CUDA;
    if (!st && cudaGraphInstantiate(&mg->cycle_graph, g, 0) != cudaSuccess) st = HB_ERR_CUDA;
    if (g) cudaGraphDestroy(g);
    cudaEventDestroy(ev);
    cudaStreamDestroy(cs);
    if (st) {
        cudaGetLastError();
        mg->cycle_graph = nullptr;
        mg->graph_failed = true;
        return st;
    }
    mg->graph_x = x;
    mg->graph_b = b;
    return HB_OK;
}

// MGSolver::value (mg.hh:1098-1126): r = b - A x; rnorm0 = |r|; cycles until |r| < eps rnorm0.
// Each cycle is one replay of the captured cycle graph where it applies (the same kernels in
// the same order, so the same iterates), then the norm's read-back for the stopping test.
template <typename T> int mg_solve(hb_mg *mg, const T *b, T *x, int64_t *used, T *rnorm)
{
    hb_context *ctx = mg->ctx;
    const int top = mg->L - 1;
    const int64_t n = mg->A[top].rows;
    T *r = tp<T>(mg->r);
    HB_TRY(level_mode<T>(mg, top, HB_MODE_DEFECT, x, b, nullptr, r));
    T r0, rc = T(1e16);
    HB_TRY(norm_host<T>(mg, r, n, &r0));
    if (mg->cycle_graph && (mg->graph_x != x || mg->graph_b != b)) drop_cycle_graph(mg);
    if (!mg->cycle_graph && mg->prm.max_iters > 1) capture_cycle<T>(mg, x, b);
    int64_t u = 0;
    for (int64_t i = 0; i < mg->prm.max_iters; ++i) {
        if (mg->cycle_graph) {
            HB_CUDA_TRY(ctx, cudaGraphLaunch(mg->cycle_graph, ctx->stream));
            ctx->launches += mg->graph_kernels;
        } else {
            HB_TRY(solve_cycle<T>(mg, x, b));
        }
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, mg->norm, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
        HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        rc = std::sqrt(*static_cast<T *>(ctx->pinned));
        u = i + 1;
        if (rc < (T)mg->prm.eps * r0) break;
    }
    hb_solve_result h;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(&h, mg->cgres, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h.status == HB_DEV_TIMEOUT) return HB_ERR_TIMEOUT;
    if (used) *used = u;
    if (rnorm) { rnorm[0] = r0; rnorm[1] = rc; }
    return HB_OK;
}

inline size_t pad_entries(int64_t n) { return (size_t)hb_round_up(n > 0 ? n : 1, 64); }

// Device dot product read back to the host (one sync).
template <typename T> int dot_host(hb_context *ctx, int64_t n, const T *x, const T *y, T *dev_slot, T *out)
{
    HB_TRY(hb_launch_dot<T>(ctx, n, x, y, dev_slot));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, dev_slot, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *out = *static_cast<T *>(ctx->pinned);
    return HB_OK;
}

}  // namespace

// Preconditioned CG in FP32 with one V-cycle from a zero start as the preconditioner (damped
// Jacobi pre/post smoothing, R = P^T, coarse CG): a symmetric positive definite preconditioner
// for SPD systems with Galerkin coarse levels.  Solves A x = b on the finest level of mg from
// x = 0 until ||r|| < eps ||b||.  work: 4 vectors of the finest size (r, z, p, v).
int hb_mg_pcg_f32(hb_mg *mg, const float *b, float *x, float eps, int64_t max_iters, float *work, int64_t *used)
{
    hb_context *ctx = mg->ctx;
    const int top = mg->L - 1;
    const hb_ell *A = &mg->A[top];
    const int64_t n = A->rows;
    const int64_t ldn = (int64_t)pad_entries(n);
    float *r = work, *z = work + ldn, *p = work + 2 * ldn, *v = work + 3 * ldn;
    float *slot = tp<float>(mg->norm);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(x, 0, sizeof(float) * n, ctx->stream));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(r, b, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    float rr;
    HB_TRY(dot_host<float>(ctx, n, r, r, slot, &rr));
    const float r0 = std::sqrt(rr);
    int64_t it = 0;
    if (r0 > 0.f && max_iters > 0) {
        HB_CUDA_TRY(ctx, cudaMemsetAsync(z, 0, sizeof(float) * n, ctx->stream));
        HB_TRY(vcycle<float>(mg, top, z, r));
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(p, z, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
        float rz;
        HB_TRY(dot_host<float>(ctx, n, r, z, slot, &rz));
        while (it < max_iters) {
            HB_TRY(hb_launch_spmv_mode<float>(ctx, A, HB_MODE_SPMV, p, nullptr, nullptr, v));
            float pv;
            HB_TRY(dot_host<float>(ctx, n, p, v, slot, &pv));
            if (!(pv > 0.f)) break;                      // breakdown (not SPD / converged to 0)
            const float a = rz / pv;
            HB_TRY(hb_scaled_sum_f32(ctx, n, x, p, a));
            HB_TRY(hb_scaled_sum_f32(ctx, n, r, v, -a));
            ++it;
            HB_TRY(dot_host<float>(ctx, n, r, r, slot, &rr));
            if (std::sqrt(rr) < eps * r0) break;
            HB_CUDA_TRY(ctx, cudaMemsetAsync(z, 0, sizeof(float) * n, ctx->stream));
            HB_TRY(vcycle<float>(mg, top, z, r));
            float rz_new;
            HB_TRY(dot_host<float>(ctx, n, r, z, slot, &rz_new));
            const float beta = rz_new / rz;
            rz = rz_new;
            HB_TRY(hb_scaled_sum3_f32(ctx, n, p, z, p, beta));   // p = beta p + z
        }
    }
    hb_solve_result h;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(&h, mg->cgres, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h.status == HB_DEV_TIMEOUT) return HB_ERR_TIMEOUT;
    if (used) *used = it;
    return HB_OK;
}

int hb_mg_view(const hb_mg *mg, hb_q1_view *out)
{
    if (!mg || !out || mg->L > HB_Q1_MAXL || mg->dtype != HB_F32) return HB_ERR_INVALID;
    for (int l = 0; l < mg->L; ++l) {
        out->jac[l] = tp<float>(mg->P[l]);
        out->c[l] = tp<float>(mg->c[l]);
        out->d[l] = tp<float>(mg->d[l]);
        out->store[l] = tp<float>(mg->store[l]);
        out->xt[l] = tp<float>(mg->xt[l]);
    }
    out->n_pre = (int)mg->prm.n_pre;
    out->n_post = (int)mg->prm.n_post;
    out->coarse_inv = tp<const float>(mg->coarse_inv);
    return HB_OK;
}

int hb_mg_finest(hb_mg *mg, hb_ell *A)
{
    *A = mg->A[mg->L - 1];
    return HB_OK;
}

int hb_mg_set_dense_coarse(hb_mg *mg, void *inv)
{
    drop_cycle_graph(mg);
    mg->coarse_inv = inv;
    return HB_OK;
}

int hb_mg_enable_tail(hb_mg *mg, int64_t max_rows)
{
    if (!mg || max_rows < 0) return HB_ERR_INVALID;
    drop_cycle_graph(mg);
    mg->tail_level = -1;
    if (max_rows == 0) return HB_OK;
    if (mg->dtype != HB_F32 || mg->B.empty() || !mg->coarse_inv) return HB_ERR_UNSUPPORTED;
    int top = -1;
    for (int l = 0; l < mg->L; ++l)
        if (mg->A[l].rows <= max_rows) top = l;
    if (top < 1) return HB_OK;   // nothing to fuse above the dense coarse solve
    if (mg->tail_desc && mg->tail_top != top) {
        cudaFreeAsync(mg->tail_desc, mg->ctx->stream);
        mg->tail_desc = nullptr;
    }
    if (!mg->tail_desc) {
        hb_q1_view v;
        HB_TRY(hb_mg_view(mg, &v));
        v.L = mg->L;
        for (int l = 0; l < mg->L; ++l) {
            v.A32[l] = mg->A[l];
            v.B32[l] = mg->B[l];
        }
        HB_TRY(hb_tail_create(mg->ctx, v, top, &mg->tail_desc));
        mg->tail_top = top;
    }
    mg->tail_level = top;
    return HB_OK;
}

// ---------------------------------------------------------------------------------------
// Device-scalar PCG: every scalar of the iteration (r.z, p.v, alpha, beta, |r|) lives in device
// memory, so one iteration is a fixed sequence of launches with no host round trip.  It is
// captured once into a CUDA graph and replayed; the host reads the done flag every few
// iterations.  After convergence the guarded updates are no-ops, so replays past the stop
// leave x unchanged.
// ---------------------------------------------------------------------------------------
struct PcgScalars {
    float rz, rz_new, pv, rr, r0, eps;
    int done, it;
};

namespace {

__global__ void pcg_start_kernel(PcgScalars *s, float eps)
{
    s->r0 = sqrtf(s->rr);
    s->eps = eps;
    s->done = !(s->r0 > 0.f);
    s->it = 0;
}

// x += alpha p; r -= alpha v with alpha = rz / pv (skipped once converged or on breakdown)
__global__ void pcg_xr_kernel(int64_t n, PcgScalars *s, float *__restrict__ x, float *__restrict__ r,
                              const float *__restrict__ p, const float *__restrict__ v)
{
    if (s->done || !(s->pv > 0.f)) return;
    const float a = s->rz / s->pv, ma = -a;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = hbd::add(x[i], hbd::mul(a, p[i]));
        r[i] = hbd::add(r[i], hbd::mul(ma, v[i]));
    }
}

__global__ void pcg_check_kernel(PcgScalars *s)
{
    if (s->done) return;
    if (!(s->pv > 0.f)) { s->done = 1; return; }
    s->it += 1;
    if (sqrtf(s->rr) < s->eps * s->r0) s->done = 1;
}

// p = beta p + z with beta = rz_new / rz; rz = rz_new (one thread finalises the scalars after
// every block has used the old rz: a second tiny kernel does it)
__global__ void pcg_p_kernel(int64_t n, const PcgScalars *s, float *__restrict__ p, const float *__restrict__ z)
{
    if (s->done) return;
    const float beta = s->rz_new / s->rz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = hbd::add(hbd::mul(beta, p[i]), z[i]);
}

__global__ void pcg_roll_kernel(PcgScalars *s)
{
    if (!s->done) s->rz = s->rz_new;
}

inline unsigned ewb(hb_context *ctx, int64_t n)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8));
}

// One PCG iteration: v = A p; pv = p.v; x, r update; rr = r.r; check; z = M(r); rz_new = r.z;
// p = beta p + z; rz = rz_new.
int pcg_iteration(hb_mg *mg, float *x, float *r, float *z, float *p, float *v, PcgScalars *s)
{
    hb_context *ctx = mg->ctx;
    const hb_ell *A = &mg->A[mg->L - 1];
    const int64_t n = A->rows;
    HB_TRY(level_mode<float>(mg, mg->L - 1, HB_MODE_SPMV, p, nullptr, nullptr, v));
    HB_TRY(hb_launch_dot<float>(ctx, n, p, v, &s->pv));
    pcg_xr_kernel<<<ewb(ctx, n), 256, 0, ctx->stream>>>(n, s, x, r, p, v);
    HB_TRY(hb_check_launch(ctx, "pcg_xr_kernel"));
    HB_TRY(hb_launch_dot<float>(ctx, n, r, r, &s->rr));
    pcg_check_kernel<<<1, 1, 0, ctx->stream>>>(s);
    HB_TRY(hb_check_launch(ctx, "pcg_check_kernel"));
    HB_CUDA_TRY(ctx, cudaMemsetAsync(z, 0, sizeof(float) * n, ctx->stream));
    HB_TRY(vcycle<float>(mg, mg->L - 1, z, r));
    HB_TRY(hb_launch_dot<float>(ctx, n, r, z, &s->rz_new));
    pcg_p_kernel<<<ewb(ctx, n), 256, 0, ctx->stream>>>(n, s, p, z);
    HB_TRY(hb_check_launch(ctx, "pcg_p_kernel"));
    pcg_roll_kernel<<<1, 1, 0, ctx->stream>>>(s);
    return hb_check_launch(ctx, "pcg_roll_kernel");
}

}  // namespace

// PCG on the finest level of an FP32 hierarchy with device scalars.  work: 4 padded vectors
// (r, z, p, v) + one PcgScalars slot (16 floats).  graph (optional, in/out): a captured
// iteration for this (mg, work, x) triple, reused across calls.  check_every: iterations per
// host check of the done flag.
int hb_mg_pcg_f32_graph(hb_mg *mg, cudaStream_t capture_stream, const float *b, float *x, float eps, int64_t max_iters,
                        float *work, cudaGraphExec_t *graph, int check_every, int64_t *used)
{
    hb_context *ctx = mg->ctx;
    const int top = mg->L - 1;
    const int64_t n = mg->A[top].rows;
    const int64_t ldn = (int64_t)pad_entries(n);
    float *r = work, *z = work + ldn, *p = work + 2 * ldn, *v = work + 3 * ldn;
    PcgScalars *s = reinterpret_cast<PcgScalars *>(work + 4 * ldn);
    // start: x = 0, r = b, rr = r.r, z = M(r), p = z, rz = r.z
    HB_CUDA_TRY(ctx, cudaMemsetAsync(x, 0, sizeof(float) * n, ctx->stream));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(r, b, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    HB_TRY(hb_launch_dot<float>(ctx, n, r, r, &s->rr));
    pcg_start_kernel<<<1, 1, 0, ctx->stream>>>(s, eps);
    HB_TRY(hb_check_launch(ctx, "pcg_start_kernel"));
    HB_CUDA_TRY(ctx, cudaMemsetAsync(z, 0, sizeof(float) * n, ctx->stream));
    HB_TRY(vcycle<float>(mg, top, z, r));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(p, z, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    HB_TRY(hb_launch_dot<float>(ctx, n, r, z, &s->rz));
    if (graph && !*graph && capture_stream) {
        // capture one iteration on the capture stream (ordered after the start work)
        cudaEvent_t ev;
        HB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaStream_t saved = ctx->stream;
        cudaEventRecord(ev, saved);
        cudaStreamWaitEvent(capture_stream, ev, 0);
        cudaEventDestroy(ev);
        ctx->stream = capture_stream;
        cudaGraph_t g = nullptr;
        int st = HB_OK;
        if (cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) st = HB_ERR_CUDA;
        if (!st) st = pcg_iteration(mg, x, r, z, p, v, s);
        cudaError_t e = cudaStreamEndCapture(capture_stream, &g);
        if (!st && e != cudaSuccess) st = HB_ERR_CUDA;
        ctx->stream = saved;
        if (!st && cudaGraphInstantiate(graph, g, 0) != cudaSuccess) st = HB_ERR_CUDA;
        if (g) cudaGraphDestroy(g);
        if (st) { cudaGetLastError(); *graph = nullptr; return st; }
    }
    PcgScalars *h = static_cast<PcgScalars *>(ctx->pinned);
    int64_t launched = 0;
    const int every = std::max(1, check_every);
    while (launched < max_iters) {
        const int64_t k = std::min<int64_t>(every, max_iters - launched);
        for (int64_t i = 0; i < k; ++i) {
            if (graph && *graph) {
                HB_CUDA_TRY(ctx, cudaGraphLaunch(*graph, ctx->stream));
            } else {
                HB_TRY(pcg_iteration(mg, x, r, z, p, v, s));
            }
        }
        launched += k;
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, ctx->stream));
        HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        if (h->done) break;
    }
    if (used) *used = h->it;
    return HB_OK;
}

namespace {

// One V-cycle on the finest level (the OperatorList that MGCycleCreation<V::STATIC> builds,
// honei/math/mg.hh:567-662, run once): asynchronous on the context stream.
template <typename T> int mg_cycle(hb_mg *mg, const T *b, T *x)
{
    if (!b || !x) return HB_ERR_INVALID;
    if (mg->dtype != (sizeof(T) == 8 ? HB_F64 : HB_F32)) return HB_ERR_INVALID;
    return vcycle<T>(mg, mg->L - 1, x, b);
}

template <typename T> int jacobi_init(hb_mg *mg)
{
    for (int l = 0; l < mg->L; ++l)
        HB_TRY(hb_launch_jacobi_diag<T>(mg->ctx, &mg->A[l], (T)mg->prm.damping, tp<T>(mg->P[l])));
    return HB_OK;
}

int mg_create_impl(hb_context *ctx, int nlevels, const hb_ell *A, const hb_ell *prol, const hb_ell *res,
                   const hb_q1band *B, const hb_mg_params *params, hb_mg **out)
{
    if (!ctx || !A || !params || !out || nlevels < 1) return HB_ERR_INVALID;
    if (nlevels > 1 && !B && (!prol || !res)) return HB_ERR_INVALID;
    *out = nullptr;
    const int dt = A[0].dtype;
    if (B) {
        // square grids, each coarse side = (finer side) / 2 + 1, bands of the level's own size
        for (int l = 0; l < nlevels; ++l) {
            const int64_t m = B[l].root;
            if (B[l].dtype != dt || B[l].n != A[l].rows || m * m != B[l].n) return HB_ERR_SIZE;
            if (l > 0 && B[l - 1].root != m / 2 + 1) return HB_ERR_SIZE;
            for (int k = 0; k < 9; ++k)
                if (!B[l].band[k]) return HB_ERR_INVALID;
        }
    }
    for (int l = 0; l < nlevels; ++l) {
        HB_TRY(hb_check_ell(&A[l], dt));
        if (A[l].rows != A[l].cols) return HB_ERR_SIZE;
        if (l + 1 < nlevels && !B) {
            HB_TRY(hb_check_ell(&prol[l], dt));
            HB_TRY(hb_check_ell(&res[l], dt));
            if (prol[l].rows != A[l + 1].rows || prol[l].cols != A[l].rows) return HB_ERR_SIZE;
            if (res[l].rows != A[l].rows || res[l].cols != A[l + 1].rows) return HB_ERR_SIZE;
        }
    }
    if (params->max_iters < 0 || params->max_iters_coarse < 0 || params->n_pre < 0 || params->n_post < 0)
        return HB_ERR_INVALID;
    hb_mg *mg = new hb_mg();
    mg->ctx = ctx;
    mg->L = nlevels;
    mg->dtype = dt;
    mg->A.assign(A, A + nlevels);
    if (nlevels > 1 && !B) {
        mg->prol.assign(prol, prol + nlevels - 1);
        mg->res.assign(res, res + nlevels - 1);
    }
    if (B) mg->B.assign(B, B + nlevels);
    mg->prm = *params;
    const size_t es = dt == HB_F64 ? 8 : 4;
    const int64_t nf = A[nlevels - 1].rows;
    size_t entries = 0;
    for (int l = 0; l < nlevels; ++l) entries += 5 * pad_entries(A[l].rows);
    entries += pad_entries(nf);                        // r
    entries += 5 * pad_entries(A[0].ld);               // coarse CG work
    entries += 64;                                     // norm scalar
    size_t bytes = entries * es + 256 /* cg result */;
    if (dt == HB_F32) bytes += pad_entries(nf) * (8 + 4 + 4);   // IR: r64, b32, x32
    if (cudaMallocAsync(&mg->mem, bytes, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        delete mg;
        return HB_ERR_ALLOC;
    }
    char *p = (char *)mg->mem;
    auto take = [&](size_t n_entries, size_t esz) { void *q = p; p += n_entries * esz; return q; };
    mg->cgres = (hb_solve_result *)take(256, 1);
    for (int l = 0; l < nlevels; ++l) {
        const size_t n = pad_entries(A[l].rows);
        mg->P.push_back(take(n, es));
        mg->d.push_back(take(n, es));
        mg->c.push_back(take(n, es));
        mg->store.push_back(take(n, es));
        mg->xt.push_back(take(n, es));
    }
    mg->r = take(pad_entries(nf), es);
    mg->cgwork = take(5 * pad_entries(A[0].ld), es);
    mg->norm = take(64, es);
    if (dt == HB_F32) {
        mg->ir_r = (double *)take(pad_entries(nf), 8);
        mg->ir_b = (float *)take(pad_entries(nf), 4);
        mg->ir_x = (float *)take(pad_entries(nf), 4);
    }
    int st = cudaMemsetAsync(mg->mem, 0, bytes, ctx->stream) == cudaSuccess ? HB_OK : HB_ERR_CUDA;
    if (!st) st = dt == HB_F64 ? jacobi_init<double>(mg) : jacobi_init<float>(mg);
    if (st) {
        cudaFreeAsync(mg->mem, ctx->stream);
        delete mg;
        return st;
    }
    *out = mg;
    return HB_OK;
}

}  // namespace

extern "C" {

int hb_mg_create(hb_context *ctx, int nlevels, const hb_ell *A, const hb_ell *prol, const hb_ell *res,
                 const hb_mg_params *params, hb_mg **out)
{
    HB_RANGE("hb_mg_create");
    return mg_create_impl(ctx, nlevels, A, prol, res, nullptr, params, out);
}

int hb_mg_create_banded(hb_context *ctx, int nlevels, const hb_ell *A, const hb_q1band *B, const hb_mg_params *params,
                        hb_mg **out)
{
    HB_RANGE("hb_mg_create_banded");
    if (!B) return HB_ERR_INVALID;
    return mg_create_impl(ctx, nlevels, A, nullptr, nullptr, B, params, out);
}

int hb_mg_destroy(hb_mg *mg)
{
    if (!mg) return HB_ERR_INVALID;
    drop_cycle_graph(mg);
    // stream-ordered: the memory returns to the pool once the stream's queued work is done
    if (mg->tail_desc) cudaFreeAsync(mg->tail_desc, mg->ctx->stream);
    cudaFreeAsync(mg->mem, mg->ctx->stream);
    delete mg;
    return HB_OK;
}

int hb_mg_set_params(hb_mg *mg, const hb_mg_params *params)
{
    if (!mg || !params) return HB_ERR_INVALID;
    if (params->max_iters < 0 || params->max_iters_coarse < 0 || params->n_pre < 0 || params->n_post < 0)
        return HB_ERR_INVALID;
    const bool redo = params->damping != mg->prm.damping;
    drop_cycle_graph(mg);
    mg->prm = *params;
    if (redo) return mg->dtype == HB_F64 ? jacobi_init<double>(mg) : jacobi_init<float>(mg);
    return HB_OK;
}

int hb_mg_solve_f64(hb_mg *mg, const double *b, double *x, int64_t *used_cycles, double *rnorm_host)
{
    HB_RANGE("hb_mg_solve_f64");
    if (!mg || !b || !x) return HB_ERR_INVALID;
    if (mg->dtype != HB_F64) return HB_ERR_INVALID;
    return mg_solve<double>(mg, b, x, used_cycles, rnorm_host);
}

int hb_mg_solve_f32(hb_mg *mg, const float *b, float *x, int64_t *used_cycles, float *rnorm_host)
{
    HB_RANGE("hb_mg_solve_f32");
    if (!mg || !b || !x) return HB_ERR_INVALID;
    if (mg->dtype != HB_F32) return HB_ERR_INVALID;
    return mg_solve<float>(mg, b, x, used_cycles, rnorm_host);
}

int hb_mg_cycle_f64(hb_mg *mg, const double *b, double *x)
{
    HB_RANGE("hb_mg_cycle_f64");
    if (!mg) return HB_ERR_INVALID;
    return mg_cycle<double>(mg, b, x);
}

int hb_mg_cycle_f32(hb_mg *mg, const float *b, float *x)
{
    HB_RANGE("hb_mg_cycle_f32");
    if (!mg) return HB_ERR_INVALID;
    return mg_cycle<float>(mg, b, x);
}

int hb_mg_set_smoother(hb_mg *mg, int level, const void *P)
{
    if (!mg || !P || level < 0 || level >= mg->L) return HB_ERR_INVALID;
    const size_t es = mg->dtype == HB_F64 ? 8 : 4;
    HB_CUDA_TRY(mg->ctx, cudaMemcpyAsync(mg->P[level], P, es * mg->A[level].rows, cudaMemcpyDeviceToDevice,
                                         mg->ctx->stream));
    return HB_OK;
}

// IRSolver<double outer, float inner, Norm<l2, true>> (honei/math/ir.hh:30-78).
int hb_ir_mg_solve(hb_context *ctx, const hb_ell *A64, hb_mg *mg32, const double *b, double *x, double eps,
                   int64_t max_iters, int warm_start, int64_t *used_outer, double *rnorm_host)
{
    HB_RANGE("hb_ir_mg_solve");
    if (!ctx || !A64 || !mg32 || !b || !x || max_iters < 0) return HB_ERR_INVALID;
    HB_TRY(hb_check_ell(A64, HB_F64));
    if (mg32->dtype != HB_F32) return HB_ERR_INVALID;
    const int64_t n = A64->rows;
    if (A64->cols != n || mg32->A[mg32->L - 1].rows != n) return HB_ERR_SIZE;
    hb_context *saved = mg32->ctx;
    mg32->ctx = ctx;
    double r0 = 1e16, rc = 1e16;
    int64_t u = 0;
    int st = HB_OK;
    for (int64_t i = 0; i < max_iters && !st; ++i) {
        st = hb_launch_spmv_mode<double>(ctx, A64, HB_MODE_DEFECT, x, b, nullptr, mg32->ir_r);
        if (st) break;
        double nrm;
        st = hb_launch_dot<double>(ctx, n, mg32->ir_r, mg32->ir_r, (double *)hb_scalars(ctx) + 16);
        if (st) break;
        if (cudaMemcpyAsync(ctx->pinned, (double *)hb_scalars(ctx) + 16, 8, cudaMemcpyDeviceToHost, ctx->stream) ||
            cudaStreamSynchronize(ctx->stream)) { st = HB_ERR_CUDA; break; }
        nrm = std::sqrt(*(double *)ctx->pinned);
        if (i == 0) {
            r0 = nrm;
        } else {
            rc = nrm;
            u = i;
            if (rc < eps * r0) break;
        }
        if (warm_start) {
            st = launch_f64_to_f32(ctx, n, mg32->ir_b, mg32->ir_r);
        } else {
            st = launch_f64_to_f32_scaled(ctx, n, mg32->ir_b, mg32->ir_r, 1.0 / nrm);
            if (!st && cudaMemsetAsync(mg32->ir_x, 0, sizeof(float) * n, ctx->stream)) st = HB_ERR_CUDA;
        }
        if (st) break;
        st = mg_solve<float>(mg32, mg32->ir_b, mg32->ir_x, nullptr, nullptr);
        if (st) break;
        st = warm_start ? launch_add_f32_to_f64(ctx, n, x, mg32->ir_x)
                        : launch_add_scaled_f32_to_f64(ctx, n, x, mg32->ir_x, nrm);
    }
    mg32->ctx = saved;
    if (st) return st;
    if (used_outer) *used_outer = u;
    if (rnorm_host) { rnorm_host[0] = r0; rnorm_host[1] = rc; }
    return HB_OK;
}

// The same outer loop around an FP32 CG inner solve that restarts from zero each step.
int hb_ir_cg_solve(hb_context *ctx, const hb_ell *A64, const hb_ell *A32, const double *b, double *x, double eps,
                   float inner_eps, int64_t inner_max_iters, int64_t max_iters, int64_t *used_outer,
                   int64_t *inner_total, double *rnorm_host)
{
    HB_RANGE("hb_ir_cg_solve");
    if (!ctx || !A64 || !A32 || !b || !x || max_iters < 0 || inner_max_iters < 0) return HB_ERR_INVALID;
    HB_TRY(hb_check_ell(A64, HB_F64));
    HB_TRY(hb_check_ell(A32, HB_F32));
    const int64_t n = A64->rows;
    if (A64->cols != n || A32->rows != n || A32->cols != n) return HB_ERR_SIZE;
    const int64_t ld = A64->ld;
    // work: CG (5 ld floats) | r64 (ld doubles) | b32 | x32 (ld floats)
    HB_TRY(hb_ensure_work(ctx, (size_t)ld * (5 * 4 + 8 + 4 + 4)));
    float *cgw = (float *)ctx->work;
    double *r64 = (double *)(cgw + 5 * ld);
    float *b32 = (float *)(r64 + ld);
    float *x32 = b32 + ld;
    double r0 = 1e16, rc = 1e16, *dnorm = (double *)hb_scalars(ctx) + 16;
    int64_t u = 0, total = 0;
    hb_solve_result *res = hb_result(ctx) + 1;
    for (int64_t i = 0; i < max_iters; ++i) {
        HB_TRY(hb_launch_spmv_mode<double>(ctx, A64, HB_MODE_DEFECT, x, b, nullptr, r64));
        HB_TRY(hb_launch_dot<double>(ctx, n, r64, r64, dnorm));
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, dnorm, 8, cudaMemcpyDeviceToHost, ctx->stream));
        HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        if (i > 0) {
            hb_solve_result *h = (hb_solve_result *)((char *)ctx->pinned + 64);
            HB_CUDA_TRY(ctx, cudaMemcpy(h, res, sizeof(*h), cudaMemcpyDeviceToHost));
            if (h->status == HB_DEV_TIMEOUT) return HB_ERR_TIMEOUT;
            total += h->used;
        }
        const double nrm = std::sqrt(*(double *)ctx->pinned);
        if (i == 0) {
            r0 = nrm;
        } else {
            rc = nrm;
            u = i;
            if (rc < eps * r0) break;
        }
        // normalised defect: the inner CG's absolute stopping test (cg.hh:118) then means
        // "relative to this step's defect" and cannot end the inner solve early
        HB_TRY(launch_f64_to_f32_scaled(ctx, n, b32, r64, 1.0 / nrm));
        HB_CUDA_TRY(ctx, cudaMemsetAsync(x32, 0, sizeof(float) * n, ctx->stream));
        HB_TRY(hb_launch_cg<float>(ctx, A32, b32, x32, inner_max_iters, inner_eps, cgw, res));
        HB_TRY(launch_add_scaled_f32_to_f64(ctx, n, x, x32, nrm));
    }
    if (used_outer) *used_outer = u;
    if (inner_total) *inner_total = total;
    if (rnorm_host) { rnorm_host[0] = r0; rnorm_host[1] = rc; }
    return HB_OK;
}

}  // extern "C"
