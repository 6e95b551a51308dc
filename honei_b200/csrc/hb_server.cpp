// hb_server.cpp -- the request loop: admission by HBM budget, device-resident request state,
// concurrent service on several streams (continuous batching).
//
// Threads:
//   admitter        takes submitted requests in FIFO order and admits each once its estimated
//                   resident bytes fit the budget (head-of-line order is kept: no overtaking),
//                   routing small grids to the batch queue and large ones to the MG-PCG queue;
//   small workers   each owns a context + stream; takes every admitted small request waiting
//                   (up to max_batch), builds them on the device and solves them in one batched
//                   cluster launch (HB_BATCH_IR32);
//   large workers   each owns a context + stream; builds the request's hb_q1 (device-assembled
//                   matrix + Galerkin hierarchy) and runs the mixed-precision MG-PCG solve;
//   plain worker    (HB_SERVE_PLAIN_CG64) one request at a time with hb_cg_f64;
//   plain batched   (HB_SERVE_PLAIN_CG64_BATCHED) the baseline with the mixed server's
//                   concurrency: grids up to mid_max_side in batched HB_BATCH_CG64 cluster
//                   launches, larger ones on large_workers concurrent hb_cg_f64 workers.
// Requests that arrive while others are on the GPU are admitted as soon as memory frees up, and
// their work overlaps with the in-flight work on the other streams.  All device memory of a
// request is stream-ordered (cudaMallocAsync / cudaFreeAsync), so nothing synchronises the
// device.  No reference counterpart: HONEI solves one system per call on the caller's thread.
#include "hb_internal.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct Item {
    hb_request r;
    double t_submit = 0, t_admit = 0;
    int64_t bytes = 0;
    int path = 0;
};

// Device bytes a request of side M holds while resident on a path: a fixed 1 MiB (launch
// workspaces, descriptors, pool granularity) plus a per-row charge 15-25 % above what the
// stream-ordered pool was measured to hold per row on a B200 (one request at a time, sides 33 to
// 1025): batched FP32-inner refinement 204-215 B (FP64 + FP32 matrix values, int32 columns,
// coefficients, b, x, the batch work vectors); the MG-preconditioned paths 414-428 B (the
// device-built Galerkin hierarchy in FP64 and FP32, its banded copies and the refinement and PCG
// vectors); plain CG 140-146 B; batched plain CG 172-181 B.
int64_t estimate_bytes(int path, int64_t M)
{
    const int64_t n = M * M;
    int64_t per_row = 256;
    if (path == HB_PATH_MGPCG || path == HB_PATH_MGBATCH) per_row = 512;
    else if (path == HB_PATH_CG64) per_row = 176;
    else if (path == HB_PATH_BATCH_CG64) per_row = 224;
    return (int64_t(1) << 20) + per_row * n;
}

}  // namespace

struct hb_server;
static int route(const hb_server *s, int64_t M);

struct hb_server {
    hb_server_params p{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_pending, cv_work, cv_mem, cv_done;
    std::deque<Item *> pending, small_q, mid_q, large_q;
    std::vector<hb_completion> done;
    int64_t in_use = 0, peak = 0, submitted = 0, completed = 0;
    bool stop = false;
    std::thread admitter;
    std::vector<std::thread> workers;
    cudaMemPool_t pool = nullptr;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    void complete(Item *it, const hb_completion &c)
    {
        std::lock_guard<std::mutex> l(mu);
        done.push_back(c);
        in_use -= it->bytes;
        ++completed;
        delete it;
        cv_mem.notify_all();
        cv_done.notify_all();
    }

    void fail(Item *it, int status)
    {
        hb_completion c{};
        c.tag = it->r.tag;
        c.status = status;
        c.path = it->path;
        c.t_submit = it->t_submit;
        c.t_admit = it->t_admit;
        c.t_done = now();
        c.bytes = it->bytes;
        complete(it, c);
    }
};

namespace {

struct Worker {
    hb_context *ctx = nullptr;
    cudaStream_t stream = nullptr;
    int init(int device)
    {
        int st = hb_create(&ctx, device);
        if (st) return st;
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return HB_ERR_CUDA;
        }
        return hb_set_stream(ctx, stream);
    }
    ~Worker()
    {
        if (stream) cudaStreamSynchronize(stream);
        if (ctx) hb_destroy(ctx);
        if (stream) cudaStreamDestroy(stream);
    }
};

// Device copies of one request's inputs and the SPD matrix in hb_ell layout.
struct DeviceSystem {
    hb_context *ctx;
    std::vector<void *> blocks;
    hb_ell A64{}, A32{};
    double *b = nullptr, *x = nullptr, *coef = nullptr;

    int alloc(void **p, size_t bytes)
    {
        if (cudaMallocAsync(p, bytes ? bytes : 256, ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            return HB_ERR_ALLOC;
        }
        blocks.push_back(*p);
        return HB_OK;
    }
    void release()
    {
        for (void *p : blocks) cudaFreeAsync(p, ctx->stream);
        blocks.clear();
    }
    // coefficient upload; optional matrix assembly (batched and plain paths)
    int inputs(const hb_request &r, bool assemble, bool with_f32)
    {
        const int64_t M = r.M, n = M * M;
        void *p;
        int st;
        if (r.coef && M > 1) {
            if ((st = alloc(&p, (size_t)(M - 1) * (M - 1) * 8))) return st;
            coef = (double *)p;
            HB_CUDA_TRY(ctx, cudaMemcpyAsync(coef, r.coef, (size_t)(M - 1) * (M - 1) * 8, cudaMemcpyHostToDevice,
                                             ctx->stream));
        }
        if ((st = alloc(&p, (size_t)n * 8))) return st;
        b = (double *)p;
        if ((st = alloc(&p, (size_t)n * 8))) return st;
        x = (double *)p;
        if (!assemble) return HB_OK;
        int64_t K, ld;
        hb_ell_layout(n, 9, 1, &K, &ld);
        A64 = hb_ell{n, n, K, ld, nullptr, nullptr, HB_F64, 0};
        if ((st = alloc(&p, (size_t)K * ld * 4))) return st;
        A64.Aj = (int32_t *)p;
        if ((st = alloc(&p, (size_t)K * ld * 8))) return st;
        A64.Ax = p;
        if ((st = hb_q1_assemble_f64(ctx, M, coef, 1, &A64))) return st;
        if (with_f32) {
            A32 = A64;
            A32.dtype = HB_F32;
            if ((st = alloc(&p, (size_t)K * ld * 4))) return st;
            A32.Ax = p;
            if ((st = hb_ell_cast_f64_f32(ctx, &A64, &A32))) return st;
        }
        return HB_OK;
    }
    // b from the request, or b = A x_true
    int rhs(const hb_request &r, const hb_ell &A)
    {
        const int64_t n = r.M * r.M;
        if (r.b) {
            HB_CUDA_TRY(ctx, cudaMemcpyAsync(b, r.b, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream));
            return HB_OK;
        }
        if (!r.x_true) return HB_ERR_INVALID;
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(x, r.x_true, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream));
        return hb_spmv_f64(ctx, &A, x, b);
    }
};

// ||b - A x|| / ||b|| (FP64, on the device) into *rel.
int true_relres(hb_context *ctx, const hb_ell &A, const double *b, const double *x, double *tmp, double *rel)
{
    const int64_t n = A.rows;
    int st = hb_defect_f64(ctx, &A, b, x, tmp);
    double rr = 0, bb = 0;
    if (!st) st = hb_norm_l2_f64(ctx, n, tmp, 1, &rr);
    if (!st) st = hb_norm_l2_f64(ctx, n, b, 1, &bb);
    if (!st) *rel = bb > 0 ? rr / bb : rr;
    return st;
}

}  // namespace

// The path a request of side M takes on this server.
static int route(const hb_server *s, int64_t M)
{
    if (s->p.mode == HB_SERVE_PLAIN_CG64) return HB_PATH_CG64;
    if (s->p.mode == HB_SERVE_PLAIN_CG64_BATCHED) return M <= s->p.mid_max_side ? HB_PATH_BATCH_CG64 : HB_PATH_CG64;
    if (M <= s->p.small_max_side) return HB_PATH_BATCH;
    if (M <= s->p.mid_max_side) return HB_PATH_MGBATCH;
    return HB_PATH_MGPCG;
}

namespace {

void admit_loop(hb_server *s)
{
    std::unique_lock<std::mutex> l(s->mu);
    while (true) {
        s->cv_pending.wait(l, [&] { return s->stop || !s->pending.empty(); });
        if (s->stop) return;
        Item *it = s->pending.front();
        // FIFO admission: wait until the head fits (or nothing else is resident)
        s->cv_mem.wait(l, [&] { return s->stop || s->in_use == 0 || s->in_use + it->bytes <= s->p.hbm_budget_bytes; });
        if (s->stop) return;
        s->pending.pop_front();
        s->in_use += it->bytes;
        s->peak = std::max(s->peak, s->in_use);
        it->t_admit = s->now();
        if (it->path == HB_PATH_BATCH || it->path == HB_PATH_BATCH_CG64) s->small_q.push_back(it);
        else if (it->path == HB_PATH_MGBATCH) s->mid_q.push_back(it);
        else s->large_q.push_back(it);
        s->cv_work.notify_all();
    }
}

void large_loop(hb_server *s)
{
    Worker w;
    const int init = w.init(s->p.device);
    while (true) {
        Item *it;
        {
            std::unique_lock<std::mutex> l(s->mu);
            s->cv_work.wait(l, [&] { return s->stop || !s->large_q.empty(); });
            if (s->stop && s->large_q.empty()) return;
            it = s->large_q.front();
            s->large_q.pop_front();
        }
        if (init) { s->fail(it, init); continue; }
        const hb_request &r = it->r;
        const int64_t n = r.M * r.M;
        DeviceSystem ds{w.ctx};
        hb_completion c{};
        c.tag = r.tag;
        c.path = it->path;
        c.t_submit = it->t_submit;
        c.t_admit = it->t_admit;
        c.bytes = it->bytes;
        int st;
        double *tmp = nullptr;
        if (it->path == HB_PATH_CG64) {
            st = ds.inputs(r, true, false);
            if (!st) st = ds.rhs(r, ds.A64);
            if (!st && cudaMemsetAsync(ds.x, 0, n * 8, w.stream) != cudaSuccess) st = HB_ERR_CUDA;
            int64_t used = 0;
            if (!st) st = hb_cg_f64(w.ctx, &ds.A64, ds.b, ds.x, 1000000, s->p.eps, &used, nullptr);
            c.iterations = used;
            if (!st) st = ds.alloc((void **)&tmp, n * 8);
            if (!st) st = true_relres(w.ctx, ds.A64, ds.b, ds.x, tmp, &c.true_relres);
        } else {
            hb_q1 *q = nullptr;
            st = ds.inputs(r, false, false);
            if (!st) st = hb_q1_create(w.ctx, r.M, ds.coef, &q);
            hb_ell A{};
            if (!st) {
                int nl = 0;
                hb_q1_levels(q, &nl, nullptr);
                st = hb_q1_level(q, nl - 1, &A, nullptr, nullptr, nullptr);
            }
            if (!st) st = ds.rhs(r, A);
            if (!st && cudaMemsetAsync(ds.x, 0, n * 8, w.stream) != cudaSuccess) st = HB_ERR_CUDA;
            hb_batch_result info{};
            if (!st) st = hb_q1_solve(q, ds.b, ds.x, s->p.eps, s->p.inner_eps, 50, 2000, &info);
            c.iterations = info.iterations;
            c.outer = info.outer;
            c.true_relres = info.true_relres;
            if (q) hb_q1_destroy(q);
        }
        if (!st && cudaMemcpyAsync(r.x, ds.x, n * 8, cudaMemcpyDeviceToHost, w.stream) != cudaSuccess) st = HB_ERR_CUDA;
        ds.release();
        if (cudaStreamSynchronize(w.stream) != cudaSuccess && !st) st = HB_ERR_CUDA;
        cudaGetLastError();
        c.status = st;
        c.t_done = s->now();
        s->complete(it, c);
    }
}

void small_loop(hb_server *s)
{
    Worker w;
    const int init = w.init(s->p.device);
    while (true) {
        std::vector<Item *> batch;
        {
            std::unique_lock<std::mutex> l(s->mu);
            s->cv_work.wait(l, [&] { return s->stop || !s->small_q.empty(); });
            if (s->stop && s->small_q.empty()) return;
            while (!s->small_q.empty() && (int)batch.size() < std::max(1, s->p.max_batch)) {
                batch.push_back(s->small_q.front());
                s->small_q.pop_front();
            }
        }
        if (init) {
            for (Item *it : batch) s->fail(it, init);
            continue;
        }
        const int64_t count = (int64_t)batch.size();
        const bool plain = s->p.mode == HB_SERVE_PLAIN_CG64_BATCHED;
        std::vector<DeviceSystem> ds(count, DeviceSystem{w.ctx});
        std::vector<hb_batch_system> sys(count);
        std::vector<int> st(count, HB_OK);
        for (int64_t i = 0; i < count; ++i) {
            const hb_request &r = batch[i]->r;
            st[i] = ds[i].inputs(r, true, !plain);
            if (!st[i]) st[i] = ds[i].rhs(r, ds[i].A64);
            if (!st[i] && cudaMemsetAsync(ds[i].x, 0, r.M * r.M * 8, w.stream) != cudaSuccess) st[i] = HB_ERR_CUDA;
            hb_batch_system &b = sys[i];
            b = hb_batch_system{};
            b.A64 = ds[i].A64;
            b.A32 = ds[i].A32;
            b.b = ds[i].b;
            b.x = ds[i].x;
            b.mode = plain ? HB_BATCH_CG64 : HB_BATCH_IR32;
            b.max_iters = 1000000;
            b.max_outer = 50;
            b.eps = s->p.eps;
            b.inner_eps = s->p.inner_eps;
        }
        // drop failed set-ups from the launch
        std::vector<int64_t> live;
        std::vector<hb_batch_system> lsys;
        for (int64_t i = 0; i < count; ++i)
            if (!st[i]) { live.push_back(i); lsys.push_back(sys[i]); }
        std::vector<hb_batch_result> res(lsys.size());
        int bst = HB_OK;
        void *ws = nullptr;
        if (!lsys.empty()) {
            size_t bytes = 0;
            bst = hb_batch_workspace_bytes(lsys.data(), (int64_t)lsys.size(), &bytes);
            if (!bst && cudaMallocAsync(&ws, bytes, w.stream) != cudaSuccess) { cudaGetLastError(); bst = HB_ERR_ALLOC; }
            if (!bst) bst = hb_batch_solve(w.ctx, lsys.data(), (int64_t)lsys.size(), ws, &s->p.batch_cfg, res.data());
            if (ws) cudaFreeAsync(ws, w.stream);
        }
        for (size_t k = 0; k < live.size(); ++k) {
            const int64_t i = live[k];
            if (bst) { st[i] = bst; continue; }
            const hb_request &r = batch[i]->r;
            if (cudaMemcpyAsync(r.x, ds[i].x, r.M * r.M * 8, cudaMemcpyDeviceToHost, w.stream) != cudaSuccess)
                st[i] = HB_ERR_CUDA;
        }
        for (auto &d : ds) d.release();
        if (cudaStreamSynchronize(w.stream) != cudaSuccess) cudaGetLastError();
        const double t = s->now();
        size_t k = 0;
        for (int64_t i = 0; i < count; ++i) {
            hb_completion c{};
            c.tag = batch[i]->r.tag;
            c.path = plain ? HB_PATH_BATCH_CG64 : HB_PATH_BATCH;
            c.t_submit = batch[i]->t_submit;
            c.t_admit = batch[i]->t_admit;
            c.bytes = batch[i]->bytes;
            c.t_done = t;
            c.status = st[i];
            if (k < live.size() && live[k] == i) {
                if (!st[i]) {
                    c.iterations = res[k].iterations;
                    c.outer = res[k].outer;
                    c.true_relres = res[k].true_relres;
                    c.status = res[k].status;
                }
                ++k;
            }
            s->complete(batch[i], c);
        }
    }
}

// Mid-size grids: every waiting request (up to max_batch) gets its hb_q1 (device-built
// hierarchy) and all of them are solved in one batched MG-PCG cluster launch.
void mid_loop(hb_server *s)
{
    Worker w;
    const int init = w.init(s->p.device);
    while (true) {
        std::vector<Item *> batch;
        {
            std::unique_lock<std::mutex> l(s->mu);
            s->cv_work.wait(l, [&] { return s->stop || !s->mid_q.empty(); });
            if (s->stop && s->mid_q.empty()) return;
            while (!s->mid_q.empty() && (int)batch.size() < std::max(1, s->p.max_batch)) {
                batch.push_back(s->mid_q.front());
                s->mid_q.pop_front();
            }
        }
        if (init) {
            for (Item *it : batch) s->fail(it, init);
            continue;
        }
        const int64_t count = (int64_t)batch.size();
        std::vector<DeviceSystem> ds(count, DeviceSystem{w.ctx});
        std::vector<hb_q1 *> qs(count, nullptr);
        std::vector<int> st(count, HB_OK);
        for (int64_t i = 0; i < count; ++i) {
            const hb_request &r = batch[i]->r;
            st[i] = ds[i].inputs(r, false, false);
            if (!st[i]) st[i] = hb_q1_create(w.ctx, r.M, ds[i].coef, &qs[i]);
            hb_ell A{};
            if (!st[i]) {
                int nl = 0;
                hb_q1_levels(qs[i], &nl, nullptr);
                st[i] = hb_q1_level(qs[i], nl - 1, &A, nullptr, nullptr, nullptr);
            }
            if (!st[i]) st[i] = ds[i].rhs(r, A);
            if (!st[i] && cudaMemsetAsync(ds[i].x, 0, r.M * r.M * 8, w.stream) != cudaSuccess) st[i] = HB_ERR_CUDA;
        }
        std::vector<int64_t> live;
        std::vector<hb_q1 *> lq;
        std::vector<const double *> lb;
        std::vector<double *> lx;
        for (int64_t i = 0; i < count; ++i)
            if (!st[i]) { live.push_back(i); lq.push_back(qs[i]); lb.push_back(ds[i].b); lx.push_back(ds[i].x); }
        std::vector<hb_batch_result> res(live.size());
        int bst = HB_OK;
        if (!live.empty())
            bst = hb_q1_batch_solve(w.ctx, lq.data(), lb.data(), lx.data(), (int64_t)live.size(), s->p.eps,
                                    s->p.inner_eps, 50, 2000, &s->p.mid_cfg, res.data());
        for (size_t k = 0; k < live.size(); ++k) {
            const int64_t i = live[k];
            if (bst) { st[i] = bst; continue; }
            const hb_request &r = batch[i]->r;
            if (cudaMemcpyAsync(r.x, ds[i].x, r.M * r.M * 8, cudaMemcpyDeviceToHost, w.stream) != cudaSuccess)
                st[i] = HB_ERR_CUDA;
        }
        for (hb_q1 *q : qs)
            if (q) hb_q1_destroy(q);
        for (auto &d : ds) d.release();
        if (cudaStreamSynchronize(w.stream) != cudaSuccess) cudaGetLastError();
        const double t = s->now();
        size_t k = 0;
        for (int64_t i = 0; i < count; ++i) {
            hb_completion c{};
            c.tag = batch[i]->r.tag;
            c.path = HB_PATH_MGBATCH;
            c.t_submit = batch[i]->t_submit;
            c.t_admit = batch[i]->t_admit;
            c.bytes = batch[i]->bytes;
            c.t_done = t;
            c.status = st[i];
            if (k < live.size() && live[k] == i) {
                if (!st[i]) {
                    c.iterations = res[k].iterations;
                    c.outer = res[k].outer;
                    c.true_relres = res[k].true_relres;
                    c.status = res[k].status;
                }
                ++k;
            }
            s->complete(batch[i], c);
        }
    }
}

}  // namespace

extern "C" {

int hb_server_create(const hb_server_params *params, hb_server **out)
{
    if (!params || !out) return HB_ERR_INVALID;
    *out = nullptr;
    if (params->mode != HB_SERVE_MIXED && params->mode != HB_SERVE_PLAIN_CG64 &&
        params->mode != HB_SERVE_PLAIN_CG64_BATCHED)
        return HB_ERR_INVALID;
    if (params->hbm_budget_bytes <= 0) return HB_ERR_INVALID;
    hb_server *s = new hb_server();
    s->p = *params;
    if (s->p.large_workers < 1) s->p.large_workers = 1;
    if (s->p.small_workers < 1) s->p.small_workers = 1;
    if (s->p.max_batch < 1) s->p.max_batch = 256;
    if (s->p.batch_cfg.cluster == 0) s->p.batch_cfg = hb_batch_config{2, 512, 0, 0};
    if (s->p.mid_cfg.cluster == 0) s->p.mid_cfg = hb_batch_config{16, 512, 0, 0};
    s->t0 = std::chrono::steady_clock::now();
    s->admitter = std::thread(admit_loop, s);
    // the pool's high-water marks from here on (hb_server_pool_stats)
    if (cudaDeviceGetDefaultMemPool(&s->pool, s->p.device) == cudaSuccess) {
        unsigned long long zero = 0;
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrUsedMemHigh, &zero);
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReservedMemHigh, &zero);
    } else {
        cudaGetLastError();
        s->pool = nullptr;
    }
    if (s->p.mode == HB_SERVE_PLAIN_CG64) {
        s->workers.emplace_back(large_loop, s);   // one request at a time
    } else if (s->p.mode == HB_SERVE_PLAIN_CG64_BATCHED) {
        for (int i = 0; i < s->p.large_workers; ++i) s->workers.emplace_back(large_loop, s);
        for (int i = 0; i < s->p.small_workers; ++i) s->workers.emplace_back(small_loop, s);
    } else {
        for (int i = 0; i < s->p.large_workers; ++i) s->workers.emplace_back(large_loop, s);
        for (int i = 0; i < s->p.small_workers; ++i) s->workers.emplace_back(small_loop, s);
        if (s->p.mid_max_side > s->p.small_max_side)
            for (int i = 0; i < std::max(1, s->p.mid_workers); ++i) s->workers.emplace_back(mid_loop, s);
    }
    *out = s;
    return HB_OK;
}

int hb_server_submit(hb_server *s, const hb_request *req)
{
    if (!s || !req || req->M < 1 || !req->x || (!req->b && !req->x_true)) return HB_ERR_INVALID;
    if (req->M * req->M > INT32_MAX) return HB_ERR_UNSUPPORTED;
    Item *it = new Item();
    it->r = *req;
    it->path = route(s, req->M);
    it->bytes = estimate_bytes(it->path, req->M);
    std::lock_guard<std::mutex> l(s->mu);
    if (it->bytes > s->p.hbm_budget_bytes) {
        delete it;
        return HB_ERR_CAPACITY;
    }
    it->t_submit = s->now();
    s->pending.push_back(it);
    ++s->submitted;
    s->cv_pending.notify_all();
    return HB_OK;
}

int hb_server_poll(hb_server *s, hb_completion *out, int max, int *n, int wait_ms)
{
    if (!s || !n || (max > 0 && !out)) return HB_ERR_INVALID;
    std::unique_lock<std::mutex> l(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(l, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    const int k = std::min<int>(max, (int)s->done.size());
    for (int i = 0; i < k; ++i) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return HB_OK;
}

int hb_server_drain(hb_server *s)
{
    if (!s) return HB_ERR_INVALID;
    std::unique_lock<std::mutex> l(s->mu);
    s->cv_done.wait(l, [&] { return s->completed >= s->submitted; });
    return HB_OK;
}

double hb_server_clock(hb_server *s) { return s ? s->now() : 0.0; }

int hb_server_stats(hb_server *s, int64_t *in_use, int64_t *peak, int64_t *submitted, int64_t *completed)
{
    if (!s) return HB_ERR_INVALID;
    std::lock_guard<std::mutex> l(s->mu);
    if (in_use) *in_use = s->in_use;
    if (peak) *peak = s->peak;
    if (submitted) *submitted = s->submitted;
    if (completed) *completed = s->completed;
    return HB_OK;
}

int hb_server_pool_stats(hb_server *s, int64_t *used_high, int64_t *reserved_high)
{
    if (!s) return HB_ERR_INVALID;
    if (!s->pool) return HB_ERR_UNSUPPORTED;
    unsigned long long u = 0, r = 0;
    if (cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrUsedMemHigh, &u) != cudaSuccess ||
        cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemHigh, &r) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    if (used_high) *used_high = (int64_t)u;
    if (reserved_high) *reserved_high = (int64_t)r;
    return HB_OK;
}

int hb_server_destroy(hb_server *s)
{
    if (!s) return HB_ERR_INVALID;
    hb_server_drain(s);
    {
        std::lock_guard<std::mutex> l(s->mu);
        s->stop = true;
        s->cv_pending.notify_all();
        s->cv_work.notify_all();
        s->cv_mem.notify_all();
    }
    s->admitter.join();
    for (auto &t : s->workers) t.join();
    for (Item *it : s->pending) delete it;
    delete s;
    return HB_OK;
}

}  // extern "C"
