// hb_cg.cu -- CGSolver<Tag, methods::NONE> (honei/math/cg.hh:63-133) as one persistent
// cooperative kernel.
//
// The reference runs 7 launches, 2 device->host scalar round trips and 2 cudaMalloc/cudaFree
// pairs per iteration (honei/la/*-cuda.cc).  Here the loop, its scalars and its stopping test
// live on the device; per iteration there are two phases, each ending in a grid-wide reduction
// on an arrival counter (hbd::CountExchange):
//
//   phase 1  p_i = r_i + beta * p_i  (computed on the fly for every gathered column, so the
//            separate Scale+Sum passes disappear), v = A p, partial v.p
//   phase 2  lambda = alpha / v.p;  x += lambda p;  r += (-lambda) v;  partial r.r
//
// Rows are dealt to threads in lane-strided quads (hbd::quad_rows: lane l of a 128-row tile
// owns rows l, l + 32, l + 64, l + 96), so each gather instruction of a warp reads 32
// neighbouring rows' columns -- about two cache lines instead of eight for four consecutive rows
// per thread; with three ELL slots' loads in flight per step this took the 1025^2 iteration from
// 45 to 32 us.  The one-block kernel for small systems deals its rows the same way, so the two
// give bit-identical iterates.
// The gathers of x, r and p are ordinary, L1-cacheable loads: every value they read was written
// by another block before its release-arrival at an exchange that this block acquired (thread 0)
// and then passed through __syncthreads, so the memory model guarantees the current value; the
// rows of a warp then share L1 lines, where an L2-only load fetches a 32-byte sector per 8-byte
// element (about a third less time per iteration at 1025^2).
// p is double-buffered (phase 1 gathers the old p of neighbour rows while writing the new p
// of its own rows).  Every elementwise formula rounds exactly as cg.hh's operator sequence
// (ScaledSum, Scale, Sum) does on tags::CPU; the two dot products use a fixed-order tree
// (block partials, then every block sums all partials in the same order), so each block
// computes bit-identical scalars and takes the same branch at the stopping test.
#include "hb_resident.cuh"

#include <cfloat>
#include <mutex>

namespace {

constexpr int CG_THREADS = 512;

template <typename T> struct CGParams {
    int64_t rows, ld;
    int K;
    const int32_t *Aj;
    const T *Ax;
    const T *b_user;
    T *x_user;
    T *x, *r, *p0, *p1, *v;    // padded work vectors, ld entries each
    int64_t max_iters;
    T eps;
    T *partials;                // 2 * gridDim.x
    hbd::GridBarrier bar;
    hb_solve_result *res;
};

template <typename T> __device__ __forceinline__ T eps_mach();
template <> __device__ __forceinline__ double eps_mach<double>() { return DBL_EPSILON; }
template <> __device__ __forceinline__ float eps_mach<float>() { return FLT_EPSILON; }
__device__ __forceinline__ double dsqrt(double v) { return __dsqrt_rn(v); }
__device__ __forceinline__ float dsqrt(float v) { return __fsqrt_rn(v); }

// Sum of the gridDim.x block partials in a fixed tree order; identical in every block.
template <typename T>
__device__ __forceinline__ T grid_total(const T *part, T *red, T *bcast)
{
    T v = T(0);
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v = hbd::add(v, __ldcg(part + i));
    v = hbd::block_sum(v, red);
    if (threadIdx.x == 0) *bcast = v;
    __syncthreads();
    return *bcast;
}

template <typename T, int KT>
__global__ void __launch_bounds__(CG_THREADS) cg_kernel(CGParams<T> P)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    __shared__ T red[32];
    __shared__ T bcast;
    __shared__ int s_flag;
    const unsigned G = gridDim.x;
    const int64_t groups = P.ld / 4;
    const int64_t gpb = (groups + G - 1) / G;
    const int64_t g_lo = (int64_t)blockIdx.x * gpb;
    const int64_t g_hi = min(groups, g_lo + gpb);
    const hbd::CountExchange X{P.bar.count, P.bar.status};
    unsigned e = 0;
    const int64_t rows = P.rows;
    bool ok = true;

    // x (padded with zeros) from the caller's x0
    for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
        uint32_t row[4];
        hbd::quad_rows(g, groups, row);
#pragma unroll
        for (int i = 0; i < 4; ++i) P.x[row[i]] = (row[i] < rows) ? P.x_user[row[i]] : T(0);
    }
    ok = X.arrive_wait(T(0), P.partials, e, G, &s_flag);

    // r = b - A x (Defect), alpha = r.r (Norm<l2, false>)
    T acc = T(0);
    if (ok) {
        const T *xw = P.x;
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T s[4];
            hbd::ell_rows4s<T, KT, (KT > 0 ? 3 : 4)>(P.Aj, P.Ax, P.ld, P.K, row, [&](int32_t j) { return xw[j]; }, s);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const T bb = (row[i] < rows) ? P.b_user[row[i]] : T(0);
                const T rv = sub(bb, s[i]);
                acc = add(acc, mul(rv, rv));
                P.r[row[i]] = rv;
            }
        }
        acc = hbd::block_sum(acc, red);
        ok = X.arrive_wait(acc, P.partials, ++e, G, &s_flag);
    }
    T alpha = ok ? grid_total(P.partials + (e & 1u) * G, red, &bcast) : T(0);
    const T initial_defect = dsqrt(alpha);
    T current_defect = T(0);
    T beta = T(0);
    const T epsm = eps_mach<T>();
    T *pin = P.p0, *pout = P.p1;
    int64_t it = 0, used = 0;
    while (ok && it < P.max_iters) {
        // ---- phase 1: p = beta p + r (first iteration: p = r), v = A p, v.p
        const T *rw = P.r, *pw = pin;
        const bool first = (it == 0);
        acc = T(0);
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T s[4];
            hbd::ell_rows4s<T, KT, (KT > 0 ? 3 : 4)>(P.Aj, P.Ax, P.ld, P.K, row, [&](int32_t j) {
                const T rj = rw[j];
                return first ? rj : add(mul(pw[j], beta), rj);
            }, s);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const T rv = P.r[row[i]];
                const T pn = first ? rv : add(mul(pin[row[i]], beta), rv);
                acc = add(acc, mul(s[i], pn));
                pout[row[i]] = pn;
                P.v[row[i]] = s[i];
            }
        }
        acc = hbd::block_sum(acc, red);
        if (!X.arrive_wait(acc, P.partials, ++e, G, &s_flag)) break;
        const T temp = grid_total(P.partials + (e & 1u) * G, red, &bcast);
        const T lambda = alpha / (fabs(temp) > epsm ? temp : epsm);
        const T mlambda = -lambda;

        // ---- phase 2: x += lambda p; r += (-lambda) v; alpha = r.r
        acc = T(0);
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T xv[4], pv[4], rv[4], vv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xv[i] = P.x[row[i]];
                pv[i] = pout[row[i]];
                rv[i] = P.r[row[i]];
                vv[i] = P.v[row[i]];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xv[i] = add(xv[i], mul(lambda, pv[i]));
                rv[i] = add(rv[i], mul(mlambda, vv[i]));
                acc = add(acc, mul(rv[i], rv[i]));
                P.x[row[i]] = xv[i];
                P.r[row[i]] = rv[i];
            }
        }
        acc = hbd::block_sum(acc, red);
        if (!X.arrive_wait(acc, P.partials, ++e, G, &s_flag)) break;
        const T alpha_old = alpha;
        alpha = grid_total(P.partials + (e & 1u) * G, red, &bcast);
        beta = alpha / (fabs(alpha_old) > epsm ? alpha_old : epsm);
        T *t = pin; pin = pout; pout = t;
        ++it;
        current_defect = dsqrt(alpha);
        if (current_defect < P.eps * initial_defect) { used = it; break; }
        if (current_defect < P.eps) { used = it; break; }
        if (it == P.max_iters) used = it;
    }
    // x back to the caller (own rows)
    for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
        uint32_t row[4];
        hbd::quad_rows(g, groups, row);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (row[i] < rows) P.x_user[row[i]] = P.x[row[i]];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.res->used = used;
        P.res->defect0 = (double)initial_defect;
        P.res->defect = (double)current_defect;
        P.res->status = *(volatile int *)P.bar.status;
    }
}

// ---------------------------------------------------------------------------------------
// The same persistent CG with one row per thread: each block owns the same contiguous rows as
// in cg_kernel (whole groups of four), its threads walk them one row at a time with every
// slot's Aj / Ax load of the row in flight together, then every gather.  Fewer registers per
// thread than the four-row groups, so three 256-thread blocks share an SM (24 warps against 16)
// and more loads are in flight per SM.  Same formulas, same per-row summation order and the
// same exchanges; the dot products' partial sums group the rows differently, so its iterates
// differ from cg_kernel's at round-off (same bar against the reference).
// ---------------------------------------------------------------------------------------
constexpr int CG_ROW_THREADS = 256;

template <typename T, int KT>
__global__ void __launch_bounds__(CG_ROW_THREADS, 3) cg_row_kernel(CGParams<T> P)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    constexpr int KS = KT > 0 ? KT : 4;
    __shared__ T red[32];
    __shared__ T bcast;
    __shared__ int s_flag;
    const unsigned G = gridDim.x;
    const int64_t groups = P.ld / 4;
    const int64_t gpb = (groups + G - 1) / G;
    const int64_t lo = 4 * min(groups, (int64_t)blockIdx.x * gpb);
    const int64_t hi = 4 * min(groups, (int64_t)blockIdx.x * gpb + gpb);
    const int kend = KT > 0 ? KT : P.K;
    const hbd::CountExchange X{P.bar.count, P.bar.status};
    unsigned e = 0;
    const int64_t rows = P.rows;
    bool ok = true;

    // the row's sum over its slots in slot order, gathering g(j) for column j
    auto row_sum = [&](int64_t row, auto g) {
        T sm = T(0);
        for (int k0 = 0; k0 < kend; k0 += KS) {
            int32_t j[KS];
            T a[KS];
#pragma unroll
            for (int c = 0; c < KS; ++c) {
                const bool in = k0 + c < kend;
                j[c] = in ? __ldcs(P.Aj + (int64_t)(k0 + c) * P.ld + row) : -1;
                a[c] = in ? __ldcs(P.Ax + (int64_t)(k0 + c) * P.ld + row) : T(0);
            }
            T v[KS];
#pragma unroll
            for (int c = 0; c < KS; ++c) v[c] = j[c] >= 0 ? g(j[c]) : T(0);
#pragma unroll
            for (int c = 0; c < KS; ++c)
                if (j[c] >= 0) sm = add(sm, mul(a[c], v[c]));
        }
        return sm;
    };

    for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x)
        P.x[row] = row < rows ? P.x_user[row] : T(0);
    ok = X.arrive_wait(T(0), P.partials, e, G, &s_flag);

    T acc = T(0);
    if (ok) {
        const T *xw = P.x;
        for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x) {
            const T s = row_sum(row, [&](int32_t j) { return xw[j]; });
            const T bb = row < rows ? P.b_user[row] : T(0);
            const T rv = sub(bb, s);
            acc = add(acc, mul(rv, rv));
            P.r[row] = rv;
        }
        acc = hbd::block_sum(acc, red);
        ok = X.arrive_wait(acc, P.partials, ++e, G, &s_flag);
    }
    T alpha = ok ? grid_total(P.partials + (e & 1u) * G, red, &bcast) : T(0);
    const T initial_defect = dsqrt(alpha);
    T current_defect = T(0);
    T beta = T(0);
    const T epsm = eps_mach<T>();
    T *pin = P.p0, *pout = P.p1;
    int64_t it = 0, used = 0;
    while (ok && it < P.max_iters) {
        const T *rw = P.r, *pw = pin;
        const bool first = (it == 0);
        acc = T(0);
        for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x) {
            const T s = row_sum(row, [&](int32_t j) {
                const T rj = rw[j];
                return first ? rj : add(mul(pw[j], beta), rj);
            });
            const T rv = P.r[row];
            const T pn = first ? rv : add(mul(pin[row], beta), rv);
            acc = add(acc, mul(s, pn));
            pout[row] = pn;
            P.v[row] = s;
        }
        acc = hbd::block_sum(acc, red);
        if (!X.arrive_wait(acc, P.partials, ++e, G, &s_flag)) break;
        const T temp = grid_total(P.partials + (e & 1u) * G, red, &bcast);
        const T lambda = alpha / (fabs(temp) > epsm ? temp : epsm);
        const T mlambda = -lambda;
        acc = T(0);
        for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x) {
            const T xv = add(P.x[row], mul(lambda, pout[row]));
            const T rv = add(P.r[row], mul(mlambda, P.v[row]));
            acc = add(acc, mul(rv, rv));
            P.x[row] = xv;
            P.r[row] = rv;
        }
        acc = hbd::block_sum(acc, red);
        if (!X.arrive_wait(acc, P.partials, ++e, G, &s_flag)) break;
        const T alpha_old = alpha;
        alpha = grid_total(P.partials + (e & 1u) * G, red, &bcast);
        beta = alpha / (fabs(alpha_old) > epsm ? alpha_old : epsm);
        T *t = pin; pin = pout; pout = t;
        ++it;
        current_defect = dsqrt(alpha);
        if (current_defect < P.eps * initial_defect) { used = it; break; }
        if (current_defect < P.eps) { used = it; break; }
        if (it == P.max_iters) used = it;
    }
    for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x)
        if (row < rows) P.x_user[row] = P.x[row];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.res->used = used;
        P.res->defect0 = (double)initial_defect;
        P.res->defect = (double)current_defect;
        P.res->status = *(volatile int *)P.bar.status;
    }
}

// ---------------------------------------------------------------------------------------
// Small systems (at most SMALL_GROUPS row groups, e.g. the coarsest MG level): the same
// iteration in one block, thread t owning row group t, p exchanged through shared memory and
// the matrix slots held in registers, so an iteration is two block reductions and no global
// round trip or grid barrier.  For these sizes the cooperative kernel runs as a single block
// with the same thread-to-group mapping and the same reduction tree (threads without rows add
// exact zeros), so both kernels produce bit-identical iterates.
// ---------------------------------------------------------------------------------------
constexpr int SMALL_GROUPS = 256;

// Block-wide fixed-order total, identical in every thread.  A single-warp block (systems of at
// most 128 rows, e.g. the 9^2 coarse grid) reduces with shuffles only: the block tree of one warp
// is the warp tree plus exact zeros, so both paths give the same value.
template <typename T>
__device__ __forceinline__ T block_total(T v, T *red, T *bcast)
{
    if (blockDim.x == 32) {
        v = hbd::warp_sum(v);
        return __shfl_sync(0xffffffffu, v, 0);
    }
    v = hbd::block_sum(v, red);
    if (threadIdx.x == 0) *bcast = v;
    __syncthreads();
    return *bcast;
}

__device__ __forceinline__ void block_sync()
{
    if (blockDim.x == 32) __syncwarp();
    else __syncthreads();
}

template <typename T, int KT>
__global__ void __launch_bounds__(SMALL_GROUPS) cg_small_kernel(CGParams<T> P)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    constexpr int KR = KT > 0 ? KT : 1;
    __shared__ __align__(16) T sp[4 * SMALL_GROUPS];
    __shared__ T red[32];
    __shared__ T bcast;
    const int64_t rows = P.rows;
    const int64_t groups = P.ld / 4;
    const int64_t g = threadIdx.x;
    const bool own = g < groups;
    // the rows of this thread's quad, lane-strided exactly as in cg_kernel
    uint32_t row[4] = {0, 0, 0, 0};
    if (own) hbd::quad_rows(g, groups, row);

    int32_t aj[KR][4];
    T ax[KR][4];
    if (KT > 0) {
#pragma unroll
        for (int k = 0; k < KR; ++k) {
            if (own) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    aj[k][i] = __ldcs(P.Aj + (int64_t)k * P.ld + row[i]);
                    ax[k][i] = __ldcs(P.Ax + (int64_t)k * P.ld + row[i]);
                }
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) { aj[k][i] = -1; ax[k][i] = T(0); }
            }
        }
    }
    // s = A sp on the thread's own rows, slots in the reference order
    auto product = [&](T (&s)[4]) {
#pragma unroll
        for (int i = 0; i < 4; ++i) s[i] = T(0);
        if (!own) return;
        if (KT > 0) {
#pragma unroll
            for (int k = 0; k < KR; ++k)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (aj[k][i] >= 0) s[i] = add(s[i], mul(ax[k][i], sp[aj[k][i]]));
        } else {
            for (int k = 0; k < P.K; ++k)
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int32_t j = __ldg(P.Aj + (int64_t)k * P.ld + row[i]);
                    if (j >= 0) s[i] = add(s[i], mul(__ldg(P.Ax + (int64_t)k * P.ld + row[i]), sp[j]));
                }
        }
    };

    T x[4], r[4], p[4], v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        x[i] = (own && row[i] < rows) ? P.x_user[row[i]] : T(0);
        if (own) sp[row[i]] = x[i];
    }
    block_sync();
    // r = b - A x, alpha = r.r
    T acc = T(0);
    product(v);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const T bb = (own && row[i] < rows) ? P.b_user[row[i]] : T(0);
        r[i] = sub(bb, v[i]);
        acc = add(acc, mul(r[i], r[i]));
        p[i] = T(0);
    }
    T alpha = block_total(acc, red, &bcast);
    const T initial_defect = dsqrt(alpha);
    T current_defect = T(0);
    T beta = T(0);
    const T epsm = eps_mach<T>();
    int64_t it = 0, used = 0;
    while (it < P.max_iters) {
        const bool first = (it == 0);
        // every lane's gathers of the previous p are done before p is rewritten (the block
        // path's reductions end in __syncthreads; shuffles do not order shared memory)
        if (blockDim.x == 32) __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            p[i] = first ? r[i] : add(mul(p[i], beta), r[i]);
            if (own) sp[row[i]] = p[i];
        }
        block_sync();
        product(v);
        acc = T(0);
#pragma unroll
        for (int i = 0; i < 4; ++i) acc = add(acc, mul(v[i], p[i]));
        const T temp = block_total(acc, red, &bcast);
        const T lambda = alpha / (fabs(temp) > epsm ? temp : epsm);
        const T mlambda = -lambda;
        acc = T(0);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            x[i] = add(x[i], mul(lambda, p[i]));
            r[i] = add(r[i], mul(mlambda, v[i]));
            acc = add(acc, mul(r[i], r[i]));
        }
        const T alpha_old = alpha;
        alpha = block_total(acc, red, &bcast);
        beta = alpha / (fabs(alpha_old) > epsm ? alpha_old : epsm);
        ++it;
        current_defect = dsqrt(alpha);
        if (current_defect < P.eps * initial_defect) { used = it; break; }
        if (current_defect < P.eps) { used = it; break; }
        if (it == P.max_iters) used = it;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (own && row[i] < rows) P.x_user[row[i]] = x[i];
    if (threadIdx.x == 0) {
        P.res->used = used;
        P.res->defect0 = (double)initial_defect;
        P.res->defect = (double)current_defect;
        P.res->status = 0;
    }
}

template <typename T, int KT>
int launch_cg_small(hb_context *ctx, const CGParams<T> &P, int64_t groups)
{
    const int threads = (int)std::max<int64_t>(32, (groups + 31) / 32 * 32);
    cg_small_kernel<T, KT><<<1, threads, 0, ctx->stream>>>(P);
    return hb_check_launch(ctx, "cg_small_kernel");
}

// ---------------------------------------------------------------------------------------
// Resident-operator form, for systems whose rows fit the shared memory of one block per SM:
// each block owns a contiguous row range, keeps its ELL rows (Ax, and Aj as window offsets),
// x and v of its rows, and r and p on its column window (its own rows plus the columns its rows
// reach) in shared memory for the whole solve.  p on the window is formed redundantly by every
// block that holds it (the same p = beta p + r, bit for bit), so only r crosses blocks: each
// block stores its rows of r, and after the second exchange of an iteration reads the window's
// other rows (the halo) from L2 together with the partials.  Both reductions per iteration go
// through the arrival-counter exchange.  A column outside the window (a block whose rows reach
// further than the window capacity) is gathered from the global r and p, which every block also
// stores for its rows; the arithmetic is the same either way.  Per row the product sums the
// slots in slot order skipping padding, as the ELL product does; the dot products are sums per
// thread over its rows, a block tree and a tree over the block partials -- deterministic, the
// same in every block.
// ---------------------------------------------------------------------------------------
template <typename T> struct ResParams {
    CGParams<T> c;
    int64_t rpb;     // rows per block
    int64_t wcap;    // window capacity: entries of r and of p held in shared memory
    hbd::CountExchange X;
};

template <typename T, int KT>
__global__ void __launch_bounds__(hbr::RES_THREADS, 1) cg_res_kernel(const ResParams<T> Q)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    extern __shared__ __align__(16) unsigned char res_smem[];
    __shared__ T red[32];
    __shared__ T bcast[2];
    __shared__ int s_flag, s_min, s_max;
    const CGParams<T> &P = Q.c;
    const int K = KT > 0 ? KT : P.K;
    const int64_t rpb = Q.rpb, wcap = Q.wcap;
    const unsigned G = gridDim.x;
    T *Ax_s = (T *)res_smem;                    // [K][rpb]
    T *r_w = Ax_s + (int64_t)K * rpb;           // [wcap]
    T *p_w = r_w + wcap;                        // [wcap]
    T *x_s = p_w + wcap;                        // [rpb]
    T *v_s = x_s + rpb;                         // [rpb]
    int32_t *Aj_s = (int32_t *)(v_s + rpb);     // [K][rpb]
    const hbr::ResWindow win = hbr::res_stage<T, KT>(P.Aj, P.Ax, P.ld, P.K, P.rows, rpb, wcap, Ax_s, Aj_s, &s_min, &s_max);
    const int64_t lo = win.lo, wlo = win.wlo, W = win.W, own = win.own();
    const int nr = win.nr;

    // r = b - A x (Defect), alpha = r.r
    T acc = T(0);
    for (int il = threadIdx.x; il < nr; il += blockDim.x) {
        T s = T(0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int32_t c = Aj_s[(int64_t)k * rpb + il];
            if (c == -1) continue;
            s = add(s, mul(Ax_s[(int64_t)k * rpb + il], P.x_user[hbr::res_column(c, wlo)]));
        }
        const T r = sub(P.b_user[lo + il], s);
        r_w[own + il] = r;
        x_s[il] = P.x_user[lo + il];
        __stcg(P.r + lo + il, r);
        acc = add(acc, mul(r, r));
    }
    acc = hbr::res_partial(acc, red);
    unsigned e = 0;
    if (threadIdx.x == 0) __stcg(P.partials + (e & 1u) * G + blockIdx.x, acc);
    bool ok = Q.X.arrive_synced(e, G, &s_flag);
    T pv[hbr::RES_MAX_BLOCKS / 32];
    T alpha = T(0);
    if (ok) {
        hbr::res_total_load(P.partials + (e & 1u) * G, G, pv);
        hbr::res_halo(P.r, r_w, win);
        alpha = hbr::res_total_sum(G, pv, &bcast[0]);
    }
    const T initial_defect = dsqrt(alpha);
    T current_defect = T(0);
    T beta = T(0);
    const T epsm = eps_mach<T>();
    T *pin = P.p0, *pout = P.p1;
    int64_t it = 0, used = 0;
    while (ok && it < P.max_iters) {
        // ---- phase 1: p = beta p + r on the window (first iteration: p = r), v = A p, v.p
        const bool first = (it == 0);
        for (int64_t w = threadIdx.x; w < W; w += blockDim.x) p_w[w] = first ? r_w[w] : add(mul(p_w[w], beta), r_w[w]);
        __syncthreads();
        acc = T(0);
        for (int il = threadIdx.x; il < nr; il += blockDim.x) {
            T s = T(0);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int32_t c = Aj_s[(int64_t)k * rpb + il];
                if (c == -1) continue;
                T pj;
                if (c >= 0) {
                    pj = p_w[c];
                } else {
                    const int64_t j = hbr::res_column(c, wlo);
                    const T rj = __ldca(P.r + j);
                    pj = first ? rj : add(mul(__ldca(pin + j), beta), rj);
                }
                s = add(s, mul(Ax_s[(int64_t)k * rpb + il], pj));
            }
            v_s[il] = s;
            const T pi = p_w[own + il];
            __stcg(pout + lo + il, pi);
            acc = add(acc, mul(s, pi));
        }
        acc = hbr::res_partial(acc, red);
        ++e;
        if (threadIdx.x == 0) __stcg(P.partials + (e & 1u) * G + blockIdx.x, acc);
        if (!Q.X.arrive_synced(e, G, &s_flag)) break;
        hbr::res_total_load(P.partials + (e & 1u) * G, G, pv);
        const T temp = hbr::res_total_sum(G, pv, &bcast[1]);
        const T lambda = alpha / (fabs(temp) > epsm ? temp : epsm);
        const T mlambda = -lambda;

        // ---- phase 2: x += lambda p; r += (-lambda) v; alpha = r.r
        acc = T(0);
        for (int il = threadIdx.x; il < nr; il += blockDim.x) {
            x_s[il] = add(x_s[il], mul(lambda, p_w[own + il]));
            const T r = add(r_w[own + il], mul(mlambda, v_s[il]));
            r_w[own + il] = r;
            __stcg(P.r + lo + il, r);
            acc = add(acc, mul(r, r));
        }
        acc = hbr::res_partial(acc, red);
        ++e;
        if (threadIdx.x == 0) __stcg(P.partials + (e & 1u) * G + blockIdx.x, acc);
        if (!Q.X.arrive_synced(e, G, &s_flag)) break;
        hbr::res_total_load(P.partials + (e & 1u) * G, G, pv);
        hbr::res_halo(P.r, r_w, win);
        const T alpha_old = alpha;
        alpha = hbr::res_total_sum(G, pv, &bcast[0]);
        beta = alpha / (fabs(alpha_old) > epsm ? alpha_old : epsm);
        T *t = pin; pin = pout; pout = t;
        ++it;
        current_defect = dsqrt(alpha);
        if (current_defect < P.eps * initial_defect) { used = it; break; }
        if (current_defect < P.eps) { used = it; break; }
        if (it == P.max_iters) used = it;
    }
    for (int il = threadIdx.x; il < nr; il += blockDim.x) P.x_user[lo + il] = x_s[il];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.res->used = used;
        P.res->defect0 = (double)initial_defect;
        P.res->defect = (double)current_defect;
        P.res->status = *(volatile int *)Q.X.status;
    }
}

template <typename T, int KT>
int launch_cg_res(hb_context *ctx, CGParams<T> &P, bool *launched)
{
    *launched = false;
    hbr::ResPlan plan;
    if (!hbr::res_plan<T>(ctx, P.rows, KT > 0 ? KT : P.K, 2, 2, (const void *)cg_res_kernel<T, KT>, &plan)) return HB_OK;
    ResParams<T> Q;
    Q.c = P;
    Q.rpb = plan.rpb;
    Q.wcap = plan.wcap;
    Q.X.count = P.bar.count;
    Q.X.status = P.bar.status;
    void *args[] = {&Q};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)cg_res_kernel<T, KT>, dim3(plan.blocks),
                                                dim3(hbr::RES_THREADS), args, plan.smem, ctx->stream);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchCooperativeKernel(cg_res_kernel)"); return HB_ERR_CUDA; }
    *launched = true;
    return hb_check_launch(ctx, "cg_res_kernel");
}

template <typename T, int KT>
int launch_cg_kt(hb_context *ctx, CGParams<T> &P, int blocks)
{
    void *args[] = {&P};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)cg_kernel<T, KT>, dim3(blocks), dim3(CG_THREADS),
                                                args, 0, ctx->stream);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchCooperativeKernel(cg_kernel)"); return HB_ERR_CUDA; }
    return hb_check_launch(ctx, "cg_kernel");
}

template <typename T, int KT>
int cg_max_blocks(hb_context *ctx)
{
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, cg_kernel<T, KT>, CG_THREADS, 0);
    return std::max(1, occ) * ctx->num_sms;
}

// The one-row-per-thread kernel: every co-resident block (for systems large enough to fill
// them), else about one row per thread.
template <typename T, int KT>
int launch_cg_row(hb_context *ctx, CGParams<T> &P)
{
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, cg_row_kernel<T, KT>, CG_ROW_THREADS, 0) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    const int64_t maxb = (int64_t)std::max(1, occ) * ctx->num_sms;
    const int64_t want = (P.ld + CG_ROW_THREADS - 1) / CG_ROW_THREADS;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(maxb, 4096)));
    void *args[] = {&P};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)cg_row_kernel<T, KT>, dim3(blocks),
                                                dim3(CG_ROW_THREADS), args, 0, ctx->stream);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchCooperativeKernel(cg_row_kernel)"); return HB_ERR_CUDA; }
    return hb_check_launch(ctx, "cg_row_kernel");
}

}  // namespace

template <typename T>
int hb_launch_cg(hb_context *ctx, const hb_ell *A, const T *b, T *x, int64_t max_iters, T eps, T *work,
                 hb_solve_result *res)
{
    const int64_t ld = A->ld;
    CGParams<T> P;
    P.rows = A->rows;
    P.ld = ld;
    P.K = (int)A->K;
    P.Aj = A->Aj;
    P.Ax = (const T *)A->Ax;
    P.b_user = b;
    P.x_user = x;
    P.x = work; P.r = work + ld; P.p0 = work + 2 * ld; P.p1 = work + 3 * ld; P.v = work + 4 * ld;
    P.max_iters = max_iters;
    P.eps = eps;
    P.partials = (T *)hb_partials(ctx);
    unsigned *bar = hb_bar(ctx);
    P.bar.count = bar;
    P.bar.gen = bar + 1;
    P.bar.status = (int *)(bar + 2);
    P.res = res;
    const int64_t groups = ld / 4;
    const bool k9 = (A->K == 9);
    if (groups <= SMALL_GROUPS)
        return k9 ? launch_cg_small<T, 9>(ctx, P, groups) : launch_cg_small<T, 0>(ctx, P, groups);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), ctx->stream));
    const int maxb = k9 ? cg_max_blocks<T, 9>(ctx) : cg_max_blocks<T, 0>(ctx);
    // about one row group per thread for small systems; all co-resident blocks otherwise
    const int64_t want = (groups + CG_THREADS - 1) / CG_THREADS;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(maxb, 4096)));
    if (ctx->cg_resident) {
        bool launched = false;
        const int st = k9 ? launch_cg_res<T, 9>(ctx, P, &launched) : launch_cg_res<T, 0>(ctx, P, &launched);
        if (st || launched) return st;
    }
    if (ctx->cg_row_layout) return k9 ? launch_cg_row<T, 9>(ctx, P) : launch_cg_row<T, 0>(ctx, P);
    return k9 ? launch_cg_kt<T, 9>(ctx, P, blocks) : launch_cg_kt<T, 0>(ctx, P, blocks);
}
template int hb_launch_cg<double>(hb_context *, const hb_ell *, const double *, double *, int64_t, double,
                                  double *, hb_solve_result *);
template int hb_launch_cg<float>(hb_context *, const hb_ell *, const float *, float *, int64_t, float, float *,
                                 hb_solve_result *);

namespace {

template <typename T>
int cg_impl(hb_context *ctx, const hb_ell *A, const T *b, T *x, int64_t max_iters, T eps,
            int64_t *used_iters, T *final_defect, int dtype)
{
    if (!ctx || !A || !b || !x || !used_iters || max_iters < 0) return HB_ERR_INVALID;
    int st = hb_check_ell(A, dtype);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    st = hb_ensure_work(ctx, (size_t)A->ld * sizeof(T) * 5);
    if (st) return st;
    st = hb_launch_cg<T>(ctx, A, b, x, max_iters, eps, (T *)ctx->work, hb_result(ctx));
    if (st) return st;
    hb_solve_result *h = (hb_solve_result *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, hb_result(ctx), sizeof(hb_solve_result), cudaMemcpyDeviceToHost,
                                     ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h->status == HB_DEV_TIMEOUT) return HB_ERR_TIMEOUT;
    *used_iters = h->used;
    if (final_defect) *final_defect = (T)h->defect;
    return HB_OK;
}

}  // namespace

namespace {

// One block waits for a second block that never comes, at a grid barrier (COUNTER false) or at
// an arrival-counter exchange (COUNTER true): the wait runs to its limit (HB_WAIT_NS), records
// HB_DEV_TIMEOUT and the kernel returns.
template <bool COUNTER>
__global__ void wait_timeout_kernel(hbd::GridBarrier bar, double *slots, hb_solve_result *res)
{
    __shared__ int s_flag;
    bool ok;
    if (COUNTER) ok = hbd::CountExchange{bar.count, bar.status}.arrive_wait(1.0, slots, 0u, 2u, &s_flag);
    else ok = bar.sync(2, &s_flag);
    if (threadIdx.x == 0) {
        res->used = ok ? 1 : 0;
        res->status = *(volatile int *)bar.status;
    }
}

}  // namespace

extern "C" {

int hb_selftest_wait_timeout(hb_context *ctx)
{
    if (!ctx) return HB_ERR_INVALID;
    unsigned *w = hb_bar(ctx);
    hbd::GridBarrier bar;
    bar.count = w;
    bar.gen = w + 1;
    bar.status = (int *)(w + 2);
    hb_solve_result *h = (hb_solve_result *)ctx->pinned;
    bool as_designed = true;
    for (int counter = 0; counter < 2; ++counter) {
        HB_CUDA_TRY(ctx, cudaMemsetAsync(w, 0, 4 * sizeof(unsigned), ctx->stream));
        if (counter) wait_timeout_kernel<true><<<1, 32, 0, ctx->stream>>>(bar, hb_partials(ctx), hb_result(ctx));
        else wait_timeout_kernel<false><<<1, 32, 0, ctx->stream>>>(bar, hb_partials(ctx), hb_result(ctx));
        int st = hb_check_launch(ctx, "wait_timeout_kernel");
        if (st) return st;
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, hb_result(ctx), sizeof(hb_solve_result), cudaMemcpyDeviceToHost,
                                         ctx->stream));
        HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        as_designed = as_designed && h->status == HB_DEV_TIMEOUT && h->used == 0;
    }
    // leave the barrier words clean for the next cooperative launch
    HB_CUDA_TRY(ctx, cudaMemsetAsync(w, 0, 4 * sizeof(unsigned), ctx->stream));
    return as_designed ? HB_ERR_TIMEOUT : HB_ERR_CUDA;
}

int hb_cg_f64(hb_context *ctx, const hb_ell *A, const double *b, double *x, int64_t max_iters,
              double eps, int64_t *used_iters, double *final_defect)
{
    HB_RANGE("hb_cg_f64");
    return cg_impl<double>(ctx, A, b, x, max_iters, eps, used_iters, final_defect, HB_F64);
}

int hb_cg_f32(hb_context *ctx, const hb_ell *A, const float *b, float *x, int64_t max_iters,
              float eps, int64_t *used_iters, float *final_defect)
{
    HB_RANGE("hb_cg_f32");
    return cg_impl<float>(ctx, A, b, x, max_iters, eps, used_iters, final_defect, HB_F32);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Allocation-free CG: hb_cg_f64_noalloc.
//
// For callers that cannot allocate device memory at solve time: real-time or embedded hosts
// that forbid allocation after start-up (an allocation can block for an unbounded time), and
// processes whose device memory is entirely reserved by another framework's caching
// allocator (a cudaMalloc there fails although the memory is idle).  The work vectors, the
// reduction partials, the barrier words and the result record live in one file-scope
// __device__ array instead of a context's cudaMalloc'd workspace.  Every GPU that loads this
// library in a process holds its own copy of the array (NOALLOC_BYTES, about 5.3 MB) until the
// process exits.  Each call copies its result record to the host and synchronises its stream.
// ---------------------------------------------------------------------------------------
namespace {

constexpr int64_t NOALLOC_MAX_ROWS = 131072;       // rows (= ld bound, a multiple of 64)
constexpr int NOALLOC_MAX_BLOCKS = 1024;
constexpr size_t NOALLOC_WORK_BYTES = 5 * (size_t)NOALLOC_MAX_ROWS * sizeof(double);
constexpr size_t NOALLOC_PART_BYTES = 2 * (size_t)NOALLOC_MAX_BLOCKS * sizeof(double);
constexpr size_t NOALLOC_BAR_BYTES = 256;
constexpr size_t NOALLOC_RES_BYTES = 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_WORK_BYTES + NOALLOC_PART_BYTES + NOALLOC_BAR_BYTES + NOALLOC_RES_BYTES;
constexpr int NOALLOC_MAX_DEVICES = 64;

}  // namespace

static __device__ __align__(256) unsigned char hb_cg_noalloc_scratch[NOALLOC_BYTES];

namespace {

// The symbol's device address, looked up per device with that device current.  In host code
// the name hb_cg_noalloc_scratch is only a host-side stand-in; kernels must be given this
// address.  A lookup that fails is not cached: the next call on that device tries again.
struct NoAllocDevice {
    void *base = nullptr;
    int num_sms = 0;
};
NoAllocDevice g_noalloc[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mutex;

int noalloc_setup(int device, NoAllocDevice *out)
{
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return HB_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocDevice &d = g_noalloc[device];
    if (!d.base) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, hb_cg_noalloc_scratch);
        if (e != cudaSuccess || !p) { cudaGetLastError(); return HB_ERR_CUDA; }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess || sms <= 0) { cudaGetLastError(); return HB_ERR_CUDA; }
        d.num_sms = sms;
        d.base = p;
    }
    *out = d;
    return HB_OK;
}

template <int KT>
int noalloc_launch(cudaStream_t stream, int num_sms, CGParams<double> &P, int64_t groups)
{
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, cg_kernel<double, KT>, CG_THREADS, 0) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    const int64_t maxb = (int64_t)std::max(1, occ) * num_sms;
    const int64_t want = (groups + CG_THREADS - 1) / CG_THREADS;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(maxb, NOALLOC_MAX_BLOCKS)));
    void *args[] = {&P};
    if (cudaLaunchCooperativeKernel((const void *)cg_kernel<double, KT>, dim3(blocks), dim3(CG_THREADS), args, 0,
                                    stream) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    return HB_OK;
}

}  // namespace

extern "C" int hb_cg_f64_noalloc(const hb_ell *A, const double *b, double *x, int64_t max_iters, double eps,
                                 int64_t *used_iters, double *final_defect, void *stream_)
{
    if (!A || !b || !x || !used_iters || max_iters < 0) return HB_ERR_INVALID;
    int st = hb_check_ell(A, HB_F64);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    if (A->rows > NOALLOC_MAX_ROWS || A->ld > NOALLOC_MAX_ROWS) return HB_ERR_UNSUPPORTED;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return HB_ERR_CUDA; }
    cudaStream_t stream = (cudaStream_t)stream_;
    if (stream) {
        // the scratch address belongs to the current device: a stream of another device
        // would run the kernel against a foreign device's address
        int sdev = -1;
        if (cudaStreamGetDevice(stream, &sdev) != cudaSuccess) { cudaGetLastError(); return HB_ERR_INVALID; }
        if (sdev != device) return HB_ERR_INVALID;
    }
    NoAllocDevice d;
    st = noalloc_setup(device, &d);
    if (st) return st;
    char *base = (char *)d.base;
    double *work = (double *)base;
    double *partials = (double *)(base + NOALLOC_WORK_BYTES);
    unsigned *bar = (unsigned *)(base + NOALLOC_WORK_BYTES + NOALLOC_PART_BYTES);
    hb_solve_result *res = (hb_solve_result *)(base + NOALLOC_WORK_BYTES + NOALLOC_PART_BYTES + NOALLOC_BAR_BYTES);
    // the barrier words must start at zero; everything else is written before it is read
    if (cudaMemsetAsync(bar, 0, NOALLOC_BAR_BYTES, stream) != cudaSuccess) { cudaGetLastError(); return HB_ERR_CUDA; }
    const int64_t ld = A->ld;
    CGParams<double> P;
    P.rows = A->rows;
    P.ld = ld;
    P.K = (int)A->K;
    P.Aj = A->Aj;
    P.Ax = (const double *)A->Ax;
    P.b_user = b;
    P.x_user = x;
    P.x = work; P.r = work + ld; P.p0 = work + 2 * ld; P.p1 = work + 3 * ld; P.v = work + 4 * ld;
    P.max_iters = max_iters;
    P.eps = eps;
    P.partials = partials;
    P.bar.count = bar;
    P.bar.gen = bar + 1;
    P.bar.status = (int *)(bar + 2);
    P.res = res;
    const int64_t groups = ld / 4;
    st = (A->K == 9) ? noalloc_launch<9>(stream, d.num_sms, P, groups) : noalloc_launch<0>(stream, d.num_sms, P, groups);
    if (st) return st;
    hb_solve_result h;
    if (cudaMemcpyAsync(&h, res, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    if (h.status == HB_DEV_TIMEOUT) return HB_ERR_TIMEOUT;
    *used_iters = h.used;
    if (final_defect) *final_defect = h.defect;
    return HB_OK;
}
