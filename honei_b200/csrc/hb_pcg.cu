// hb_pcg.cu -- CGSolver<Tag, methods::VAR> (honei/math/cg.hh:140-219): CG with a
// preconditioner container P, either a vector (Jacobi: Product(z, P, r) is the element product)
// or an ELL matrix (SPAI / SAINV approximate inverses: z = P r), as one persistent cooperative
// kernel.
//
// Reference iteration (after r = b - A x, p = P r, d0 = ||r||, alpha_new = r.p):
//   v = A p;  lambda = alpha_new / guard(v.p);  x += lambda p;  r += (-lambda) v;
//   stop when ||r|| < eps d0, ||r|| < eps or at max_iters;
//   z = P r;  alpha = alpha_new;  alpha_new = r.z;  p = p * (alpha_new / guard(alpha)) + z
// with guard(t) = |t| > eps_mach ? t : eps_mach * (t / |t|) (the sign-keeping form of this
// solver).  Per iteration on the device:
//   phase 1  p = p * t + z for every gathered column (z = P r recomputed from r for a vector
//            P, read for a matrix P), v = A p, partial v.p
//   phase 2  x += lambda p; r += (-lambda) v; partial r.r (vector P: also z = P r and r.z)
//   phase 3  (matrix P only) z = P r, partial r.z
// separated by bounded grid-wide exchanges on an arrival counter; every block sums the partials in one fixed order, so all
// blocks hold the same scalars and take the same branches.  Elementwise formulas round as the
// reference's operator sequence (ScaledSum, Scale, Sum, ElementProduct); the dot products use
// the fixed-order tree of the plain CG kernel.
#include "hb_resident.cuh"

#include <cfloat>

namespace {

constexpr int PCG_THREADS = 256;

template <typename T> struct PCGParams {
    int64_t rows, ld;
    int K;
    const int32_t *Aj;
    const T *Ax;
    const T *Pd;                // vector preconditioner (padded view of the caller's), or null
    int64_t Pld;
    int PK;
    const int32_t *Pj;          // matrix preconditioner, or null
    const T *Px;
    const T *b_user;
    T *x_user;
    T *x, *r, *p0, *p1, *v, *z; // padded work vectors, ld entries each
    int64_t max_iters;
    T eps;
    T *partials;                // 3 * gridDim.x
    hbd::GridBarrier bar;
    hb_solve_result *res;
};

template <typename T> __device__ __forceinline__ T eps_mach();
template <> __device__ __forceinline__ double eps_mach<double>() { return DBL_EPSILON; }
template <> __device__ __forceinline__ float eps_mach<float>() { return FLT_EPSILON; }
__device__ __forceinline__ double dsqrt(double v) { return __dsqrt_rn(v); }
__device__ __forceinline__ float dsqrt(float v) { return __fsqrt_rn(v); }

// The sign-keeping division guard of CGSolver<VAR> (cg.hh:172, 206).
template <typename T> __device__ __forceinline__ T guard(T t)
{
    const T e = eps_mach<T>();
    return fabs(t) > e ? t : e * (t / fabs(t));
}

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

template <typename T, int KT, bool PMAT>
__global__ void __launch_bounds__(PCG_THREADS) pcg_var_kernel(PCGParams<T> P)
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
    T *slotA = P.partials, *slotB = P.partials + G, *slotC = P.partials + 2 * G;
    // grid-wide reductions on the arrival counter; no slot is written at two consecutive
    // exchanges (A; B, C; A; B (C); [C;] A ...), so fixed slot arrays suffice
    const hbd::CountExchange X{P.bar.count, P.bar.status};
    unsigned e = 0;
    const int64_t rows = P.rows;
    bool ok = true;

    // z = P r on the thread's own rows (matrix P: a gathered product of the current r)
    auto precon4 = [&](const uint32_t (&row)[4], const T (&rv)[4], T (&zv)[4]) {
        if (PMAT) {
            const T *rw = P.r;
            hbd::ell_rows4s<T, 0>(P.Pj, P.Px, P.Pld, P.PK, row, [&](int32_t j) { return rw[j]; }, zv);
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) zv[i] = mul(P.Pd[row[i]], rv[i]);
        }
    };

    for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
        T xv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) xv[i] = (row[i] < rows) ? P.x_user[row[i]] : T(0);
        for (int i = 0; i < 4; ++i) P.x[row[i]] = xv[i];
    }
    ok = X.arrive(e++, G, &s_flag);

    // r = b - A x (Defect)
    T rr = T(0), rp = T(0);
    if (ok) {
        const T *xw = P.x;
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T s[4], rv[4];
            hbd::ell_rows4s<T, KT, (KT > 0 ? 3 : 4)>(P.Aj, P.Ax, P.ld, P.K, row, [&](int32_t j) { return xw[j]; }, s);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const T bb = (row[i] < rows) ? P.b_user[row[i]] : T(0);
                rv[i] = sub(bb, s[i]);
            }
            for (int i = 0; i < 4; ++i) P.r[row[i]] = rv[i];
            if (!PMAT) {
                // p = P r, ||r||^2, r.p
                T pv[4];
                precon4(row, rv, pv);
                for (int i = 0; i < 4; ++i) P.p0[row[i]] = pv[i];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    rr = add(rr, mul(rv[i], rv[i]));
                    rp = add(rp, mul(rv[i], pv[i]));
                }
            }
        }
        ok = X.arrive(e++, G, &s_flag);
    }
    if (PMAT && ok) {
        // p = P r needs every row of r
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T rv[4], pv[4];
            for (int i = 0; i < 4; ++i) rv[i] = P.r[row[i]];
            precon4(row, rv, pv);
            for (int i = 0; i < 4; ++i) P.p0[row[i]] = pv[i];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                rr = add(rr, mul(rv[i], rv[i]));
                rp = add(rp, mul(rv[i], pv[i]));
            }
        }
    }
    rr = hbd::block_sum(rr, red);
    if (threadIdx.x == 0) slotB[blockIdx.x] = rr;
    rp = hbd::block_sum(rp, red);
    if (threadIdx.x == 0) slotC[blockIdx.x] = rp;
    if (ok) ok = X.arrive(e++, G, &s_flag);
    const T initial_defect = ok ? dsqrt(grid_total(slotB, red, &bcast)) : T(0);
    T alpha_new = ok ? grid_total(slotC, red, &bcast) : T(0);
    T current_defect = T(0);
    T talpha = T(0);
    T *pin = P.p0, *pout = P.p1;
    int64_t it = 0, used = 0;
    while (ok && it < P.max_iters) {
        // ---- phase 1: p = p * talpha + z (after the first iteration), v = A p, v.p
        const bool first = (it == 0);
        const T *pw = pin, *rw = P.r, *zw = P.z, *dw = P.Pd;
        T acc = T(0);
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T s[4];
            hbd::ell_rows4s<T, KT, (KT > 0 ? 3 : 4)>(P.Aj, P.Ax, P.ld, P.K, row, [&](int32_t j) {
                const T pj = pw[j];
                if (first) return pj;
                const T zj = PMAT ? zw[j] : mul(dw[j], rw[j]);
                return add(mul(pj, talpha), zj);
            }, s);
            T pv[4], pn[4];
            for (int i = 0; i < 4; ++i) pv[i] = pin[row[i]];
            if (first) {
#pragma unroll
                for (int i = 0; i < 4; ++i) pn[i] = pv[i];
            } else {
                T zv[4];
                if (PMAT) {
                    for (int i = 0; i < 4; ++i) zv[i] = P.z[row[i]];
                } else {
                    T rv[4];
                    for (int i = 0; i < 4; ++i) rv[i] = P.r[row[i]];
                    precon4(row, rv, zv);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) pn[i] = add(mul(pv[i], talpha), zv[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) acc = add(acc, mul(s[i], pn[i]));
            for (int i = 0; i < 4; ++i) pout[row[i]] = pn[i];
            for (int i = 0; i < 4; ++i) P.v[row[i]] = s[i];
        }
        acc = hbd::block_sum(acc, red);
        if (threadIdx.x == 0) slotA[blockIdx.x] = acc;
        if (!X.arrive(e++, G, &s_flag)) break;
        const T temp = grid_total(slotA, red, &bcast);
        const T lambda = alpha_new / guard(temp);
        const T mlambda = -lambda;

        // ---- phase 2: x += lambda p; r += (-lambda) v; r.r (vector P: z = P r, r.z)
        rr = T(0);
        T rz = T(0);
        for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
            T xv[4], pv[4], rv[4], vv[4];
            for (int i = 0; i < 4; ++i) xv[i] = P.x[row[i]];
            for (int i = 0; i < 4; ++i) pv[i] = pout[row[i]];
            for (int i = 0; i < 4; ++i) rv[i] = P.r[row[i]];
            for (int i = 0; i < 4; ++i) vv[i] = P.v[row[i]];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xv[i] = add(xv[i], mul(pv[i], lambda));
                rv[i] = add(rv[i], mul(vv[i], mlambda));
                rr = add(rr, mul(rv[i], rv[i]));
            }
            for (int i = 0; i < 4; ++i) P.x[row[i]] = xv[i];
            for (int i = 0; i < 4; ++i) P.r[row[i]] = rv[i];
            if (!PMAT) {
                T zv[4];
                precon4(row, rv, zv);
#pragma unroll
                for (int i = 0; i < 4; ++i) rz = add(rz, mul(rv[i], zv[i]));
            }
        }
        rr = hbd::block_sum(rr, red);
        if (threadIdx.x == 0) slotB[blockIdx.x] = rr;
        if (!PMAT) {
            rz = hbd::block_sum(rz, red);
            if (threadIdx.x == 0) slotC[blockIdx.x] = rz;
        }
        if (!X.arrive(e++, G, &s_flag)) break;
        ++it;
        current_defect = dsqrt(grid_total(slotB, red, &bcast));
        if (current_defect < P.eps * initial_defect) { used = it; break; }
        if (current_defect < P.eps) { used = it; break; }
        if (it == P.max_iters) { used = it; break; }

        // ---- phase 3 (matrix P): z = P r, r.z
        if (PMAT) {
            rz = T(0);
            for (int64_t g = g_lo + threadIdx.x; g < g_hi; g += blockDim.x) {
            uint32_t row[4];
            hbd::quad_rows(g, groups, row);
                T rv[4], zv[4];
                for (int i = 0; i < 4; ++i) rv[i] = P.r[row[i]];
                precon4(row, rv, zv);
                for (int i = 0; i < 4; ++i) P.z[row[i]] = zv[i];
#pragma unroll
                for (int i = 0; i < 4; ++i) rz = add(rz, mul(rv[i], zv[i]));
            }
            rz = hbd::block_sum(rz, red);
            if (threadIdx.x == 0) slotC[blockIdx.x] = rz;
            if (!X.arrive(e++, G, &s_flag)) break;
        }
        const T alpha = alpha_new;
        alpha_new = grid_total(slotC, red, &bcast);
        talpha = alpha_new / guard(alpha);
        T *t = pin; pin = pout; pout = t;
    }
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
// Resident-operator form for a vector (Jacobi) preconditioner, on systems whose rows fit the
// shared memory of one block per SM (hb_resident.cuh): the block's ELL rows, x and v of its rows,
// and r, p and the preconditioner's diagonal on its column window stay in shared memory for the
// whole solve.  p = p * t + P r is formed redundantly on the window (bit for bit what its owner
// forms), so only r crosses blocks, through its halo.  Per iteration two arrival-counter
// exchanges: v.p, then (r.r, r.z) together.  The arithmetic per element is the streaming
// kernel's; the dot products use the resident reduction tree.
// ---------------------------------------------------------------------------------------
template <typename T> struct PCGResParams {
    PCGParams<T> c;
    int64_t rpb, wcap;
    hbd::CountExchange X;
};

template <typename T, int KT>
__global__ void __launch_bounds__(hbr::RES_THREADS, 1) pcg_res_kernel(const PCGResParams<T> Q)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    extern __shared__ __align__(16) unsigned char res_smem[];
    __shared__ T red[32];
    __shared__ T bcast[3];
    __shared__ int s_flag, s_min, s_max;
    const PCGParams<T> &P = Q.c;
    const int K = KT > 0 ? KT : P.K;
    const int64_t rpb = Q.rpb, wcap = Q.wcap;
    const unsigned G = gridDim.x;
    T *Ax_s = (T *)res_smem;                    // [K][rpb]
    T *r_w = Ax_s + (int64_t)K * rpb;           // [wcap]
    T *p_w = r_w + wcap;                        // [wcap]
    T *d_w = p_w + wcap;                        // [wcap] preconditioner diagonal
    T *x_s = d_w + wcap;                        // [rpb]
    T *v_s = x_s + rpb;                         // [rpb]
    int32_t *Aj_s = (int32_t *)(v_s + rpb);     // [K][rpb]
    const hbr::ResWindow win = hbr::res_stage<T, KT>(P.Aj, P.Ax, P.ld, P.K, P.rows, rpb, wcap, Ax_s, Aj_s, &s_min, &s_max);
    const int64_t lo = win.lo, wlo = win.wlo, W = win.W, own = win.own();
    const int nr = win.nr;
    for (int64_t w = threadIdx.x; w < W; w += blockDim.x) d_w[w] = P.Pd[wlo + w];
    __syncthreads();
    auto slots = [&](unsigned e) { return P.partials + (e & 1u) * 2u * G; };

    // r = b - A x (Defect); p = P r; ||r||^2 and r.p
    T rr = T(0), rp = T(0);
    for (int il = threadIdx.x; il < nr; il += blockDim.x) {
        T s = T(0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int32_t c = Aj_s[(int64_t)k * rpb + il];
            if (c == -1) continue;
            s = add(s, mul(Ax_s[(int64_t)k * rpb + il], P.x_user[hbr::res_column(c, wlo)]));
        }
        const T r = sub(P.b_user[lo + il], s);
        const T z = mul(d_w[own + il], r);
        r_w[own + il] = r;
        x_s[il] = P.x_user[lo + il];
        __stcg(P.r + lo + il, r);
        __stcg(P.p0 + lo + il, z);
        rr = add(rr, mul(r, r));
        rp = add(rp, mul(r, z));
    }
    rr = hbr::res_partial(rr, red);
    if (threadIdx.x == 0) __stcg(slots(0) + blockIdx.x, rr);
    __syncthreads();
    rp = hbr::res_partial(rp, red);
    unsigned e = 0;
    if (threadIdx.x == 0) __stcg(slots(0) + G + blockIdx.x, rp);
    bool ok = Q.X.arrive_synced(e, G, &s_flag);
    T pv[hbr::RES_MAX_BLOCKS / 32], pz[hbr::RES_MAX_BLOCKS / 32];
    T initial_defect = T(0), alpha_new = T(0);
    if (ok) {
        hbr::res_total_load(slots(e), G, pv);
        hbr::res_total_load(slots(e) + G, G, pz);
        hbr::res_halo(P.r, r_w, win);
        initial_defect = dsqrt(hbr::res_total_sum(G, pv, &bcast[0]));
        alpha_new = hbr::res_total_sum(G, pz, &bcast[1]);
        for (int64_t w = threadIdx.x; w < W; w += blockDim.x) p_w[w] = mul(d_w[w], r_w[w]);
        __syncthreads();
    }
    T current_defect = T(0);
    T talpha = T(0);
    T *pin = P.p0, *pout = P.p1;
    int64_t it = 0, used = 0;
    while (ok && it < P.max_iters) {
        // ---- phase 1: p = p * talpha + P r on the window (after the first iteration), v = A p, v.p
        const bool first = (it == 0);
        if (!first) {
            for (int64_t w = threadIdx.x; w < W; w += blockDim.x) p_w[w] = add(mul(p_w[w], talpha), mul(d_w[w], r_w[w]));
            __syncthreads();
        }
        T acc = T(0);
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
                    pj = __ldca(pin + j);
                    if (!first) pj = add(mul(pj, talpha), mul(__ldca(P.Pd + j), __ldca(P.r + j)));
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
        if (threadIdx.x == 0) __stcg(slots(e) + blockIdx.x, acc);
        if (!Q.X.arrive_synced(e, G, &s_flag)) break;
        hbr::res_total_load(slots(e), G, pv);
        const T temp = hbr::res_total_sum(G, pv, &bcast[2]);
        const T lambda = alpha_new / guard(temp);
        const T mlambda = -lambda;

        // ---- phase 2: x += p lambda; r += v (-lambda); r.r and r.z (z = P r)
        rr = T(0);
        T rz = T(0);
        for (int il = threadIdx.x; il < nr; il += blockDim.x) {
            x_s[il] = add(x_s[il], mul(p_w[own + il], lambda));
            const T r = add(r_w[own + il], mul(v_s[il], mlambda));
            r_w[own + il] = r;
            __stcg(P.r + lo + il, r);
            rr = add(rr, mul(r, r));
            rz = add(rz, mul(r, mul(d_w[own + il], r)));
        }
        rr = hbr::res_partial(rr, red);
        ++e;
        if (threadIdx.x == 0) __stcg(slots(e) + blockIdx.x, rr);
        __syncthreads();
        rz = hbr::res_partial(rz, red);
        if (threadIdx.x == 0) __stcg(slots(e) + G + blockIdx.x, rz);
        if (!Q.X.arrive_synced(e, G, &s_flag)) break;
        hbr::res_total_load(slots(e), G, pv);
        hbr::res_total_load(slots(e) + G, G, pz);
        hbr::res_halo(P.r, r_w, win);
        ++it;
        current_defect = dsqrt(hbr::res_total_sum(G, pv, &bcast[0]));
        const T rz_total = hbr::res_total_sum(G, pz, &bcast[1]);
        if (current_defect < P.eps * initial_defect) { used = it; break; }
        if (current_defect < P.eps) { used = it; break; }
        if (it == P.max_iters) { used = it; break; }
        const T alpha = alpha_new;
        alpha_new = rz_total;
        talpha = alpha_new / guard(alpha);
        T *t = pin; pin = pout; pout = t;
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
int launch_pcg_res(hb_context *ctx, PCGParams<T> &P, bool *launched)
{
    *launched = false;
    hbr::ResPlan plan;
    if (!hbr::res_plan<T>(ctx, P.rows, KT > 0 ? KT : P.K, 3, 2, (const void *)pcg_res_kernel<T, KT>, &plan))
        return HB_OK;
    PCGResParams<T> Q;
    Q.c = P;
    Q.rpb = plan.rpb;
    Q.wcap = plan.wcap;
    Q.X.count = P.bar.count;
    Q.X.status = P.bar.status;
    void *args[] = {&Q};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)pcg_res_kernel<T, KT>, dim3(plan.blocks),
                                                dim3(hbr::RES_THREADS), args, plan.smem, ctx->stream);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchCooperativeKernel(pcg_res_kernel)"); return HB_ERR_CUDA; }
    *launched = true;
    return hb_check_launch(ctx, "pcg_res_kernel");
}

template <typename T, int KT, bool PMAT>
int launch_pcg(hb_context *ctx, PCGParams<T> &P, int64_t groups)
{
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pcg_var_kernel<T, KT, PMAT>, PCG_THREADS, 0);
    const int64_t maxb = (int64_t)std::max(1, occ) * ctx->num_sms;
    const int64_t want = (groups + PCG_THREADS - 1) / PCG_THREADS;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(maxb, 2048)));
    void *args[] = {&P};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)pcg_var_kernel<T, KT, PMAT>, dim3(blocks),
                                                dim3(PCG_THREADS), args, 0, ctx->stream);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchCooperativeKernel(pcg_var_kernel)"); return HB_ERR_CUDA; }
    return hb_check_launch(ctx, "pcg_var_kernel");
}

template <typename T>
int pcg_impl(hb_context *ctx, const hb_ell *A, const T *Pd, const hb_ell *Pm, const T *b, T *x, int64_t max_iters,
             T eps, int64_t *used_iters, T *final_defect, int dtype)
{
    if (!ctx || !A || !b || !x || !used_iters || max_iters < 0 || (!Pd && !Pm)) return HB_ERR_INVALID;
    int st = hb_check_ell(A, dtype);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    if (Pm) {
        if ((st = hb_check_ell(Pm, dtype))) return st;
        if (Pm->rows != A->rows || Pm->cols != A->cols) return HB_ERR_SIZE;
    }
    const int64_t ld = A->ld, n = A->rows;
    // work: x, r, p0, p1, v, z and (vector P) a zero-padded copy of P
    st = hb_ensure_work(ctx, (size_t)ld * sizeof(T) * 7);
    if (st) return st;
    T *w = (T *)ctx->work;
    PCGParams<T> P;
    P.rows = n;
    P.ld = ld;
    P.K = (int)A->K;
    P.Aj = A->Aj;
    P.Ax = (const T *)A->Ax;
    P.x = w; P.r = w + ld; P.p0 = w + 2 * ld; P.p1 = w + 3 * ld; P.v = w + 4 * ld; P.z = w + 5 * ld;
    P.Pd = nullptr; P.Pj = nullptr; P.Px = nullptr; P.Pld = 0; P.PK = 0;
    if (Pd) {
        T *pd = w + 6 * ld;
        HB_CUDA_TRY(ctx, cudaMemsetAsync(pd + n, 0, (size_t)(ld - n) * sizeof(T), ctx->stream));
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(pd, Pd, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
        P.Pd = pd;
    } else {
        P.Pj = Pm->Aj; P.Px = (const T *)Pm->Ax; P.Pld = Pm->ld; P.PK = (int)Pm->K;
        if (Pm->ld != ld) return HB_ERR_SIZE;
    }
    P.b_user = b;
    P.x_user = x;
    P.max_iters = max_iters;
    P.eps = eps;
    P.partials = (T *)hb_partials(ctx);
    unsigned *bar = hb_bar(ctx);
    P.bar.count = bar;
    P.bar.gen = bar + 1;
    P.bar.status = (int *)(bar + 2);
    P.res = hb_result(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), ctx->stream));
    const int64_t groups = ld / 4;
    const bool k9 = (A->K == 9);
    if (Pd && ctx->cg_resident && groups > 0) {
        bool launched = false;
        st = k9 ? launch_pcg_res<T, 9>(ctx, P, &launched) : launch_pcg_res<T, 0>(ctx, P, &launched);
        if (!st && !launched) st = k9 ? launch_pcg<T, 9, false>(ctx, P, groups) : launch_pcg<T, 0, false>(ctx, P, groups);
    } else if (Pd) st = k9 ? launch_pcg<T, 9, false>(ctx, P, groups) : launch_pcg<T, 0, false>(ctx, P, groups);
    else st = k9 ? launch_pcg<T, 9, true>(ctx, P, groups) : launch_pcg<T, 0, true>(ctx, P, groups);
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

extern "C" {

int hb_cg_var_diag_f64(hb_context *ctx, const hb_ell *A, const double *P, const double *b, double *x,
                       int64_t max_iters, double eps, int64_t *used_iters, double *final_defect)
{
    HB_RANGE("hb_cg_var_diag_f64");
    return pcg_impl<double>(ctx, A, P, nullptr, b, x, max_iters, eps, used_iters, final_defect, HB_F64);
}

int hb_cg_var_diag_f32(hb_context *ctx, const hb_ell *A, const float *P, const float *b, float *x,
                       int64_t max_iters, float eps, int64_t *used_iters, float *final_defect)
{
    HB_RANGE("hb_cg_var_diag_f32");
    return pcg_impl<float>(ctx, A, P, nullptr, b, x, max_iters, eps, used_iters, final_defect, HB_F32);
}

int hb_cg_var_ell_f64(hb_context *ctx, const hb_ell *A, const hb_ell *P, const double *b, double *x,
                      int64_t max_iters, double eps, int64_t *used_iters, double *final_defect)
{
    HB_RANGE("hb_cg_var_ell_f64");
    return pcg_impl<double>(ctx, A, nullptr, P, b, x, max_iters, eps, used_iters, final_defect, HB_F64);
}

int hb_cg_var_ell_f32(hb_context *ctx, const hb_ell *A, const hb_ell *P, const float *b, float *x,
                      int64_t max_iters, float eps, int64_t *used_iters, float *final_defect)
{
    HB_RANGE("hb_cg_var_ell_f32");
    return pcg_impl<float>(ctx, A, nullptr, P, b, x, max_iters, eps, used_iters, final_defect, HB_F32);
}

}  // extern "C"
