// hb_batch.cu -- many independent SPD-style systems of uneven size in one persistent launch.
//
// One thread-block cluster solves one system at a time: rows are split over the cluster's
// CTAs (4 consecutive rows per thread, as everywhere in this library), the two reductions of
// every CG iteration go through each CTA's shared memory and distributed shared memory
// (DSMEM), and the phases are separated by the hardware cluster barrier instead of a grid
// barrier.  Clusters pull systems from a device work counter; the host orders the systems
// largest first, so the long solves start first (longest-processing-time scheduling).
//
// Every CTA of a cluster sums the CTA partials in rank order, so all of them hold the same
// scalars and take the same branches: control flow is uniform across the cluster, which is
// what makes the hardware cluster barrier safe here.  A system's arithmetic depends only on
// the system and on (cluster size, threads per CTA), never on which cluster runs it or on the
// rest of the batch: results are bit-identical alone and in any mix.
//
// Modes (per system):
//   HB_BATCH_CG64  CGSolver<NONE> (honei/math/cg.hh:63-133) in FP64, reference update
//                  formulas and dual stopping rule, as hb_cg_f64.
//   HB_BATCH_IR32  FP64 iterative refinement (honei/math/ir.hh:30-78 loop shape): FP64 defect,
//                  norm and update; inner CG in FP32 with FP32 accumulation on the normalised
//                  defect (scaled mode) to inner_eps; stop at ||r|| < eps ||r0||.
#include "hb_spmv_core.cuh"

#include <cooperative_groups.h>
#include <algorithm>
#include <cfloat>
#include <numeric>
#include <vector>

namespace cgx = cooperative_groups;

namespace {

struct BatchDesc {
    int64_t n, ld;
    int32_t K, mode;
    const int32_t *Aj;
    const double *Ax64;
    const float *Ax32;
    const double *b;
    double *x;
    char *work;
    int64_t max_iters, max_outer;
    double eps, inner_eps;
    hb_batch_result *res;
};

struct Smem {
    double red64[32];
    float red32[32];
    double slot64[2 * 16];      // [phase][rank]: every CTA's partial, pushed by its owner
    float slot32[2 * 16];
    long long item;
};

template <typename T> __device__ __forceinline__ T *red_of(Smem &s);
template <> __device__ __forceinline__ double *red_of<double>(Smem &s) { return s.red64; }
template <> __device__ __forceinline__ float *red_of<float>(Smem &s) { return s.red32; }
template <typename T> __device__ __forceinline__ T *slot_of(Smem &s);
template <> __device__ __forceinline__ double *slot_of<double>(Smem &s) { return s.slot64; }
template <> __device__ __forceinline__ float *slot_of<float>(Smem &s) { return s.slot32; }

__device__ __forceinline__ double dsqrt(double v) { return __dsqrt_rn(v); }
__device__ __forceinline__ float dsqrt(float v) { return __fsqrt_rn(v); }
template <typename T> __device__ __forceinline__ T eps_mach();
template <> __device__ __forceinline__ double eps_mach<double>() { return DBL_EPSILON; }
template <> __device__ __forceinline__ float eps_mach<float>() { return FLT_EPSILON; }

// Cluster-wide sum in a fixed order (thread partials -> CTA tree -> CTA partials in rank
// order), identical in every CTA.  Each CTA pushes its total into every CTA's slot for its
// rank (DSMEM stores before the cluster barrier), so after the barrier each CTA sums local
// shared memory.  The two slot sets alternate: a set is rewritten only two barriers later,
// after every CTA has read it.
template <typename T> __device__ T cluster_total(T v, Smem &s, int &phase)
{
    v = hbd::block_sum(v, red_of<T>(s));
    cgx::cluster_group cl = cgx::this_cluster();
    const unsigned nb = cl.num_blocks();
    T *slot = slot_of<T>(s) + 16 * phase;
    if (threadIdx.x < 32) {
        // warp 0: the CTA total to every lane; lane q stores it into CTA q's slot of this rank
        v = __shfl_sync(0xffffffffu, v, 0);
        if (threadIdx.x < nb) *cl.map_shared_rank(slot + cl.block_rank(), threadIdx.x) = v;
    }
    cl.sync();
    T t = T(0);
    for (unsigned r = 0; r < nb; ++r) t = hbd::add(t, slot[r]);
    phase ^= 1;
    return t;
}

struct Range {
    int64_t lo, hi;   // row groups of 4 owned by this CTA
};

// The CG loop of honei/math/cg.hh:95-126 on one cluster.  On entry r holds the initial defect,
// x the initial guess (both padded to ld), alpha = r.r (already reduced).  p = beta p + r is
// formed inside the SpMV gather (p double-buffered), exactly as in the grid-wide cg_kernel.
template <typename T, int KT>
__device__ void cluster_cg(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t ld, int K, Range rg,
                           T *x, T *r, T *p0, T *p1, T *v, T alpha, T eps, int64_t max_iters, Smem &s, int &phase,
                           int64_t &used_out, T &d0_out, T &d_out)
{
    using hbd::add; using hbd::mul;
    const T initial_defect = dsqrt(alpha);
    T current_defect = T(0);
    T beta = T(0);
    const T epsm = eps_mach<T>();
    T *pin = p0, *pout = p1;
    int64_t it = 0, used = 0;
    while (it < max_iters) {
        const bool first = (it == 0);
        T acc = T(0);
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            T sm[4];
            const T *rw = r, *pw = pin;
            hbd::ell_rows4<T, KT, 4>(Aj, Ax, ld, K, 4 * g, [&](int32_t j) {
                const T rj = __ldca(rw + j);
                return first ? rj : add(mul(__ldca(pw + j), beta), rj);
            }, sm);
            T rv[4], pv[4], pn[4];
            hbd::ld4(r + 4 * g, rv);
            hbd::ld4(pin + 4 * g, pv);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                pn[i] = first ? rv[i] : add(mul(pv[i], beta), rv[i]);
                acc = add(acc, mul(sm[i], pn[i]));
            }
            hbd::st4(pout + 4 * g, pn);
            hbd::st4(v + 4 * g, sm);
        }
        const T temp = cluster_total<T>(acc, s, phase);
        const T lambda = alpha / (fabs(temp) > epsm ? temp : epsm);
        const T mlambda = -lambda;
        acc = T(0);
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            T xv[4], pv[4], rv[4], vv[4];
            hbd::ld4(x + 4 * g, xv);
            hbd::ld4(pout + 4 * g, pv);
            hbd::ld4(r + 4 * g, rv);
            hbd::ld4(v + 4 * g, vv);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xv[i] = add(xv[i], mul(lambda, pv[i]));
                rv[i] = add(rv[i], mul(mlambda, vv[i]));
                acc = add(acc, mul(rv[i], rv[i]));
            }
            hbd::st4(x + 4 * g, xv);
            hbd::st4(r + 4 * g, rv);
        }
        const T alpha_old = alpha;
        alpha = cluster_total<T>(acc, s, phase);
        beta = alpha / (fabs(alpha_old) > epsm ? alpha_old : epsm);
        T *t = pin; pin = pout; pout = t;
        ++it;
        current_defect = dsqrt(alpha);
        if (current_defect < eps * initial_defect) { used = it; break; }
        if (current_defect < eps) { used = it; break; }
        if (it == max_iters) used = it;
    }
    used_out = used;
    d0_out = initial_defect;
    d_out = current_defect;
}

// The same CG loop with one row per thread instead of a group of four: every slot's Aj / Ax load
// of the row is in flight at once, then every gather, with fewer registers per thread (so more
// threads per SM).  Same formulas, same per-row summation order; the dot products' partial sums
// group the rows differently, so its iterates differ from the four-row layout's at round-off.
template <typename T, int KT>
__device__ void cluster_cg1(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t ld, int K, Range rg,
                            T *x, T *r, T *p0, T *p1, T *v, T alpha, T eps, int64_t max_iters, Smem &s, int &phase,
                            int64_t &used_out, T &d0_out, T &d_out)
{
    using hbd::add; using hbd::mul;
    constexpr int KS = KT > 0 ? KT : 4;
    const T initial_defect = dsqrt(alpha);
    T current_defect = T(0);
    T beta = T(0);
    const T epsm = eps_mach<T>();
    T *pin = p0, *pout = p1;
    int64_t it = 0, used = 0;
    const int64_t lo = 4 * rg.lo, hi = 4 * rg.hi;
    const int kend = KT > 0 ? KT : K;
    while (it < max_iters) {
        const bool first = (it == 0);
        T acc = T(0);
        for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x) {
            T sm = T(0);
            for (int k0 = 0; k0 < kend; k0 += KS) {
                int32_t j[KS];
                T a[KS];
#pragma unroll
                for (int c = 0; c < KS; ++c) {
                    const bool in = k0 + c < kend;
                    j[c] = in ? __ldcs(Aj + (int64_t)(k0 + c) * ld + row) : -1;
                    a[c] = in ? __ldcs(Ax + (int64_t)(k0 + c) * ld + row) : T(0);
                }
                T g[KS];
#pragma unroll
                for (int c = 0; c < KS; ++c) {
                    if (j[c] >= 0) {
                        const T rj = __ldca(r + j[c]);
                        g[c] = first ? rj : add(mul(__ldca(pin + j[c]), beta), rj);
                    } else {
                        g[c] = T(0);
                    }
                }
#pragma unroll
                for (int c = 0; c < KS; ++c)
                    if (j[c] >= 0) sm = add(sm, mul(a[c], g[c]));
            }
            const T rv = r[row];
            const T pn = first ? rv : add(mul(pin[row], beta), rv);
            acc = add(acc, mul(sm, pn));
            pout[row] = pn;
            v[row] = sm;
        }
        const T temp = cluster_total<T>(acc, s, phase);
        const T lambda = alpha / (fabs(temp) > epsm ? temp : epsm);
        const T mlambda = -lambda;
        acc = T(0);
        for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x) {
            const T xv = add(x[row], mul(lambda, pout[row]));
            const T rv = add(r[row], mul(mlambda, v[row]));
            acc = add(acc, mul(rv, rv));
            x[row] = xv;
            r[row] = rv;
        }
        const T alpha_old = alpha;
        alpha = cluster_total<T>(acc, s, phase);
        beta = alpha / (fabs(alpha_old) > epsm ? alpha_old : epsm);
        T *t = pin; pin = pout; pout = t;
        ++it;
        current_defect = dsqrt(alpha);
        if (current_defect < eps * initial_defect) { used = it; break; }
        if (current_defect < eps) { used = it; break; }
        if (it == max_iters) used = it;
    }
    used_out = used;
    d0_out = initial_defect;
    d_out = current_defect;
}

// rv = b - A x over the owned groups (FP64), returns the thread's partial r.r.
template <int KT>
__device__ double defect64(const BatchDesc &d, Range rg, const double *xw, double *rw)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    double acc = 0.0;
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
        double sm[4], rv[4];
        hbd::ell_rows4<double, KT, 4>(d.Aj, d.Ax64, d.ld, d.K, 4 * g, [&](int32_t j) { return __ldca(xw + j); }, sm);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t row = 4 * g + i;
            const double bb = row < d.n ? d.b[row] : 0.0;
            rv[i] = sub(bb, sm[i]);
            acc = add(acc, mul(rv[i], rv[i]));
        }
        hbd::st4(rw + 4 * g, rv);
    }
    return acc;
}

// defect64 with one row per thread (the layout of cluster_cg1): rv = b - A x, the thread's r.r.
template <int KT>
__device__ double defect64_1(const BatchDesc &d, Range rg, const double *xw, double *rw)
{
    using hbd::add; using hbd::mul; using hbd::sub;
    constexpr int KS = KT > 0 ? KT : 4;
    const int kend = KT > 0 ? KT : d.K;
    double acc = 0.0;
    for (int64_t row = 4 * rg.lo + threadIdx.x; row < 4 * rg.hi; row += blockDim.x) {
        double sm = 0.0;
        for (int k0 = 0; k0 < kend; k0 += KS) {
            int32_t j[KS];
            double a[KS];
#pragma unroll
            for (int c = 0; c < KS; ++c) {
                const bool in = k0 + c < kend;
                j[c] = in ? __ldcs(d.Aj + (int64_t)(k0 + c) * d.ld + row) : -1;
                a[c] = in ? __ldcs(d.Ax64 + (int64_t)(k0 + c) * d.ld + row) : 0.0;
            }
            double g[KS];
#pragma unroll
            for (int c = 0; c < KS; ++c) g[c] = j[c] >= 0 ? __ldca(xw + j[c]) : 0.0;
#pragma unroll
            for (int c = 0; c < KS; ++c)
                if (j[c] >= 0) sm = add(sm, mul(a[c], g[c]));
        }
        const double bb = row < d.n ? d.b[row] : 0.0;
        const double rv = sub(bb, sm);
        acc = add(acc, mul(rv, rv));
        rw[row] = rv;
    }
    return acc;
}

template <int KT, int RPT>
__device__ double defect_any(const BatchDesc &d, Range rg, const double *xw, double *rw)
{
    if (RPT == 1) return defect64_1<KT>(d, rg, xw, rw);
    return defect64<KT>(d, rg, xw, rw);
}

template <int KT, int RPT>
__device__ void solve_system(const BatchDesc &d, Smem &s, int &phase)
{
    cgx::cluster_group cl = cgx::this_cluster();
    const unsigned rank = cl.block_rank(), nb = cl.num_blocks();
    const int64_t groups = d.ld / 4;
    const int64_t gpc = (groups + nb - 1) / nb;
    Range rg{(int64_t)rank * gpc, min(groups, (int64_t)(rank + 1) * gpc)};
    const int64_t ld = d.ld;
    double *xw = (double *)d.work;
    double *r64 = xw + ld;
    // x (padded) from the caller; ||b||
    double bb = 0.0;
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
        double xv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t row = 4 * g + i;
            xv[i] = row < d.n ? d.x[row] : 0.0;
            const double bv = row < d.n ? d.b[row] : 0.0;
            bb = hbd::add(bb, hbd::mul(bv, bv));
        }
        hbd::st4(xw + 4 * g, xv);
    }
    const double bnorm = dsqrt(cluster_total<double>(bb, s, phase));   // also orders x before gathers
    hb_batch_result res{};
    if (d.mode == HB_BATCH_CG64) {
        double *p0 = xw + 2 * ld, *p1 = xw + 3 * ld, *v = xw + 4 * ld;
        const double alpha = cluster_total<double>(defect_any<KT, RPT>(d, rg, xw, r64), s, phase);
        int64_t used;
        double d0, d1;
        if (RPT == 1)
            cluster_cg1<double, KT>(d.Aj, d.Ax64, ld, d.K, rg, xw, r64, p0, p1, v, alpha, d.eps, d.max_iters, s, phase,
                                    used, d0, d1);
        else
            cluster_cg<double, KT>(d.Aj, d.Ax64, ld, d.K, rg, xw, r64, p0, p1, v, alpha, d.eps, d.max_iters, s, phase,
                                   used, d0, d1);
        res.iterations = used;
        res.defect0 = d0;
        res.defect = d1;
    } else {
        float *x32 = (float *)(r64 + ld);
        float *r32 = x32 + ld, *q0 = x32 + 2 * ld, *q1 = x32 + 3 * ld, *v32 = x32 + 4 * ld;
        double nrm0 = 0.0, nrm = 0.0;
        int64_t outer = 0, total = 0;
        while (true) {
            nrm = dsqrt(cluster_total<double>(defect_any<KT, RPT>(d, rg, xw, r64), s, phase));
            if (outer == 0) nrm0 = nrm;
            else if (nrm < d.eps * nrm0) break;
            if (nrm == 0.0 || outer >= d.max_outer) break;
            const double sc = 1.0 / nrm;
            float acc = 0.f;
            for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
                double rv[4];
                float rf[4], zf[4] = {0.f, 0.f, 0.f, 0.f};
                hbd::ld4(r64 + 4 * g, rv);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    rf[i] = (float)hbd::mul(rv[i], sc);
                    acc = hbd::add(acc, hbd::mul(rf[i], rf[i]));
                }
                hbd::st4(r32 + 4 * g, rf);
                hbd::st4(x32 + 4 * g, zf);
            }
            const float alpha32 = cluster_total<float>(acc, s, phase);
            int64_t used;
            float d0, d1;
            if (RPT == 1)
                cluster_cg1<float, KT>(d.Aj, d.Ax32, ld, d.K, rg, x32, r32, q0, q1, v32, alpha32, (float)d.inner_eps,
                                       d.max_iters, s, phase, used, d0, d1);
            else
                cluster_cg<float, KT>(d.Aj, d.Ax32, ld, d.K, rg, x32, r32, q0, q1, v32, alpha32, (float)d.inner_eps,
                                      d.max_iters, s, phase, used, d0, d1);
            total += used;
            for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
                double xv[4];
                float cf[4];
                hbd::ld4(xw + 4 * g, xv);
                hbd::ld4(x32 + 4 * g, cf);
#pragma unroll
                for (int i = 0; i < 4; ++i) xv[i] = hbd::add(xv[i], hbd::mul(nrm, (double)cf[i]));
                hbd::st4(xw + 4 * g, xv);
            }
            cl.sync();
            ++outer;
        }
        res.iterations = total;
        res.outer = outer;
        res.defect0 = nrm0;
        res.defect = nrm;
    }
    // x back to the caller and the true FP64 relative residual
    cl.sync();
    const double rr = cluster_total<double>(defect_any<KT, RPT>(d, rg, xw, r64), s, phase);
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x)
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (4 * g + i < d.n) d.x[4 * g + i] = xw[4 * g + i];
    if (rank == 0 && threadIdx.x == 0) {
        res.true_relres = bnorm > 0.0 ? dsqrt(rr) / bnorm : dsqrt(rr);
        res.status = HB_OK;
        *d.res = res;
    }
}

template <int THREADS, int RPT>
__global__ void __launch_bounds__(THREADS, RPT == 1 && THREADS == 256 ? 3 : 0) batch_kernel(const BatchDesc *__restrict__ descs, int64_t count,
                                                        unsigned long long *counter)
{
    __shared__ Smem s;
    cgx::cluster_group cl = cgx::this_cluster();
    int phase = 0;
    while (true) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) s.item = (long long)atomicAdd(counter, 1ull);
        cl.sync();
        const long long item = *cl.map_shared_rank(&s.item, 0);
        cl.sync();
        if (item >= count) break;
        const BatchDesc d = descs[item];
        if (d.K == 9) solve_system<9, RPT>(d, s, phase);
        else solve_system<0, RPT>(d, s, phase);
    }
}

size_t sys_work_bytes(const hb_batch_system &s)
{
    const size_t ld = (size_t)s.A64.ld;
    const size_t b = s.mode == HB_BATCH_CG64 ? 5 * ld * 8 : ld * (8 + 8 + 5 * 4);
    return (b + 255) / 256 * 256;
}

size_t desc_bytes(int64_t count) { return ((size_t)count * sizeof(BatchDesc) + 255) / 256 * 256; }
size_t result_bytes(int64_t count) { return ((size_t)count * sizeof(hb_batch_result) + 255) / 256 * 256; }

int check_system(const hb_batch_system &s)
{
    int st = hb_check_ell(&s.A64, HB_F64);
    if (st) return st;
    if (s.A64.rows != s.A64.cols) return HB_ERR_SIZE;
    if (!s.b || !s.x) return HB_ERR_INVALID;
    if (s.mode != HB_BATCH_CG64 && s.mode != HB_BATCH_IR32) return HB_ERR_INVALID;
    if (s.mode == HB_BATCH_IR32) {
        st = hb_check_ell(&s.A32, HB_F32);
        if (st) return st;
        if (s.A32.rows != s.A64.rows || s.A32.K != s.A64.K || s.A32.ld != s.A64.ld || s.A32.Aj != s.A64.Aj)
            return HB_ERR_SIZE;   // the FP32 copy shares the FP64 matrix's index array
    }
    if (s.max_iters < 0 || s.max_outer < 0) return HB_ERR_INVALID;
    return HB_OK;
}

template <int THREADS, int RPT> int launch_batch(hb_context *ctx, int cluster, int max_clusters, int64_t count, void *ws)
{
    auto kern = batch_kernel<THREADS, RPT>;
    if (cluster > 8) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaFuncSetAttribute(non-portable cluster)"); return HB_ERR_CUDA; }
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(cluster);
    int max_active = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&max_active, kern, &cfg);
    if (e != cudaSuccess || max_active < 1) {
        hb_note_error(ctx, e == cudaSuccess ? cudaErrorInvalidConfiguration : e, "cudaOccupancyMaxActiveClusters");
        return HB_ERR_UNSUPPORTED;
    }
    if (max_clusters > 0) max_active = std::min(max_active, max_clusters);
    const int64_t clusters = std::max<int64_t>(1, std::min<int64_t>(max_active, count));
    cfg.gridDim = dim3((unsigned)(clusters * cluster));
    const BatchDesc *descs = (const BatchDesc *)((char *)ws + 256);
    unsigned long long *counter = (unsigned long long *)ws;
    e = cudaLaunchKernelEx(&cfg, kern, descs, count, counter);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchKernelEx(batch_kernel)"); return HB_ERR_CUDA; }
    return hb_check_launch(ctx, "batch_kernel");
}

int zero_x(hb_context *ctx, const hb_batch_system *sys, int64_t count)
{
    for (int64_t i = 0; i < count; ++i)
        HB_CUDA_TRY(ctx, cudaMemsetAsync(sys[i].x, 0, sizeof(double) * sys[i].A64.rows, ctx->stream));
    return HB_OK;
}

}  // namespace

extern "C" {

int hb_batch_workspace_bytes(const hb_batch_system *sys, int64_t count, size_t *bytes)
{
    if (!bytes || count < 0 || (count > 0 && !sys)) return HB_ERR_INVALID;
    size_t total = 256 + desc_bytes(count) + result_bytes(count);
    for (int64_t i = 0; i < count; ++i) total += sys_work_bytes(sys[i]);
    *bytes = total;
    return HB_OK;
}

int hb_batch_prepare(hb_context *ctx, const hb_batch_system *sys, int64_t count, void *ws)
{
    if (!ctx || !ws || count < 0 || (count > 0 && !sys)) return HB_ERR_INVALID;
    if ((uintptr_t)ws % 256) return HB_ERR_INVALID;
    for (int64_t i = 0; i < count; ++i) {
        int st = check_system(sys[i]);
        if (st) return st;
    }
    // largest systems first; work vectors laid out in that order
    std::vector<int64_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return sys[a].A64.rows > sys[b].A64.rows; });
    char *base = (char *)ws;
    hb_batch_result *results = (hb_batch_result *)(base + 256 + desc_bytes(count));
    char *work = base + 256 + desc_bytes(count) + result_bytes(count);
    std::vector<BatchDesc> d(count);
    for (int64_t k = 0; k < count; ++k) {
        const hb_batch_system &s = sys[order[k]];
        BatchDesc &o = d[k];
        o.n = s.A64.rows;
        o.ld = s.A64.ld;
        o.K = (int32_t)s.A64.K;
        o.mode = s.mode;
        o.Aj = s.A64.Aj;
        o.Ax64 = (const double *)s.A64.Ax;
        o.Ax32 = s.mode == HB_BATCH_IR32 ? (const float *)s.A32.Ax : nullptr;
        o.b = s.b;
        o.x = s.x;
        o.work = work;
        work += sys_work_bytes(s);
        o.max_iters = s.max_iters;
        o.max_outer = s.max_outer;
        o.eps = s.eps;
        o.inner_eps = s.inner_eps;
        o.res = results + order[k];
    }
    if (count) {
        HB_CUDA_TRY(ctx, cudaMemcpyAsync(base + 256, d.data(), count * sizeof(BatchDesc), cudaMemcpyHostToDevice,
                                         ctx->stream));
        HB_CUDA_TRY(ctx, cudaMemsetAsync(results, 0, count * sizeof(hb_batch_result), ctx->stream));
    }
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return HB_OK;
}

int hb_batch_run(hb_context *ctx, int64_t count, void *ws, const hb_batch_config *cfg)
{
    if (!ctx || !ws || count < 0) return HB_ERR_INVALID;
    if (count == 0) return HB_OK;
    const int cluster = cfg ? cfg->cluster : 4;
    const int threads = cfg ? cfg->threads : 512;
    const int max_clusters = cfg ? cfg->max_clusters : 0;
    const int rpt = cfg && cfg->rows_per_thread ? cfg->rows_per_thread : 4;
    if (cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8 && cluster != 16) return HB_ERR_INVALID;
    if (rpt != 1 && rpt != 4) return HB_ERR_INVALID;
    HB_CUDA_TRY(ctx, cudaMemsetAsync(ws, 0, 256, ctx->stream));
    if (threads == 256) return rpt == 1 ? launch_batch<256, 1>(ctx, cluster, max_clusters, count, ws)
                                        : launch_batch<256, 4>(ctx, cluster, max_clusters, count, ws);
    if (threads == 512) return rpt == 1 ? launch_batch<512, 1>(ctx, cluster, max_clusters, count, ws)
                                        : launch_batch<512, 4>(ctx, cluster, max_clusters, count, ws);
    return HB_ERR_INVALID;
}

int hb_batch_results(hb_context *ctx, int64_t count, void *ws, hb_batch_result *results_host)
{
    if (!ctx || !ws || count < 0 || (count > 0 && !results_host)) return HB_ERR_INVALID;
    if (count == 0) return HB_OK;
    const char *base = (const char *)ws;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(results_host, base + 256 + desc_bytes(count), count * sizeof(hb_batch_result),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return HB_OK;
}

int hb_batch_solve(hb_context *ctx, const hb_batch_system *sys, int64_t count, void *ws, const hb_batch_config *cfg,
                   hb_batch_result *results_host)
{
    HB_RANGE("hb_batch_solve");
    int st = hb_batch_prepare(ctx, sys, count, ws);
    if (st) return st;
    st = hb_batch_run(ctx, count, ws, cfg);
    if (st) return st;
    return hb_batch_results(ctx, count, ws, results_host);
}

int hb_batch_tune(hb_context *ctx, const hb_batch_system *sys, int64_t count, void *ws, hb_batch_config *best,
                  double *times_ms)
{
    HB_RANGE("hb_batch_tune");
    if (!ctx || !best) return HB_ERR_INVALID;
    int st = hb_batch_prepare(ctx, sys, count, ws);
    if (st) return st;
    const int clusters[5] = {1, 2, 4, 8, 16};
    const int threads[2] = {256, 512};
    const int rows[2] = {4, 1};
    cudaEvent_t e0, e1;
    HB_CUDA_TRY(ctx, cudaEventCreate(&e0));
    HB_CUDA_TRY(ctx, cudaEventCreate(&e1));
    double best_ms = 1e300;
    int k = 0;
    for (int rpt : rows)
    for (int c : clusters)
        for (int t : threads) {
            hb_batch_config cfg{c, t, 0, rpt};
            float ms = -1.f;
            // warm-up then one timed run, every run from x = 0
            st = zero_x(ctx, sys, count);
            if (!st) st = hb_batch_run(ctx, count, ws, &cfg);
            if (!st) st = zero_x(ctx, sys, count);
            if (!st) {
                cudaEventRecord(e0, ctx->stream);
                st = hb_batch_run(ctx, count, ws, &cfg);
                cudaEventRecord(e1, ctx->stream);
                if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
            }
            if (st == HB_ERR_UNSUPPORTED) { st = HB_OK; ms = -1.f; }
            if (st) break;
            if (times_ms) times_ms[k] = ms;
            if (ms > 0 && ms < best_ms) { best_ms = ms; *best = cfg; }
            ++k;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

}  // extern "C"
