// hb_q1batch.cu -- many served Q1 systems (hb_q1) solved in one persistent launch, one
// thread-block cluster per system at a time.
//
// Each cluster runs the algorithm of hb_q1_solve for its system: FP64 iterative refinement
// (defect, norm, scaled FP32 right-hand side, update) around FP32 CG preconditioned by one
// V(n_pre, n_post) cycle -- damped Jacobi sweeps x' = x + P (b - A x), defect, restriction R,
// zero coarse start, the exact dense solve on the coarsest level, prolongation added with P,
// post-smoothing; the levels are the system's banded FP32 copies and the transfers are
// matrix-free, as in the served solve -- with every kernel replaced by a phase of the cluster:
// the rows of each level are split over the cluster's CTAs (4 consecutive rows per thread), a
// hardware cluster barrier separates phases that read other CTAs' rows, and the dot products are
// fixed-order reductions through each CTA's shared memory and distributed shared memory.  Every
// elementwise and per-row formula rounds as the served solve's kernels do; only the dot products'
// summation order differs from the grid-wide reductions.  A system's arithmetic depends on the
// system and the launch shape only, so results are bit-identical alone and in any mix.
//
// Vectors written inside the kernel are read through L2 (ld.global.cg): a CTA's L1 does not see
// other CTAs' writes.  Clusters take systems largest first from a device counter; the systems'
// matrices, hierarchy and vectors are the hb_q1 objects' own, so nothing is allocated per
// request beyond the descriptor table.
#include "hb_spmv_core.cuh"

#include <cooperative_groups.h>
#include <algorithm>
#include <numeric>
#include <vector>

namespace cgx = cooperative_groups;

namespace {

// A level's banded FP32 matrix (nine bands LL .. UU, root = grid side).
struct QBand {
    int64_t n, root;
    const float *b[9];
};

struct QLevel {
    int64_t n, ld, side;   // rows, padded vector length, grid side (coarser side = side / 2 + 1)
    QBand A;
    const float *jac;
    float *c, *d, *store, *xt;
};

struct QSys {
    int L, n_pre, n_post;
    QLevel lv[HB_Q1_MAXL];
    const float *inv;
    int64_t n, ld;
    int K;
    const int32_t *Aj;
    const double *Ax64;
    const double *b;
    double *x, *r64;
    float *b32, *x32, *r, *z, *p, *v;
    double eps, inner_eps;
    int64_t max_outer, max_inner;
    hb_batch_result *res;
};

struct QSmem {
    double red64[32];
    float red32[32];
    double slot64[2 * 16];      // [phase][rank]: every CTA's partial, pushed by its owner
    float slot32[2 * 16];
    long long item;
};

template <typename T> __device__ __forceinline__ T *red_of(QSmem &s);
template <> __device__ __forceinline__ double *red_of<double>(QSmem &s) { return s.red64; }
template <> __device__ __forceinline__ float *red_of<float>(QSmem &s) { return s.red32; }
template <typename T> __device__ __forceinline__ T *slot_of(QSmem &s);
template <> __device__ __forceinline__ double *slot_of<double>(QSmem &s) { return s.slot64; }
template <> __device__ __forceinline__ float *slot_of<float>(QSmem &s) { return s.slot32; }

// Cluster-wide sum in a fixed order (thread partials -> CTA tree -> CTA partials in rank
// order), the same in every CTA; its cluster barrier also orders the phase's writes before
// the next phase's reads.  Each CTA pushes its total into every CTA's slot for its rank (DSMEM
// stores before the barrier), so after it each CTA sums local shared memory; the two slot sets
// alternate, a set being rewritten only two barriers later.
template <typename T> __device__ __forceinline__ T cluster_total(T v, QSmem &s, int &phase)
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

__device__ __forceinline__ void csync() { cgx::this_cluster().sync(); }

// 4 values through L2 (16-byte aligned)
__device__ __forceinline__ void ldcg4(const float *p, float (&v)[4])
{
    const float4 t = __ldcg(reinterpret_cast<const float4 *>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ldcg4(const double *p, double (&v)[4])
{
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Row groups of 4 owned by this CTA for a vector of ld entries.
struct Range {
    int64_t lo, hi;
};
__device__ __forceinline__ Range range_of(int64_t ld)
{
    cgx::cluster_group cl = cgx::this_cluster();
    const int64_t groups = ld / 4, nb = cl.num_blocks(), rank = cl.block_rank();
    const int64_t per = (groups + nb - 1) / nb;
    return Range{rank * per, min(groups, (rank + 1) * per)};
}

// s = A x on rows r0..r0+3 of a banded level, the nine bands summed in ascending column order
// (the ELL row's order: bit-identical to the ELL product of the same matrix); rows >= n give 0.
__device__ __forceinline__ void band_rows4(const QBand &B, int64_t r0, const float *x, float (&s)[4])
{
    using hbd::add; using hbd::mul;
    const int64_t n = B.n, root = B.root;
    float a[9][4];
    if (r0 + 4 <= n) {
#pragma unroll
        for (int k = 0; k < 9; ++k) hbd::ld4_stream(B.b[k] + r0, a[k]);
    } else {
#pragma unroll
        for (int k = 0; k < 9; ++k)
#pragma unroll
            for (int i = 0; i < 4; ++i) a[k][i] = (r0 + i < n) ? B.b[k][r0 + i] : 0.f;
    }
    float lo[6], mid[6], hi[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const int64_t jl = r0 - root - 1 + t, jm = r0 - 1 + t, jh = r0 + root - 1 + t;
        lo[t] = (jl >= 0 && jl < n) ? __ldca(x + jl) : 0.f;
        mid[t] = (jm >= 0 && jm < n) ? __ldca(x + jm) : 0.f;
        hi[t] = (jh >= 0 && jh < n) ? __ldca(x + jh) : 0.f;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t r = r0 + i;
        float v = 0.f;
        if (r < n) {
            if (r - root - 1 >= 0) v = add(v, mul(a[0][i], lo[i]));
            if (r - root >= 0) v = add(v, mul(a[1][i], lo[i + 1]));
            if (r - root + 1 >= 0) v = add(v, mul(a[2][i], lo[i + 2]));
            if (r - 1 >= 0) v = add(v, mul(a[3][i], mid[i]));
            v = add(v, mul(a[4][i], mid[i + 1]));
            if (r + 1 < n) v = add(v, mul(a[5][i], mid[i + 2]));
            if (r + root - 1 < n) v = add(v, mul(a[6][i], hi[i]));
            if (r + root < n) v = add(v, mul(a[7][i], hi[i + 1]));
            if (r + root + 1 < n) v = add(v, mul(a[8][i], hi[i + 2]));
        }
        s[i] = v;
    }
}

__device__ __forceinline__ bool fine_boundary(int64_t R, int64_t C, int64_t Mf)
{
    return R == 0 || C == 0 || R == Mf - 1 || C == Mf - 1;
}

// (P c)[k] for fine node k of a grid of side Mf (coarse side Mc): the bilinear interpolation with
// Dirichlet fine rows zero, summed over coarse nodes in ascending order (the PROLMAT row).
__device__ __forceinline__ float prolong_row(int64_t k, int64_t Mf, int64_t Mc, const float *c)
{
    using hbd::add; using hbd::mul;
    const int64_t R = k / Mf, C = k - R * Mf;
    float s = 0.f;
    if (fine_boundary(R, C, Mf)) return s;
    int64_t ri[2], ci[2];
    float wr[2], wc[2];
    int nr, nc;
    if (R & 1) { ri[0] = (R - 1) / 2; ri[1] = (R + 1) / 2; wr[0] = wr[1] = 0.5f; nr = 2; }
    else { ri[0] = R / 2; wr[0] = 1.f; nr = 1; }
    if (C & 1) { ci[0] = (C - 1) / 2; ci[1] = (C + 1) / 2; wc[0] = wc[1] = 0.5f; nc = 2; }
    else { ci[0] = C / 2; wc[0] = 1.f; nc = 1; }
    for (int a = 0; a < nr; ++a)
        for (int q = 0; q < nc; ++q) s = add(s, mul(wr[a] * wc[q], __ldca(c + ri[a] * Mc + ci[q])));
    return s;
}

// (P^T f)[k] for coarse node k: fine nodes in ascending order (the transposed PROLMAT row).
__device__ __forceinline__ float restrict_row(int64_t k, int64_t Mf, int64_t Mc, const float *f)
{
    using hbd::add; using hbd::mul;
    const int64_t r = k / Mc, c = k - r * Mc;
    float s = 0.f;
    for (int64_t R = 2 * r - 1; R <= 2 * r + 1; ++R) {
        if (R < 0 || R >= Mf) continue;
        const float wr = (R == 2 * r) ? 1.f : 0.5f;
        for (int64_t C = 2 * c - 1; C <= 2 * c + 1; ++C) {
            if (C < 0 || C >= Mf || fine_boundary(R, C, Mf)) continue;
            const float wc = (C == 2 * c) ? 1.f : 0.5f;
            s = add(s, mul(wr * wc, __ldca(f + R * Mf + C)));
        }
    }
    return s;
}

// One damped Jacobi sweep out = x + jac (b - A x) on a level (ell_spmv_kernel, HB_MODE_JACOBI).
__device__ __forceinline__ void jacobi(const QLevel &lv, const float *x, const float *b, float *out)
{
    const Range rg = range_of(lv.ld);
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
        float s[4], xx[4], bb[4], pp[4], o[4];
        band_rows4(lv.A, 4 * g, x, s);
        ldcg4(x + 4 * g, xx);
        ldcg4(b + 4 * g, bb);
        ldcg4(lv.jac + 4 * g, pp);
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = hbd::add(xx[i], hbd::mul(pp[i], hbd::sub(bb[i], s[i])));
        hbd::st4(out + 4 * g, o);
    }
}

// sweeps x -> xt -> x ...; the result ends in x (an odd count copies back)
__device__ __forceinline__ void smooth(const QLevel &lv, float *x, const float *b, int sweeps)
{
    float *cur = x, *other = lv.xt;
    for (int s = 0; s < sweeps; ++s) {
        jacobi(lv, cur, b, other);
        csync();
        float *t = cur; cur = other; other = t;
    }
    if (cur != x) {
        const Range rg = range_of(lv.ld);
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            float v[4];
            ldcg4(cur + 4 * g, v);
            hbd::st4(x + 4 * g, v);
        }
        csync();
    }
}

// z = M(r): one V-cycle from zero (z must be zero on entry), the hb_mg vcycle recursion unrolled.
__device__ __forceinline__ void vcycle(const QSys &S, float *z, const float *r)
{
    const int top = S.L - 1;
    auto X = [&](int l) -> float * { return l == top ? z : S.lv[l].c; };
    auto B = [&](int l) -> const float * { return l == top ? r : S.lv[l].d; };
    for (int l = top; l >= 1; --l) {
        const QLevel &lv = S.lv[l];
        smooth(lv, X(l), B(l), S.n_pre);
        {   // store = B - A X
            const Range rg = range_of(lv.ld);
            const float *x = X(l), *b = B(l);
            for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
                float s[4], bb[4], o[4];
                band_rows4(lv.A, 4 * g, x, s);
                ldcg4(b + 4 * g, bb);
#pragma unroll
                for (int i = 0; i < 4; ++i) o[i] = hbd::sub(bb[i], s[i]);
                hbd::st4(lv.store + 4 * g, o);
            }
        }
        csync();
        {   // d_{l-1} = R store; c_{l-1} = 0
            const QLevel &cv = S.lv[l - 1];
            const Range rg = range_of(cv.ld);
            const float *st = lv.store;
            for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
                float s[4], zero[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    s[i] = (4 * g + i < cv.n) ? restrict_row(4 * g + i, lv.side, cv.side, st) : 0.f;
                hbd::st4(cv.d + 4 * g, s);
                hbd::st4(cv.c + 4 * g, zero);
            }
        }
        csync();
    }
    {   // coarsest level: X(0) = inv B(0), one thread per row, j in order
        const QLevel &l0 = S.lv[0];
        cgx::cluster_group cl = cgx::this_cluster();
        const int64_t n0 = l0.n;
        float *x0 = X(0);
        const float *b0 = B(0);
        const int64_t tid = (int64_t)cl.block_rank() * blockDim.x + threadIdx.x, nt = (int64_t)cl.num_blocks() * blockDim.x;
        for (int64_t i = tid; i < n0; i += nt) {
            float acc = 0.f;
            for (int64_t j = 0; j < n0; ++j) acc = hbd::add(acc, hbd::mul(__ldg(S.inv + i * n0 + j), __ldcg(b0 + j)));
            x0[i] = acc;
        }
    }
    csync();
    for (int l = 1; l <= top; ++l) {
        const QLevel &lv = S.lv[l];
        {   // X += P c_{l-1}
            const Range rg = range_of(lv.ld);
            const float *c = X(l - 1);
            float *x = X(l);
            const int64_t Mc = S.lv[l - 1].side;
            for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
                float s[4], xx[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) s[i] = (4 * g + i < lv.n) ? prolong_row(4 * g + i, lv.side, Mc, c) : 0.f;
                ldcg4(x + 4 * g, xx);
#pragma unroll
                for (int i = 0; i < 4; ++i) xx[i] = hbd::add(xx[i], s[i]);
                hbd::st4(x + 4 * g, xx);
            }
        }
        csync();
        smooth(lv, X(l), B(l), S.n_post);
    }
}

// FP32 PCG on the finest level from x32 = 0 (the served solve's device-scalar PCG).
__device__ __forceinline__ int64_t pcg(const QSys &S, QSmem &sm, int &phase)
{
    const QLevel &top = S.lv[S.L - 1];
    const Range rg = range_of(S.ld);
    float *x = S.x32, *r = S.r, *z = S.z, *p = S.p, *v = S.v;
    const float eps = (float)S.inner_eps;
    // x = 0, r = b, z = 0, rr = r.r
    float acc = 0.f;
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
        float bb[4], zero[4] = {0.f, 0.f, 0.f, 0.f};
        ldcg4(S.b32 + 4 * g, bb);
#pragma unroll
        for (int i = 0; i < 4; ++i) acc = hbd::add(acc, hbd::mul(bb[i], bb[i]));
        hbd::st4(x + 4 * g, zero);
        hbd::st4(r + 4 * g, bb);
        hbd::st4(z + 4 * g, zero);
    }
    float rr = cluster_total<float>(acc, sm, phase);
    const float r0 = sqrtf(rr);
    if (!(r0 > 0.f)) return 0;
    vcycle(S, z, r);
    // p = z, rz = r.z
    acc = 0.f;
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
        float zz[4], rv[4];
        ldcg4(z + 4 * g, zz);
        ldcg4(r + 4 * g, rv);
        hbd::st4(p + 4 * g, zz);
#pragma unroll
        for (int i = 0; i < 4; ++i) acc = hbd::add(acc, hbd::mul(rv[i], zz[i]));
    }
    float rz = cluster_total<float>(acc, sm, phase);
    int64_t it = 0;
    while (it < S.max_inner) {
        // v = A p, pv = p.v
        acc = 0.f;
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            float s[4], pp[4];
            band_rows4(top.A, 4 * g, p, s);
            ldcg4(p + 4 * g, pp);
            hbd::st4(v + 4 * g, s);
#pragma unroll
            for (int i = 0; i < 4; ++i) acc = hbd::add(acc, hbd::mul(pp[i], s[i]));
        }
        const float pv = cluster_total<float>(acc, sm, phase);
        if (!(pv > 0.f)) break;
        const float a = rz / pv, ma = -a;
        // x += a p; r -= a v; rr = r.r; z = 0
        acc = 0.f;
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            float xx[4], pp[4], rv[4], vv[4], zero[4] = {0.f, 0.f, 0.f, 0.f};
            ldcg4(x + 4 * g, xx);
            ldcg4(p + 4 * g, pp);
            ldcg4(r + 4 * g, rv);
            ldcg4(v + 4 * g, vv);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xx[i] = hbd::add(xx[i], hbd::mul(a, pp[i]));
                rv[i] = hbd::add(rv[i], hbd::mul(ma, vv[i]));
                acc = hbd::add(acc, hbd::mul(rv[i], rv[i]));
            }
            hbd::st4(x + 4 * g, xx);
            hbd::st4(r + 4 * g, rv);
            hbd::st4(z + 4 * g, zero);
        }
        rr = cluster_total<float>(acc, sm, phase);
        ++it;
        if (sqrtf(rr) < eps * r0) break;
        vcycle(S, z, r);
        // rz_new = r.z; p = beta p + z
        acc = 0.f;
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            float zz[4], rv[4];
            ldcg4(z + 4 * g, zz);
            ldcg4(r + 4 * g, rv);
#pragma unroll
            for (int i = 0; i < 4; ++i) acc = hbd::add(acc, hbd::mul(rv[i], zz[i]));
        }
        const float rz_new = cluster_total<float>(acc, sm, phase);
        const float beta = rz_new / rz;
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            float zz[4], pp[4];
            ldcg4(z + 4 * g, zz);
            ldcg4(p + 4 * g, pp);
#pragma unroll
            for (int i = 0; i < 4; ++i) pp[i] = hbd::add(hbd::mul(beta, pp[i]), zz[i]);
            hbd::st4(p + 4 * g, pp);
        }
        rz = rz_new;
        csync();
    }
    return it;
}

// r64 = b - A64 x (FP64), returns the thread's partial r.r
__device__ __forceinline__ double defect64(const QSys &S, Range rg)
{
    double acc = 0.0;
    const double *xw = S.x;
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
        double s[4], rv[4];
        hbd::ell_rows4<double, 0, 4>(S.Aj, S.Ax64, S.ld, S.K, 4 * g, [&](int32_t j) { return __ldca(xw + j); }, s);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t row = 4 * g + i;
            const double bb = row < S.n ? __ldcg(S.b + row) : 0.0;
            rv[i] = hbd::sub(bb, s[i]);
            acc = hbd::add(acc, hbd::mul(rv[i], rv[i]));
        }
        hbd::st4(S.r64 + 4 * g, rv);
    }
    return acc;
}

__device__ __forceinline__ void solve_q1(const QSys &S, QSmem &sm, int &phase)
{
    cgx::cluster_group cl = cgx::this_cluster();
    const Range rg = range_of(S.ld);
    // ||b||
    double bb = 0.0;
    for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t row = 4 * g + i;
            const double v = row < S.n ? __ldcg(S.b + row) : 0.0;
            bb = hbd::add(bb, hbd::mul(v, v));
        }
    const double bnorm = sqrt(cluster_total<double>(bb, sm, phase));
    double nrm = 0.0, nrm0 = 0.0;
    int64_t outer = 0, inner = 0;
    while (true) {
        nrm = sqrt(cluster_total<double>(defect64(S, rg), sm, phase));
        if (outer == 0) nrm0 = nrm;
        else if (nrm < S.eps * nrm0) break;
        if (nrm == 0.0 || outer >= S.max_outer) break;
        const double sc = 1.0 / nrm;
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            double rv[4];
            float bf[4];
            ldcg4(S.r64 + 4 * g, rv);
#pragma unroll
            for (int i = 0; i < 4; ++i) bf[i] = (float)hbd::mul(rv[i], sc);
            hbd::st4(S.b32 + 4 * g, bf);
        }
        csync();
        inner += pcg(S, sm, phase);
        // x += nrm * x32 (own rows of the caller's unpadded x)
        for (int64_t g = rg.lo + threadIdx.x; g < rg.hi; g += blockDim.x) {
            float cf[4];
            ldcg4(S.x32 + 4 * g, cf);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t row = 4 * g + i;
                if (row < S.n) S.x[row] = hbd::add(__ldcg(S.x + row), hbd::mul(nrm, (double)cf[i]));
            }
        }
        csync();
        ++outer;
    }
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
        hb_batch_result res{};
        res.iterations = inner;
        res.outer = outer;
        res.defect0 = nrm0;
        res.defect = nrm;
        res.true_relres = bnorm > 0.0 ? nrm / bnorm : nrm;
        res.status = HB_OK;
        *S.res = res;
    }
    csync();
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) q1batch_kernel(const QSys *__restrict__ systems, int64_t count,
                                                          unsigned long long *counter)
{
    __shared__ QSmem s;
    cgx::cluster_group cl = cgx::this_cluster();
    int phase = 0;
    while (true) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) s.item = (long long)atomicAdd(counter, 1ull);
        cl.sync();
        const long long item = *cl.map_shared_rank(&s.item, 0);
        cl.sync();
        if (item >= count) break;
        solve_q1(systems[item], s, phase);
    }
}


int build_levels(const hb_q1_view &v, int L, QSys &S);

int build(const hb_q1_view &v, const double *b, double *x, double eps, double inner_eps, int64_t max_outer,
          int64_t max_inner, hb_batch_result *res, QSys &S)
{
    S = QSys{};
    int st = build_levels(v, v.L, S);
    if (st) return st;
    S.n = v.A64.rows;
    S.ld = v.A64.ld;
    S.K = (int)v.A64.K;
    S.Aj = v.A64.Aj;
    S.Ax64 = (const double *)v.A64.Ax;
    S.b = b;
    S.x = x;
    S.r64 = v.r64;
    S.b32 = v.b32;
    S.x32 = v.x32;
    S.r = v.r;
    S.z = v.z;
    S.p = v.p;
    S.v = v.v;
    S.eps = eps;
    S.inner_eps = inner_eps;
    S.max_outer = max_outer;
    S.max_inner = max_inner;
    S.res = res;
    if (S.ld != S.lv[v.L - 1].ld) return HB_ERR_SIZE;
    return HB_OK;
}

// Levels 0..L-1 of a view into S (banded FP32 levels, Jacobi diagonals, vectors, coarse inverse).
int build_levels(const hb_q1_view &v, int L, QSys &S)
{
    S.L = L;
    S.n_pre = v.n_pre;
    S.n_post = v.n_post;
    for (int l = 0; l < L; ++l) {
        QLevel &q = S.lv[l];
        const hb_q1band &bb = v.B32[l];
        q.n = v.A32[l].rows;
        q.ld = v.A32[l].ld;
        q.side = bb.root;
        if (bb.n != q.n || bb.root * bb.root != q.n || bb.dtype != HB_F32) return HB_ERR_SIZE;
        if (l > 0 && S.lv[l - 1].side != q.side / 2 + 1) return HB_ERR_SIZE;
        q.A.n = bb.n;
        q.A.root = bb.root;
        for (int k = 0; k < 9; ++k) {
            q.A.b[k] = (const float *)bb.band[k];
            if (!q.A.b[k] || ((uintptr_t)q.A.b[k] & 15)) return HB_ERR_INVALID;
        }
        q.jac = v.jac[l];
        q.c = v.c[l];
        q.d = v.d[l];
        q.store = v.store[l];
        q.xt = v.xt[l];
    }
    S.inv = v.coarse_inv;
    if (!S.inv) return HB_ERR_INVALID;
    return HB_OK;
}

// The coarse part of a served system's cycle in one launch: one cluster runs the V-cycle of
// levels 0..S.L-1 (S.L - 1 = the fused top level) on X = z (zero on entry) and B = r.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) q1_tail_kernel(const QSys *__restrict__ S, float *z, const float *r)
{
    vcycle(*S, z, r);
}

constexpr int TAIL_CLUSTER = 16, TAIL_THREADS = 256;

template <int THREADS> int launch(hb_context *ctx, int cluster, int max_clusters, const QSys *sys, int64_t count,
                                  unsigned long long *counter)
{
    auto kern = q1batch_kernel<THREADS>;
    if (cluster > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_UNSUPPORTED;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(THREADS);
    cfg.stream = ctx->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(cluster);
    int max_active = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&max_active, kern, &cfg);
    if (e != cudaSuccess || max_active < 1) {
        cudaGetLastError();
        return HB_ERR_UNSUPPORTED;
    }
    if (max_clusters > 0) max_active = std::min(max_active, max_clusters);
    const int64_t clusters = std::max<int64_t>(1, std::min<int64_t>(max_active, count));
    cfg.gridDim = dim3((unsigned)(clusters * cluster));
    e = cudaLaunchKernelEx(&cfg, kern, sys, count, counter);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchKernelEx(q1batch_kernel)"); return HB_ERR_CUDA; }
    return hb_check_launch(ctx, "q1batch_kernel");
}

}  // namespace

int hb_tail_create(hb_context *ctx, const hb_q1_view &v, int top, void **desc)
{
    if (!ctx || !desc || top < 1 || top >= v.L) return HB_ERR_INVALID;
    QSys S{};
    int st = build_levels(v, top + 1, S);
    if (st) return st;
    S.n_pre = v.n_pre;
    S.n_post = v.n_post;
    void *d = nullptr;
    if (cudaMallocAsync(&d, sizeof(QSys), ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_ALLOC;
    }
    if (cudaMemcpyAsync(d, &S, sizeof(QSys), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(d, ctx->stream);
        return HB_ERR_CUDA;
    }
    if (TAIL_CLUSTER > 8 &&
        cudaFuncSetAttribute(q1_tail_kernel<TAIL_THREADS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(d, ctx->stream);
        return HB_ERR_UNSUPPORTED;
    }
    *desc = d;
    return HB_OK;
}

int hb_tail_launch(hb_context *ctx, const void *desc, float *z, const float *r)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = TAIL_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(TAIL_CLUSTER);
    cfg.blockDim = dim3(TAIL_THREADS);
    cfg.stream = ctx->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, q1_tail_kernel<TAIL_THREADS>, (const QSys *)desc, z, r);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "cudaLaunchKernelEx(q1_tail_kernel)"); return HB_ERR_CUDA; }
    return hb_check_launch(ctx, "q1_tail_kernel");
}

extern "C" {

int hb_q1_batch_solve(hb_context *ctx, hb_q1 *const *systems, const double *const *b, double *const *x, int64_t count,
                      double eps, double inner_eps, int64_t max_outer, int64_t max_inner, const hb_batch_config *cfg,
                      hb_batch_result *results)
{
    HB_RANGE("hb_q1_batch_solve");
    if (!ctx || count < 0 || (count > 0 && (!systems || !b || !x || !results))) return HB_ERR_INVALID;
    if (max_outer < 0 || max_inner < 0) return HB_ERR_INVALID;
    if (count == 0) return HB_OK;
    const int cluster = cfg ? cfg->cluster : 8;
    const int threads = cfg ? cfg->threads : 256;
    const int max_clusters = cfg ? cfg->max_clusters : 0;
    if (cluster < 1 || cluster > 16 || (threads != 256 && threads != 512)) return HB_ERR_INVALID;
    std::vector<QSys> host((size_t)count);
    std::vector<int64_t> order((size_t)count);
    for (int64_t i = 0; i < count; ++i) {
        for (int64_t j = 0; j < i; ++j)
            if (systems[j] == systems[i]) return HB_ERR_INVALID;   // one cluster per system at a time
    }
    std::vector<int64_t> rows((size_t)count);
    for (int64_t i = 0; i < count; ++i) {
        hb_q1_view v;
        int st = hb_q1_view_of(systems[i], &v);
        if (st) return st;
        if (!b[i] || !x[i]) return HB_ERR_INVALID;
        order[i] = i;
        rows[i] = v.A64.rows;
    }
    // largest first (longest-processing-time order)
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t c) { return rows[a] > rows[c]; });
    const size_t sys_bytes = ((size_t)count * sizeof(QSys) + 255) / 256 * 256;
    const size_t res_bytes = ((size_t)count * sizeof(hb_batch_result) + 255) / 256 * 256;
    void *mem = nullptr;
    if (cudaMallocAsync(&mem, sys_bytes + res_bytes + 256, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_ALLOC;
    }
    QSys *dsys = (QSys *)mem;
    hb_batch_result *dres = (hb_batch_result *)((char *)mem + sys_bytes);
    unsigned long long *counter = (unsigned long long *)((char *)mem + sys_bytes + res_bytes);
    int st = HB_OK;
    for (int64_t k = 0; k < count && !st; ++k) {
        const int64_t i = order[k];
        hb_q1_view v;
        hb_q1_view_of(systems[i], &v);
        st = build(v, b[i], x[i], eps, inner_eps, max_outer, max_inner, dres + i, host[k]);
    }
    if (!st && cudaMemcpyAsync(dsys, host.data(), (size_t)count * sizeof(QSys), cudaMemcpyHostToDevice, ctx->stream) !=
                   cudaSuccess)
        st = HB_ERR_CUDA;
    if (!st && cudaMemsetAsync(counter, 0, sizeof(unsigned long long), ctx->stream) != cudaSuccess) st = HB_ERR_CUDA;
    if (!st) st = threads == 256 ? launch<256>(ctx, cluster, max_clusters, dsys, count, counter)
                                 : launch<512>(ctx, cluster, max_clusters, dsys, count, counter);
    if (!st && cudaMemcpyAsync(results, dres, (size_t)count * sizeof(hb_batch_result), cudaMemcpyDeviceToHost,
                               ctx->stream) != cudaSuccess)
        st = HB_ERR_CUDA;
    cudaFreeAsync(mem, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && !st) st = HB_ERR_CUDA;
    cudaGetLastError();
    return st;
}

}  // extern "C"
