// hb_q1.cu -- device-side multigrid setup for Q1 grids of any side: bilinear transfer matrices
// and Galerkin coarse operators R A P, all in hb_ell layout, built without the host.
//
// Coarsening: the coarse grid of an Mf x Mf grid keeps the fine nodes with even index plus the
// last node (side Mc = Mf/2 + 1; for odd Mf the usual 2:1 coarsening).  Prolongation is the
// bilinear interpolation of Prolongation<Tag, methods::NONE> (honei/math/prolongation.hh:42-139)
// with the fine Dirichlet rows zeroed; restriction is its transpose (the Transposition of
// honei/math/mg.hh:496).  The Galerkin operator replaces rediscretisation so that jumping
// cell coefficients stay convergent; coarse nodes without fine support (the last line of an
// even-sided grid) get identity rows.  Identical, entry for entry, to honei_b200/problems.py
// (prolongation_csr, transpose_csr, galerkin_csr) up to the summation order of R A P.
#include "hb_internal.cuh"

#include <cmath>
#include <vector>

namespace {

__device__ __forceinline__ int64_t coarse_of(int64_t k, int64_t Mf, int64_t Mc)
{
    return k == Mf - 1 ? Mc - 1 : k / 2;
}

// 1-D interpolation of fine coordinate i: up to two (coarse index, weight) pairs, ascending.
__device__ __forceinline__ int interp1(int64_t i, int64_t Mf, int64_t Mc, int64_t (&c)[2], double (&w)[2])
{
    if (i % 2 == 0 || i == Mf - 1) {
        c[0] = coarse_of(i, Mf, Mc);
        w[0] = 1.0;
        return 1;
    }
    c[0] = coarse_of(i - 1, Mf, Mc);
    c[1] = coarse_of(i + 1, Mf, Mc);
    w[0] = w[1] = 0.5;
    return 2;
}

__device__ __forceinline__ bool boundary(int64_t i, int64_t j, int64_t M)
{
    return i == 0 || j == 0 || i == M - 1 || j == M - 1;
}

// P: Nf x Nc, K = 4.  Row f = (fi, fj): products of the 1-D weights, coarse index ascending.
template <typename T>
__global__ void prolongation_kernel(int64_t Mf, int64_t Mc, int64_t ld, int32_t *__restrict__ Aj, T *__restrict__ Ax)
{
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < ld; f += (int64_t)gridDim.x * blockDim.x) {
        int32_t jj[4] = {-1, -1, -1, -1};
        T vv[4] = {T(0), T(0), T(0), T(0)};
        if (f < Mf * Mf) {
            const int64_t fi = f / Mf, fj = f - fi * Mf;
            if (!boundary(fi, fj, Mf)) {
                int64_t ci[2], cj[2];
                double wi[2], wj[2];
                const int ni = interp1(fi, Mf, Mc, ci, wi), nj = interp1(fj, Mf, Mc, cj, wj);
                int k = 0;
                for (int a = 0; a < ni; ++a)
                    for (int b = 0; b < nj; ++b) {
                        jj[k] = (int32_t)(ci[a] * Mc + cj[b]);
                        vv[k] = (T)(wi[a] * wj[b]);
                        ++k;
                    }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            Aj[s * ld + f] = jj[s];
            Ax[s * ld + f] = vv[s];
        }
    }
}

// Weight of coarse index c in fine coordinate i's interpolation (0 if none).
__device__ __forceinline__ double weight_of(int64_t i, int64_t c, int64_t Mf, int64_t Mc)
{
    if (i < 0 || i >= Mf) return 0.0;
    int64_t cc[2];
    double w[2];
    const int n = interp1(i, Mf, Mc, cc, w);
    for (int a = 0; a < n; ++a)
        if (cc[a] == c) return w[a];
    return 0.0;
}

// R = P^T: Nc x Nf, K = 9.  Row c = (ci, cj): fine nodes f near (fc(ci), fc(cj)) with a
// non-zero weight, fine index ascending, fine boundary nodes skipped.
template <typename T>
__global__ void restriction_kernel(int64_t Mf, int64_t Mc, int64_t ld, int32_t *__restrict__ Aj, T *__restrict__ Ax)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ld; c += (int64_t)gridDim.x * blockDim.x) {
        int32_t jj[9];
        T vv[9];
#pragma unroll
        for (int s = 0; s < 9; ++s) { jj[s] = -1; vv[s] = T(0); }
        if (c < Mc * Mc) {
            const int64_t ci = c / Mc, cj = c - ci * Mc;
            const int64_t pi = min(2 * ci, Mf - 1), pj = min(2 * cj, Mf - 1);
            int k = 0;
            for (int a = -1; a <= 1; ++a) {
                const int64_t fi = pi + a;
                const double wa = weight_of(fi, ci, Mf, Mc);
                if (wa == 0.0) continue;
                for (int b = -1; b <= 1; ++b) {
                    const int64_t fj = pj + b;
                    const double wb = weight_of(fj, cj, Mf, Mc);
                    if (wb == 0.0 || boundary(fi, fj, Mf)) continue;
                    jj[k] = (int32_t)(fi * Mf + fj);
                    vv[k] = (T)(wa * wb);
                    ++k;
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 9; ++s) {
            Aj[s * ld + c] = jj[s];
            Ax[s * ld + c] = vv[s];
        }
    }
}

// Galerkin coarse row c of R A P (FP64): sum over the fine rows f that interpolate from c and
// over their stencil entries g of w_f * a_fg * P[g, J], accumulated per coarse neighbour J in a
// fixed order.  J is always within one coarse step of c; a violation sets *bad.
__global__ void galerkin_kernel(int64_t Mf, int64_t Mc, const int32_t *__restrict__ Aj, const double *__restrict__ Ax,
                                int64_t ldf, int Kf, int64_t ldc, int32_t *__restrict__ Cj, double *__restrict__ Cx,
                                int *bad)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ldc; c += (int64_t)gridDim.x * blockDim.x) {
        double acc[9];
#pragma unroll
        for (int s = 0; s < 9; ++s) acc[s] = 0.0;
        const bool live = c < Mc * Mc;
        int64_t ci = 0, cj = 0;
        if (live) {
            ci = c / Mc;
            cj = c - ci * Mc;
            const int64_t pi = min(2 * ci, Mf - 1), pj = min(2 * cj, Mf - 1);
            for (int a = -1; a <= 1; ++a) {
                const int64_t fi = pi + a;
                const double wa = weight_of(fi, ci, Mf, Mc);
                if (wa == 0.0) continue;
                for (int b = -1; b <= 1; ++b) {
                    const int64_t fj = pj + b;
                    const double wb = weight_of(fj, cj, Mf, Mc);
                    if (wb == 0.0 || boundary(fi, fj, Mf)) continue;
                    const double wf = wa * wb;
                    const int64_t f = fi * Mf + fj;
                    for (int k = 0; k < Kf; ++k) {
                        const int32_t g = Aj[k * ldf + f];
                        if (g < 0) continue;
                        const double afg = Ax[k * ldf + f];
                        const int64_t gi = g / Mf, gj = g - gi * Mf;
                        if (boundary(gi, gj, Mf)) continue;
                        int64_t gci[2], gcj[2];
                        double gwi[2], gwj[2];
                        const int ni = interp1(gi, Mf, Mc, gci, gwi), nj = interp1(gj, Mf, Mc, gcj, gwj);
                        for (int p = 0; p < ni; ++p)
                            for (int q = 0; q < nj; ++q) {
                                const int64_t di = gci[p] - ci, dj = gcj[q] - cj;
                                if (di < -1 || di > 1 || dj < -1 || dj > 1) { atomicExch(bad, 1); continue; }
                                acc[(di + 1) * 3 + (dj + 1)] += wf * afg * gwi[p] * gwj[q];
                            }
                    }
                }
            }
        }
        bool any = false;
#pragma unroll
        for (int s = 0; s < 9; ++s) any |= (acc[s] != 0.0);
        if (live && !any) acc[4] = 1.0;   // no fine support: identity row
#pragma unroll
        for (int s = 0; s < 9; ++s) {
            const int64_t di = s / 3 - 1, dj = s % 3 - 1;
            const int64_t Ji = ci + di, Jj = cj + dj;
            const bool in = live && Ji >= 0 && Ji < Mc && Jj >= 0 && Jj < Mc && acc[s] != 0.0;
            Cj[s * ldc + c] = in ? (int32_t)(Ji * Mc + Jj) : -1;
            Cx[s * ldc + c] = in ? acc[s] : 0.0;
        }
    }
}

inline unsigned grid_for(hb_context *ctx, int64_t n)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 16));
}

}  // namespace

extern "C" {

int hb_q1_coarse_side(int64_t Mf) { return (int)(Mf / 2 + 1); }

int hb_q1_transfers(hb_context *ctx, int64_t Mf, hb_ell *P, hb_ell *R)
{
    if (!ctx || !P || !R || Mf < 3) return HB_ERR_INVALID;
    const int64_t Mc = Mf / 2 + 1, Nf = Mf * Mf, Nc = Mc * Mc;
    int64_t K, ld;
    hb_ell_layout(Nf, 4, 1, &K, &ld);
    if (P->K != 4 || P->ld != ld) return HB_ERR_SIZE;
    hb_ell_layout(Nc, 9, 1, &K, &ld);
    if (R->K != 9 || R->ld != ld) return HB_ERR_SIZE;
    P->rows = Nf; P->cols = Nc;
    R->rows = Nc; R->cols = Nf;
    if (P->dtype != R->dtype) return HB_ERR_INVALID;
    int st = hb_check_ell(P, P->dtype);
    if (!st) st = hb_check_ell(R, R->dtype);
    if (st) return st;
    if (P->dtype == HB_F64) {
        prolongation_kernel<double><<<grid_for(ctx, P->ld), 256, 0, ctx->stream>>>(Mf, Mc, P->ld, P->Aj, (double *)P->Ax);
        restriction_kernel<double><<<grid_for(ctx, R->ld), 256, 0, ctx->stream>>>(Mf, Mc, R->ld, R->Aj, (double *)R->Ax);
    } else {
        prolongation_kernel<float><<<grid_for(ctx, P->ld), 256, 0, ctx->stream>>>(Mf, Mc, P->ld, P->Aj, (float *)P->Ax);
        restriction_kernel<float><<<grid_for(ctx, R->ld), 256, 0, ctx->stream>>>(Mf, Mc, R->ld, R->Aj, (float *)R->Ax);
    }
    return hb_check_launch(ctx, "q1 transfer kernels");
}

int hb_q1_galerkin(hb_context *ctx, int64_t Mf, const hb_ell *Af, hb_ell *Ac)
{
    if (!ctx || !Af || !Ac || Mf < 3) return HB_ERR_INVALID;
    int st = hb_check_ell(Af, HB_F64);
    if (st) return st;
    const int64_t Mc = Mf / 2 + 1;
    if (Af->rows != Mf * Mf || Af->cols != Mf * Mf) return HB_ERR_SIZE;
    int64_t K, ld;
    hb_ell_layout(Mc * Mc, 9, 1, &K, &ld);
    if (Ac->K != 9 || Ac->ld != ld) return HB_ERR_SIZE;
    Ac->rows = Ac->cols = Mc * Mc;
    Ac->dtype = HB_F64;
    st = hb_check_ell(Ac, HB_F64);
    if (st) return st;
    int *bad = (int *)hb_scalars(ctx) + 64;   // sticky until the caller clears it
    galerkin_kernel<<<grid_for(ctx, ld), 256, 0, ctx->stream>>>(Mf, Mc, Af->Aj, (const double *)Af->Ax, Af->ld,
                                                                (int)Af->K, ld, Ac->Aj, (double *)Ac->Ax, bad);
    return hb_check_launch(ctx, "galerkin_kernel");
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// hb_q1: one SPD Q1 system resident on the device with everything its solves need -- the FP64
// matrix (Dirichlet couplings eliminated), its FP32 copy (shared index array), the FP32 MG
// hierarchy (device-built transfers and Galerkin levels) and the work vectors.  All memory is
// stream-ordered (cudaMallocAsync / cudaFreeAsync on the context stream), so creating and
// destroying systems never synchronises the device.
// ---------------------------------------------------------------------------------------
struct hb_q1 {
    hb_context *ctx = nullptr;
    int64_t M = 0;
    int L = 0;
    std::vector<int64_t> sides;
    std::vector<hb_ell> A64, A32, P32, R32;
    std::vector<hb_q1band> B32;     // banded copies of the FP32 levels (the cycle's operator)
    std::vector<void *> blocks;
    hb_mg *mg = nullptr;
    double *r64 = nullptr;
    float *b32 = nullptr, *x32 = nullptr, *pcg_work = nullptr;
    double *gj = nullptr;          // Gauss-Jordan workspace n x 2n (coarsest level)
    float *coarse_inv = nullptr;   // exact inverse of the coarsest FP64 matrix, as FP32
    cudaStream_t cap = nullptr;    // private stream for capturing the PCG iteration
    cudaGraphExec_t graph = nullptr;
};

namespace {

template <bool SMEM>
__global__ void dense_inverse_kernel(int64_t n, const int32_t *__restrict__ Aj, const double *__restrict__ Ax,
                                     int64_t ld, int K, double *__restrict__ Wg, float *__restrict__ inv, int *singular);

int q1_alloc(hb_q1 *q, void **p, size_t bytes)
{
    if (cudaMallocAsync(p, bytes ? bytes : 256, q->ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_ALLOC;
    }
    q->blocks.push_back(*p);
    return HB_OK;
}

int q1_ell(hb_q1 *q, int64_t rows, int64_t cols, int64_t ncpr, int dtype, const int32_t *share_Aj, hb_ell *e)
{
    int64_t K, ld;
    hb_ell_layout(rows, ncpr, 1, &K, &ld);
    e->rows = rows;
    e->cols = cols;
    e->K = K;
    e->ld = ld;
    e->dtype = dtype;
    e->pad_ = 0;
    void *p;
    if (share_Aj) {
        e->Aj = const_cast<int32_t *>(share_Aj);
    } else {
        int st = q1_alloc(q, &p, (size_t)K * ld * sizeof(int32_t));
        if (st) return st;
        e->Aj = (int32_t *)p;
    }
    int st = q1_alloc(q, &p, (size_t)K * ld * (dtype == HB_F64 ? 8 : 4));
    if (st) return st;
    e->Ax = p;
    return HB_OK;
}

void q1_free(hb_q1 *q)
{
    if (q->graph) cudaGraphExecDestroy(q->graph);
    if (q->cap) cudaStreamDestroy(q->cap);
    if (q->mg) hb_mg_destroy(q->mg);
    for (void *p : q->blocks) cudaFreeAsync(p, q->ctx->stream);
    delete q;
}

int q1_build(hb_q1 *q, const double *coef)
{
    hb_context *ctx = q->ctx;
    const int L = q->L;
    q->A64.resize(L);
    q->A32.resize(L);
    q->P32.resize(L > 1 ? L - 1 : 0);
    q->R32.resize(L > 1 ? L - 1 : 0);
    int st;
    for (int l = 0; l < L; ++l) {
        const int64_t n = q->sides[l] * q->sides[l];
        if ((st = q1_ell(q, n, n, 9, HB_F64, nullptr, &q->A64[l]))) return st;
        if ((st = q1_ell(q, n, n, 9, HB_F32, q->A64[l].Aj, &q->A32[l]))) return st;
    }
    for (int l = 0; l + 1 < L; ++l) {
        const int64_t nf = q->sides[l + 1] * q->sides[l + 1], nc = q->sides[l] * q->sides[l];
        if ((st = q1_ell(q, nf, nc, 4, HB_F32, nullptr, &q->P32[l]))) return st;
        if ((st = q1_ell(q, nc, nf, 9, HB_F32, nullptr, &q->R32[l]))) return st;
    }
    if ((st = hb_q1_assemble_f64(ctx, q->M, coef, 1, &q->A64[L - 1]))) return st;
    for (int l = L - 1; l > 0; --l)
        if ((st = hb_q1_galerkin(ctx, q->sides[l], &q->A64[l], &q->A64[l - 1]))) return st;
    for (int l = 0; l < L; ++l)
        if ((st = hb_ell_cast_f64_f32(ctx, &q->A64[l], &q->A32[l]))) return st;
    for (int l = 0; l + 1 < L; ++l)
        if ((st = hb_q1_transfers(ctx, q->sides[l + 1], &q->P32[l], &q->R32[l]))) return st;
    hb_mg_params prm{1, 200, 2, 2, 0.7, 1e-6};
    // banded copies of the FP32 levels: the cycle reads no column indices and, with matrix-free
    // transfers, no P / R matrix (hb_mg_create_banded; the same iterates as the ELL cycle)
    q->B32.resize(L);
    for (int l = 0; l < L; ++l) {
        const int64_t nl = q->A32[l].rows, ldb = hb_round_up(nl > 0 ? nl : 1, 4);
        void *bp;
        if ((st = q1_alloc(q, &bp, (size_t)ldb * 9 * 4))) return st;
        hb_q1band &bb = q->B32[l];
        bb = hb_q1band{};
        bb.n = nl;
        bb.dtype = HB_F32;
        for (int k = 0; k < 9; ++k) bb.band[k] = (float *)bp + k * ldb;
        if ((st = hb_q1band_from_ell(ctx, &q->A32[l], &bb))) return st;
    }
    if ((st = hb_mg_create_banded(ctx, L, q->A32.data(), q->B32.data(), &prm, &q->mg))) return st;
    // exact coarse solve: invert the coarsest FP64 Galerkin matrix (at most 81 x 81)
    const int64_t nc = q->A64[0].rows;
    void *p;
    if ((st = q1_alloc(q, &p, (size_t)nc * 2 * nc * 8))) return st;
    q->gj = (double *)p;
    if ((st = q1_alloc(q, &p, (size_t)nc * nc * 4))) return st;
    q->coarse_inv = (float *)p;
    int *singular = (int *)hb_scalars(ctx) + 65;
    HB_CUDA_TRY(ctx, cudaMemsetAsync(singular, 0, sizeof(int), ctx->stream));
    const size_t wbytes = (size_t)nc * 2 * nc * sizeof(double);
    // the cap is process-wide (concurrent builds): one value for every launch
    if (nc <= 128 && wbytes <= 200 * 1024 &&
        cudaFuncSetAttribute(dense_inverse_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
            cudaSuccess) {
        dense_inverse_kernel<true><<<1, 256, wbytes, ctx->stream>>>(nc, q->A64[0].Aj, (const double *)q->A64[0].Ax,
                                                                    q->A64[0].ld, (int)q->A64[0].K, q->gj,
                                                                    q->coarse_inv, singular);
    } else {
        cudaGetLastError();
        dense_inverse_kernel<false><<<1, 256, 0, ctx->stream>>>(nc, q->A64[0].Aj, (const double *)q->A64[0].Ax,
                                                                q->A64[0].ld, (int)q->A64[0].K, q->gj, q->coarse_inv,
                                                                singular);
    }
    if ((st = hb_check_launch(ctx, "dense_inverse_kernel"))) return st;
    hb_mg_set_dense_coarse(q->mg, q->coarse_inv);
    // the coarse levels of the cycle as one single-cluster launch (same arithmetic)
    if ((st = hb_mg_enable_tail(q->mg, HB_TAIL_DEFAULT_ROWS))) return st;
    const int64_t n = q->M * q->M, ldn = hb_round_up(n, 64);
    if ((st = q1_alloc(q, &p, (size_t)ldn * 8))) return st;
    q->r64 = (double *)p;
    if ((st = q1_alloc(q, &p, (size_t)ldn * 4 * 7))) return st;   // b32, x32, r, z, p, v, scalars
    q->b32 = (float *)p;
    q->x32 = q->b32 + ldn;
    q->pcg_work = q->b32 + 2 * ldn;
    if (cudaStreamCreateWithFlags(&q->cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    return HB_OK;
}

// Gauss-Jordan inverse of a small SPD matrix (one block): W = [A | I] in FP64 with partial
// pivoting (the first row of largest magnitude in the column, the row itself first); the inverse
// is stored row-major as FP32.  SMEM: W lives in dynamic shared memory (n <= 81, the coarsest
// level: 105 KB) instead of the global workspace.  The pivot is found by warp 0 (lane l scans
// rows c + l, c + l + 32, ... in order, then a shuffle reduction that keeps the lowest row among
// equal magnitudes), the same row the sequential scan picks.
template <bool SMEM>
__global__ void dense_inverse_kernel(int64_t n, const int32_t *__restrict__ Aj, const double *__restrict__ Ax,
                                     int64_t ld, int K, double *__restrict__ Wg, float *__restrict__ inv, int *singular)
{
    extern __shared__ double Ws[];
    double *W = SMEM ? Ws : Wg;
    __shared__ double fac[128];
    __shared__ int piv;
    const int64_t w = 2 * n;
    for (int64_t i = threadIdx.x; i < n * w; i += blockDim.x) W[i] = 0.0;
    __syncthreads();
    for (int64_t r = threadIdx.x; r < n; r += blockDim.x) {
        for (int k = 0; k < K; ++k) {
            const int32_t j = Aj[k * ld + r];
            if (j >= 0) W[r * w + j] = Ax[k * ld + r];
        }
        W[r * w + n + r] = 1.0;
    }
    __syncthreads();
    for (int64_t c = 0; c < n; ++c) {
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            double best = -1.0;
            int64_t p = n;
            for (int64_t r = c + lane; r < n; r += 32) {
                double v = fabs(W[r * w + c]);
                if (v != v) v = -1.0;                  // a NaN below the diagonal is never chosen
                if (v > best) { best = v; p = r; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_down_sync(0xffffffffu, best, o);
                const int64_t op = __shfl_down_sync(0xffffffffu, p, o);
                if (ob > best || (ob == best && op < p)) { best = ob; p = op; }
            }
            if (lane == 0) {
                const double dc = fabs(W[c * w + c]);
                if (dc != dc || best <= dc) p = c;       // the diagonal wins ties (and a NaN there)
                if (dc == dc && (p == c ? dc : best) == 0.0) *singular = 1;
                piv = (int)p;
            }
        }
        __syncthreads();
        if (piv != c)
            for (int64_t j = threadIdx.x; j < w; j += blockDim.x) {
                const double t = W[c * w + j];
                W[c * w + j] = W[piv * w + j];
                W[piv * w + j] = t;
            }
        __syncthreads();
        const double d = W[c * w + c];
        __syncthreads();
        for (int64_t j = threadIdx.x; j < w; j += blockDim.x) W[c * w + j] = d != 0.0 ? W[c * w + j] / d : 0.0;
        for (int64_t r = threadIdx.x; r < n; r += blockDim.x) fac[r] = W[r * w + c];
        __syncthreads();
        for (int64_t idx = threadIdx.x; idx < n * w; idx += blockDim.x) {
            const int64_t r = idx / w, j = idx - r * w;
            if (r != c) W[idx] -= fac[r] * W[c * w + j];
        }
        __syncthreads();
    }
    for (int64_t idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int64_t r = idx / n, j = idx - r * n;
        inv[idx] = (float)W[r * w + n + j];
    }
}

__global__ void scale_to_f32_kernel(int64_t n, float *__restrict__ dst, const double *__restrict__ src, double s)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (float)__dmul_rn(src[i], s);
}

__global__ void add_scaled_kernel(int64_t n, double *__restrict__ x, const float *__restrict__ c, double a)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(a, (double)c[i]));
}

int q1_norm(hb_context *ctx, int64_t n, const double *v, double *out)
{
    double *slot = hb_scalars(ctx) + 24;
    int st = hb_launch_dot<double>(ctx, n, v, v, slot);
    if (st) return st;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, slot, 8, cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *out = std::sqrt(*(double *)ctx->pinned);
    return HB_OK;
}

}  // namespace

extern "C" {

int hb_q1_create(hb_context *ctx, int64_t M, const double *coef, hb_q1 **out)
{
    HB_RANGE("hb_q1_create");
    if (!ctx || !out || M < 2) return HB_ERR_INVALID;
    if (M * M > INT32_MAX) return HB_ERR_UNSUPPORTED;
    *out = nullptr;
    hb_q1 *q = new hb_q1();
    q->ctx = ctx;
    q->M = M;
    std::vector<int64_t> s{M};
    while (s.back() > 9) s.push_back(s.back() / 2 + 1);
    q->sides.assign(s.rbegin(), s.rend());
    q->L = (int)q->sides.size();
    int st = cudaMemsetAsync((int *)hb_scalars(ctx) + 64, 0, sizeof(int), ctx->stream) == cudaSuccess ? HB_OK
                                                                                                   : HB_ERR_CUDA;
    if (!st) st = q1_build(q, coef);
    if (!st) {
        int h[2] = {0, 0};   // Galerkin stencil violation, singular coarse matrix
        if (cudaMemcpyAsync(h, (int *)hb_scalars(ctx) + 64, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream) !=
                cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            st = HB_ERR_CUDA;
        } else if (h[0] || h[1]) {
            st = HB_ERR_INVALID;
        }
    }
    if (st) {
        q1_free(q);
        return st;
    }
    *out = q;
    return HB_OK;
}

int hb_q1_destroy(hb_q1 *q)
{
    if (!q) return HB_ERR_INVALID;
    q1_free(q);
    return HB_OK;
}

int hb_q1_levels(const hb_q1 *q, int *nlevels, int64_t *sides)
{
    if (!q || !nlevels) return HB_ERR_INVALID;
    *nlevels = q->L;
    if (sides)
        for (int l = 0; l < q->L; ++l) sides[l] = q->sides[l];
    return HB_OK;
}

int hb_q1_level(const hb_q1 *q, int level, hb_ell *A64, hb_ell *A32, hb_ell *P32, hb_ell *R32)
{
    if (!q || level < 0 || level >= q->L) return HB_ERR_INVALID;
    if (A64) *A64 = q->A64[level];
    if (A32) *A32 = q->A32[level];
    if (level + 1 < q->L) {
        if (P32) *P32 = q->P32[level];
        if (R32) *R32 = q->R32[level];
    }
    return HB_OK;
}

}  // extern "C"

int hb_q1_view_of(const hb_q1 *q, hb_q1_view *out)
{
    if (!q || !out || q->L < 1 || q->L > HB_Q1_MAXL) return HB_ERR_INVALID;
    out->L = q->L;
    out->ctx = q->ctx;
    out->A64 = q->A64[q->L - 1];
    if ((int)q->B32.size() != q->L) return HB_ERR_INVALID;
    for (int l = 0; l < q->L; ++l) {
        out->A32[l] = q->A32[l];
        out->B32[l] = q->B32[l];
        if (l + 1 < q->L) {
            out->P32[l] = q->P32[l];
            out->R32[l] = q->R32[l];
        }
    }
    int st = hb_mg_view(q->mg, out);
    if (st) return st;
    if (!out->coarse_inv) return HB_ERR_INVALID;
    const int64_t ldn = q->A64[q->L - 1].ld;
    out->r64 = q->r64;
    out->b32 = q->b32;
    out->x32 = q->x32;
    out->r = q->pcg_work;
    out->z = q->pcg_work + ldn;
    out->p = q->pcg_work + 2 * ldn;
    out->v = q->pcg_work + 3 * ldn;
    return HB_OK;
}

extern "C" {

int hb_q1_set_fused_tail(hb_q1 *q, int64_t max_rows)
{
    if (!q) return HB_ERR_INVALID;
    int st = hb_mg_enable_tail(q->mg, max_rows);
    if (st) return st;
    // the captured PCG iteration holds the old cycle: capture again on the next solve
    if (q->graph) {
        cudaStreamSynchronize(q->ctx->stream);
        cudaGraphExecDestroy(q->graph);
        q->graph = nullptr;
    }
    return HB_OK;
}

int hb_q1_solve(hb_q1 *q, const double *b, double *x, double eps, double inner_eps, int64_t max_outer,
                int64_t max_inner, hb_batch_result *info)
{
    HB_RANGE("hb_q1_solve");
    if (!q || !b || !x || max_outer < 0 || max_inner < 0) return HB_ERR_INVALID;
    hb_context *ctx = q->ctx;
    const hb_ell &A = q->A64[q->L - 1];
    const int64_t n = A.rows;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 16));
    double bnorm, nrm = 0.0, nrm0 = 0.0;
    int st = q1_norm(ctx, n, b, &bnorm);
    int64_t outer = 0, inner = 0;
    while (!st) {
        st = hb_launch_spmv_mode<double>(ctx, &A, HB_MODE_DEFECT, x, b, nullptr, q->r64);
        if (!st) st = q1_norm(ctx, n, q->r64, &nrm);
        if (st) break;
        if (outer == 0) nrm0 = nrm;
        else if (nrm < eps * nrm0) break;
        if (nrm == 0.0 || outer >= max_outer) break;
        scale_to_f32_kernel<<<blocks, 256, 0, ctx->stream>>>(n, q->b32, q->r64, 1.0 / nrm);
        if ((st = hb_check_launch(ctx, "scale_to_f32_kernel"))) break;
        int64_t used = 0;
        if ((st = hb_mg_pcg_f32_graph(q->mg, q->cap, q->b32, q->x32, (float)inner_eps, max_inner, q->pcg_work,
                                      &q->graph, 4, &used)))
            break;
        inner += used;
        add_scaled_kernel<<<blocks, 256, 0, ctx->stream>>>(n, x, q->x32, nrm);
        if ((st = hb_check_launch(ctx, "add_scaled_kernel"))) break;
        ++outer;
    }
    if (st) return st;
    if (info) {
        info->iterations = inner;
        info->outer = outer;
        info->defect0 = nrm0;
        info->defect = nrm;
        info->true_relres = bnorm > 0.0 ? nrm / bnorm : nrm;
        info->status = HB_OK;
    }
    return HB_OK;
}

}  // extern "C"
