// hb_mgband.cu -- matrix-free pieces of the multigrid cycle on Q1 grids whose level matrices are
// banded (BandedMatrixQx<Q1Type> layout, hb_q1band).  A fine grid of side Mf has the coarse side
// Mf / 2 + 1 (2:1 for odd sides; for even sides the last coarse line has no fine support): on
// interior fine nodes the bilinear interpolation is the same for both.
//
//   (the level operator in the fused ELL modes is q1band_kernel's ELL-order variant,
//   hb_q1band.cu: the nine bands summed in ascending column order, LL, LD, LU, DL, DD, DU, UL,
//   UD, UU, the order of the same matrix's ELL row; a band entry the ELL row does not store is
//   zero and adds an exact zero, so the result is bit-identical to the ELL kernel)
//   prolong_add_kernel  y += P c with P the bilinear interpolation whose Dirichlet (boundary)
//                     fine rows are zero, the PROLMAT matrix of honei/math/prolongation.hh:42-139
//                     semantics, summed over coarse nodes in ascending index order (its ELL row).
//   restrict_kernel   d = P^T f summed over fine nodes in ascending index order (the ELL row of the
//                     transposed matrix, honei/math/mg.hh:496).
//
// Per fine row the cycle then reads nine values and three x windows (no column indices), and the
// transfers read the two vectors only -- no P or R matrix.
#include "hb_internal.cuh"

namespace {

__device__ __forceinline__ bool fine_boundary(int64_t R, int64_t C, int64_t Mf)
{
    return R == 0 || C == 0 || R == Mf - 1 || C == Mf - 1;
}

// y += P c (fine side Mf, coarse side Mc = Mf / 2 + 1)
template <typename T>
__global__ void prolong_add_kernel(int64_t Mf, int64_t Mc, T *__restrict__ y, const T *__restrict__ c)
{
    using hbd::add; using hbd::mul;
    const int64_t nf = Mf * Mf;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nf; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t R = k / Mf, C = k - R * Mf;
        T s = T(0);
        if (!fine_boundary(R, C, Mf)) {
            // coarse rows / columns touching this fine node, ascending, with 1-D weights
            int64_t ri[2], ci[2];
            T wr[2], wc[2];
            int nr, nc;
            if (R & 1) { ri[0] = (R - 1) / 2; ri[1] = (R + 1) / 2; wr[0] = wr[1] = T(0.5); nr = 2; }
            else { ri[0] = R / 2; wr[0] = T(1); nr = 1; }
            if (C & 1) { ci[0] = (C - 1) / 2; ci[1] = (C + 1) / 2; wc[0] = wc[1] = T(0.5); nc = 2; }
            else { ci[0] = C / 2; wc[0] = T(1); nc = 1; }
            for (int a = 0; a < nr; ++a)
                for (int q = 0; q < nc; ++q) s = add(s, mul(wr[a] * wc[q], c[ri[a] * Mc + ci[q]]));
        }
        y[k] = add(y[k], s);
    }
}

// d = P^T f
template <typename T>
__global__ void restrict_kernel(int64_t Mf, int64_t Mc, T *__restrict__ d, const T *__restrict__ f)
{
    using hbd::add; using hbd::mul;
    const int64_t nc = Mc * Mc;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nc; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = k / Mc, c = k - r * Mc;
        T s = T(0);
        for (int64_t R = 2 * r - 1; R <= 2 * r + 1; ++R) {
            if (R < 0 || R >= Mf) continue;
            const T wr = (R == 2 * r) ? T(1) : T(0.5);
            for (int64_t C = 2 * c - 1; C <= 2 * c + 1; ++C) {
                if (C < 0 || C >= Mf || fine_boundary(R, C, Mf)) continue;
                const T wc = (C == 2 * c) ? T(1) : T(0.5);
                s = add(s, mul(wr * wc, f[R * Mf + C]));
            }
        }
        d[k] = s;
    }
}

unsigned grid_of(hb_context *ctx, int64_t work)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)ctx->num_sms * 32));
}

}  // namespace

template <typename T> int hb_launch_prolong_add(hb_context *ctx, int64_t Mf, T *y, const T *c)
{
    prolong_add_kernel<T><<<grid_of(ctx, Mf * Mf), 256, 0, ctx->stream>>>(Mf, Mf / 2 + 1, y, c);
    return hb_check_launch(ctx, "prolong_add_kernel");
}
template int hb_launch_prolong_add<double>(hb_context *, int64_t, double *, const double *);
template int hb_launch_prolong_add<float>(hb_context *, int64_t, float *, const float *);

template <typename T> int hb_launch_restrict_pt(hb_context *ctx, int64_t Mf, T *d, const T *f)
{
    const int64_t Mc = Mf / 2 + 1;
    restrict_kernel<T><<<grid_of(ctx, Mc * Mc), 256, 0, ctx->stream>>>(Mf, Mc, d, f);
    return hb_check_launch(ctx, "restrict_kernel");
}
template int hb_launch_restrict_pt<double>(hb_context *, int64_t, double *, const double *);
template int hb_launch_restrict_pt<float>(hb_context *, int64_t, float *, const float *);
