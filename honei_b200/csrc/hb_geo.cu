// hb_geo.cu -- matrix-free geometric transfers of (2^k + 1)^2 grids:
// Prolongation<Tag, methods::NONE> (honei/math/prolongation.hh:42-139) and
// Restriction<Tag, methods::NONE> (honei/math/restriction.hh:41-170), each followed by
// ApplyDirichletBoundaries (honei/math/apply_dirichlet_boundaries.hh) with the 8-entry mask
// (corners bottom-left, bottom-right, top-right, top-left, then edges bottom, right, top, left;
// 2 = Dirichlet, the nodes are zeroed).
//
// The reference runs sequential loops that accumulate into the output with +=; every fine
// (prolongation) or coarse (restriction) node is written by a fixed sequence of those updates,
// so one thread per output node replays its own sequence:
//   prolongation, fine node (R, C):  both even -> the coarse value; one odd -> 0 + a/2 + b/2 of
//     the two coarse neighbours along the odd direction; both odd -> 0 + lb/4 + rb/4 + lt/4 + rt/4.
//   restriction, coarse node (r, c): the fine value at (2r, 2c), then the contributions of the
//     reference's outer iterations i in increasing order (i in {r, r+1, c, c+1}, 1 <= i <=
//     (side-1)), each in the loop order of its eight inner passes.
// Each += is evaluated in double (the reference's 0.5 / 0.25 literals are double) and stored
// as T, exactly as the reference's DenseVector<T> updates round.  No matrix is read: the
// traffic is the two vectors only.
#include "hb_internal.cuh"

namespace {

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

struct Mask {
    unsigned char m[8];
};

__device__ __forceinline__ bool dirichlet(int64_t r, int64_t c, int64_t M, const Mask &k)
{
    const bool top = r == M - 1, bottom = r == 0, left = c == 0, right = c == M - 1;
    const bool inner_r = r >= 1 && r <= M - 2, inner_c = c >= 1 && c <= M - 2;
    return (bottom && left && k.m[0]) || (bottom && right && k.m[1]) || (top && right && k.m[2]) ||
           (top && left && k.m[3]) || (bottom && inner_c && k.m[4]) || (right && inner_r && k.m[5]) ||
           (top && inner_c && k.m[6]) || (left && inner_r && k.m[7]);
}

// v += w * f, in double, stored as T
template <typename T> __device__ __forceinline__ T acc(T v, double w, T f)
{
    return (T)dadd((double)v, dmul((double)f, w));
}

template <typename T>
__global__ void prolongate_kernel(int64_t Mf, int64_t Mc, T *__restrict__ fine, const T *__restrict__ coarse, Mask mask)
{
    const int64_t nf = Mf * Mf;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nf; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t R = k / Mf, C = k - R * Mf;
        T v;
        if (dirichlet(R, C, Mf, mask)) {
            v = T(0);
        } else if (!(R & 1) && !(C & 1)) {
            v = coarse[(R / 2) * Mc + C / 2];
        } else if (!(R & 1)) {
            // row even, column odd: coarse (R/2, (C-1)/2) and (R/2, (C+1)/2)
            v = acc(T(0), 0.5, coarse[(R / 2) * Mc + (C - 1) / 2]);
            v = acc(v, 0.5, coarse[(R / 2) * Mc + (C + 1) / 2]);
        } else if (!(C & 1)) {
            // row odd, column even: the coarse nodes below and above
            v = acc(T(0), 0.5, coarse[((R - 1) / 2) * Mc + C / 2]);
            v = acc(v, 0.5, coarse[((R + 1) / 2) * Mc + C / 2]);
        } else {
            const int64_t rb = (R - 1) / 2, rt = (R + 1) / 2, cl = (C - 1) / 2, cr = (C + 1) / 2;
            v = acc(T(0), 0.25, coarse[rb * Mc + cl]);
            v = acc(v, 0.25, coarse[rb * Mc + cr]);
            v = acc(v, 0.25, coarse[rt * Mc + cl]);
            v = acc(v, 0.25, coarse[rt * Mc + cr]);
        }
        fine[k] = v;
    }
}

template <typename T>
__global__ void restrict_kernel(int64_t Mf, int64_t Mc, T *__restrict__ coarse, const T *__restrict__ fine, Mask mask)
{
    const int64_t nc = Mc * Mc, nxc = Mc - 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nc; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = k / Mc, c = k - r * Mc;
        if (dirichlet(r, c, Mc, mask)) {
            coarse[k] = T(0);
            continue;
        }
        auto F = [&](int64_t R, int64_t C) { return fine[R * Mf + C]; };
        T v = F(2 * r, 2 * c);
        // outer iterations touching (r, c), ascending and distinct
        int64_t cand[4] = {r, r + 1, c, c + 1};
        for (int a = 1; a < 4; ++a)
            for (int b = a; b > 0 && cand[b - 1] > cand[b]; --b) {
                const int64_t t = cand[b]; cand[b] = cand[b - 1]; cand[b - 1] = t;
            }
        for (int q = 0; q < 4; ++q) {
            const int64_t i = cand[q];
            if (i < 1 || i > nxc || (q > 0 && cand[q - 1] == i)) continue;
            if (r == i) v = acc(v, 0.5, F(2 * r - 1, 2 * c));
            if (r == i - 1) v = acc(v, 0.5, F(2 * r + 1, 2 * c));
            if (c == i - 1) v = acc(v, 0.5, F(2 * r, 2 * c + 1));
            if (c == i) v = acc(v, 0.5, F(2 * r, 2 * c - 1));
            if (r == i - 1 && c < nxc) v = acc(v, 0.25, F(2 * r + 1, 2 * c + 1));
            if (r == i - 1 && c >= 1) v = acc(v, 0.25, F(2 * r + 1, 2 * c - 1));
            if (r == i && c < nxc) v = acc(v, 0.25, F(2 * r - 1, 2 * c + 1));
            if (r == i && c >= 1) v = acc(v, 0.25, F(2 * r - 1, 2 * c - 1));
        }
        coarse[k] = v;
    }
}

// fine side Mf (odd) from n_fine; coarse side (Mf - 1) / 2 + 1
int sides(int64_t n_fine, int64_t *Mf, int64_t *Mc)
{
    if (n_fine < 1) return HB_ERR_INVALID;
    int64_t m = (int64_t)sqrt((double)n_fine);
    while (m * m > n_fine) --m;
    while ((m + 1) * (m + 1) <= n_fine) ++m;
    if (m * m != n_fine || !(m & 1)) return HB_ERR_UNSUPPORTED;
    *Mf = m;
    *Mc = (m - 1) / 2 + 1;
    return HB_OK;
}

template <typename T>
int transfer(hb_context *ctx, int64_t n_fine, T *out, const T *in, const uint64_t *mask, bool prolongate)
{
    if (!ctx || !out || !in || !mask) return HB_ERR_INVALID;
    int64_t Mf, Mc;
    int st = sides(n_fine, &Mf, &Mc);
    if (st) return st;
    Mask m;
    for (int i = 0; i < 8; ++i) m.m[i] = mask[i] == 2;
    const int64_t work = prolongate ? Mf * Mf : Mc * Mc;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)ctx->num_sms * 32));
    if (prolongate) prolongate_kernel<T><<<blocks, 256, 0, ctx->stream>>>(Mf, Mc, out, in, m);
    else restrict_kernel<T><<<blocks, 256, 0, ctx->stream>>>(Mf, Mc, out, in, m);
    return hb_check_launch(ctx, prolongate ? "prolongate_kernel" : "restrict_kernel");
}

}  // namespace

extern "C" {

int hb_prolongate_f64(hb_context *ctx, int64_t n_fine, double *fine, const double *coarse, const uint64_t *mask)
{
    HB_RANGE("hb_prolongate_f64");
    return transfer<double>(ctx, n_fine, fine, coarse, mask, true);
}

int hb_prolongate_f32(hb_context *ctx, int64_t n_fine, float *fine, const float *coarse, const uint64_t *mask)
{
    HB_RANGE("hb_prolongate_f32");
    return transfer<float>(ctx, n_fine, fine, coarse, mask, true);
}

int hb_restrict_f64(hb_context *ctx, int64_t n_fine, double *coarse, const double *fine, const uint64_t *mask)
{
    HB_RANGE("hb_restrict_f64");
    return transfer<double>(ctx, n_fine, coarse, fine, mask, false);
}

int hb_restrict_f32(hb_context *ctx, int64_t n_fine, float *coarse, const float *fine, const uint64_t *mask)
{
    HB_RANGE("hb_restrict_f32");
    return transfer<float>(ctx, n_fine, coarse, fine, mask, false);
}

}  // extern "C"
