// hb_order.cu -- locality order of a device ELL matrix and the product through a reordered copy.
//
// A matrix whose rows and columns were numbered at random (the permuted Q1 workload) makes
// every x gather of the product a separate 32-byte sector from L2: 37.7 M of them per product
// at 2049^2, where the natural numbering needs about a third of a sector per entry.  The fix
// does not change a single rounding: the rows are stored in a Cuthill-McKee breadth-first
// order of the matrix graph (row -> its columns), each row keeping its slots in their order,
// and the product writes row order[k]'s sum to y[order[k]].  With the columns renumbered as
// well (B = P A P^T) the gathers become local; x then goes through the same permutation first
// (xw[k] = x[order[k]]).  Either way each y entry is the same sum of the same products in the
// same order as the product on A, so y is bit-identical to Product<tags::CPU>
// (honei/la/product.hh:148-204).
#include "hb_spmv_core.cuh"

#include <algorithm>

namespace {

constexpr int ORD_THREADS = 1024;
constexpr int ORD_ITEMS = 16;                                  // (row, slot) items per thread and tile
constexpr int64_t ORD_TILE = (int64_t)ORD_THREADS * ORD_ITEMS;
constexpr unsigned long long ORD_NONE = ~0ull;
constexpr int ROWS_THREADS = 256;

// Exclusive scan of one value per thread over the block, in thread order; *total = the sum.
// smem: 33 entries.  Every thread of the block must call it.
__device__ int64_t block_exclusive_scan(int64_t v, int64_t *smem, int64_t *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int64_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    __syncthreads();
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int64_t w = lane < nw ? smem[lane] : 0;
        int64_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < nw) smem[lane] = wi - w;
        if (lane == 31) smem[32] = wi;
    }
    __syncthreads();
    const int64_t excl = smem[warp] + inc - v;
    *total = smem[32];
    return excl;
}

// Cuthill-McKee order in one block (the levels depend on each other; one block keeps every
// level's hand-over inside __syncthreads).  Start: the row with the fewest off-diagonal
// entries among rows that have one, lowest index on ties.  Level l + 1 = the rows first
// reached from level l, ordered by the position of the first row of level l that reaches
// them and, within that row, by slot -- the sequential breadth-first order, obtained in
// parallel: every (row, slot) item of the level claims its column with atomicMin on its item
// index, and the winning items are compacted in item order.  Rows the search never reaches
// follow in ascending order.  info: levels, rows reached, start row.
__global__ void __launch_bounds__(ORD_THREADS)
cm_order_kernel(int64_t n, int64_t ld, int K, const int32_t *__restrict__ Aj, int32_t *__restrict__ order,
                int32_t *__restrict__ pos, unsigned long long *__restrict__ key, int64_t *__restrict__ info)
{
    __shared__ int64_t s_scan[33];
    __shared__ unsigned long long s_best;
    const int tid = threadIdx.x;
    for (int64_t r = tid; r < n; r += blockDim.x) {
        pos[r] = -1;
        key[r] = ORD_NONE;
    }
    if (tid == 0) s_best = ORD_NONE;
    __syncthreads();
    unsigned long long best = ORD_NONE;
    for (int64_t r = tid; r < n; r += blockDim.x) {
        unsigned long long deg = 0;
        for (int k = 0; k < K; ++k) {
            const int32_t c = Aj[(int64_t)k * ld + r];
            if (c >= 0 && c != r) ++deg;
        }
        if (deg) best = min(best, (deg << 32) | (unsigned long long)r);
    }
    atomicMin(&s_best, best);
    __syncthreads();
    int64_t s = 0, e = 0, levels = 0;
    const unsigned long long start = s_best;
    if (start != ORD_NONE) {
        const int32_t r0 = (int32_t)(start & 0xffffffffull);
        if (tid == 0) { order[0] = r0; pos[r0] = 0; }
        e = 1;
    }
    __syncthreads();
    while (e > s) {
        const int64_t items = (e - s) * K;
        for (int64_t i = tid; i < items; i += blockDim.x) {
            const int64_t k = i / K;
            const int slot = (int)(i - k * K);
            const int32_t v = order[s + k];
            const int32_t c = Aj[(int64_t)slot * ld + v];
            if (c >= 0 && c != v && pos[c] < 0) atomicMin(&key[c], (unsigned long long)i);
        }
        __syncthreads();
        int64_t placed = e;
        for (int64_t t0 = 0; t0 < items; t0 += ORD_TILE) {
            int32_t cs[ORD_ITEMS];
            int cnt = 0;
#pragma unroll
            for (int j = 0; j < ORD_ITEMS; ++j) {
                const int64_t i = t0 + (int64_t)tid * ORD_ITEMS + j;
                cs[j] = -1;
                if (i < items) {
                    const int64_t k = i / K;
                    const int slot = (int)(i - k * K);
                    const int32_t v = order[s + k];
                    const int32_t c = Aj[(int64_t)slot * ld + v];
                    if (c >= 0 && c != v && pos[c] < 0 && __ldcg(key + c) == (unsigned long long)i) {
                        cs[j] = c;
                        ++cnt;
                    }
                }
            }
            int64_t total;
            int64_t at = placed + block_exclusive_scan(cnt, s_scan, &total);
#pragma unroll
            for (int j = 0; j < ORD_ITEMS; ++j) {
                if (cs[j] >= 0) {
                    order[at] = cs[j];
                    pos[cs[j]] = (int32_t)at;
                    ++at;
                }
            }
            placed += total;
            __syncthreads();
        }
        s = e;
        e = placed;
        ++levels;
    }
    const int64_t reached = e;
    int64_t placed = e;
    for (int64_t t0 = 0; t0 < n; t0 += ORD_TILE) {
        int cnt = 0;
        for (int j = 0; j < ORD_ITEMS; ++j) {
            const int64_t r = t0 + (int64_t)tid * ORD_ITEMS + j;
            if (r < n && pos[r] < 0) ++cnt;
        }
        int64_t total;
        int64_t at = placed + block_exclusive_scan(cnt, s_scan, &total);
        for (int j = 0; j < ORD_ITEMS; ++j) {
            const int64_t r = t0 + (int64_t)tid * ORD_ITEMS + j;
            if (r < n && pos[r] < 0) {
                order[at] = (int32_t)r;
                pos[r] = (int32_t)at;
                ++at;
            }
        }
        placed += total;
        __syncthreads();
    }
    if (tid == 0) {
        info[0] = levels;
        info[1] = reached;
        info[2] = start == ORD_NONE ? -1 : (int64_t)(start & 0xffffffffull);
    }
}

// The same Cuthill-McKee order on the whole GPU (cooperative launch, every block resident):
// each level's (row, slot) items are split into one contiguous chunk per block; three
// grid-wide exchanges per level separate the claims (atomicMin on the item index, as above),
// the per-block winner counts and the placement, which scans each chunk in item order and
// offsets it by the counts of the chunks before it -- so the order is item for item the one the
// single-block kernel produces.  Unreached rows follow in ascending order (a fourth pass of the
// same kind over the rows).  Every exchange is bounded (CountExchange); on a timeout the blocks
// return and the status word holds HB_DEV_TIMEOUT.
constexpr int ORDG_THREADS = 512;
constexpr int64_t CM_GRID_MIN_ROWS = 4096;     // smaller matrices: the single-block kernel
constexpr int ORDG_ITEMS = 4;
constexpr int64_t ORDG_TILE = (int64_t)ORDG_THREADS * ORDG_ITEMS;

struct OrdGrid {
    int64_t n, ld;
    int K;
    const int32_t *Aj;
    int32_t *order, *pos;
    unsigned long long *key, *best;
    int64_t *cnt, *info;
    hbd::CountExchange X;
};

// winner of item i of the level starting at s: its column c, or -1
__device__ __forceinline__ int32_t ord_item(const OrdGrid &Q, int64_t s, int64_t i, bool need_key)
{
    const int64_t k = i / Q.K;
    const int slot = (int)(i - k * Q.K);
    const int32_t v = __ldcg(Q.order + s + k);
    const int32_t c = __ldg(Q.Aj + (int64_t)slot * Q.ld + v);
    if (c < 0 || c == v || __ldcg(Q.pos + c) >= 0) return -1;
    if (need_key && __ldcg(Q.key + c) != (unsigned long long)i) return -1;
    return c;
}

__global__ void __launch_bounds__(ORDG_THREADS) cm_order_grid_kernel(OrdGrid Q)
{
    __shared__ int64_t s_scan[33];
    __shared__ int64_t s_off[2];
    __shared__ unsigned long long s_best;
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    const unsigned G = gridDim.x;
    const int64_t b = blockIdx.x;
    const int64_t gstride = (int64_t)G * blockDim.x, gtid = b * blockDim.x + tid;
    const int64_t n = Q.n;
    unsigned e = 0;
    for (int64_t r = gtid; r < n; r += gstride) {
        Q.pos[r] = -1;
        Q.key[r] = ORD_NONE;
    }
    if (tid == 0) s_best = ORD_NONE;
    __syncthreads();
    unsigned long long best = ORD_NONE;
    for (int64_t r = gtid; r < n; r += gstride) {
        unsigned long long deg = 0;
        for (int k = 0; k < Q.K; ++k) {
            const int32_t c = __ldg(Q.Aj + (int64_t)k * Q.ld + r);
            if (c >= 0 && c != r) ++deg;
        }
        if (deg) best = min(best, (deg << 32) | (unsigned long long)r);
    }
    atomicMin(&s_best, best);
    __syncthreads();
    if (tid == 0 && s_best != ORD_NONE) atomicMin(Q.best, s_best);
    if (!Q.X.arrive(e++, G, &s_flag)) return;
    const unsigned long long start = __ldcg(Q.best);
    int64_t lo = 0, hi = 0, levels = 0;
    if (start != ORD_NONE) {
        const int32_t r0 = (int32_t)(start & 0xffffffffull);
        if (gtid == 0) { Q.order[0] = r0; Q.pos[r0] = 0; }
        hi = 1;
    }
    if (!Q.X.arrive(e++, G, &s_flag)) return;
    while (hi > lo) {
        const int64_t items = (hi - lo) * Q.K;
        const int64_t cs = (items + G - 1) / G;
        const int64_t i_lo = min(items, b * cs), i_hi = min(items, i_lo + cs);
        // claims
        for (int64_t i = i_lo + tid; i < i_hi; i += blockDim.x) {
            const int32_t c = ord_item(Q, lo, i, false);
            if (c >= 0) atomicMin(Q.key + c, (unsigned long long)i);
        }
        if (!Q.X.arrive(e++, G, &s_flag)) return;
        // winners of this block's chunk
        int64_t mine = 0;
        for (int64_t i = i_lo + tid; i < i_hi; i += blockDim.x) mine += ord_item(Q, lo, i, true) >= 0;
        int64_t total;
        block_exclusive_scan(mine, s_scan, &total);
        if (tid == 0) __stcg(Q.cnt + b, total);
        if (!Q.X.arrive(e++, G, &s_flag)) return;
        // offsets: the winners of the chunks before this one, and the level's total
        if (tid == 0) {
            int64_t before = 0, all = 0;
            for (unsigned q = 0; q < G; ++q) {
                const int64_t c = __ldcg(Q.cnt + q);
                if (q < b) before += c;
                all += c;
            }
            s_off[0] = before;
            s_off[1] = all;
        }
        __syncthreads();
        int64_t at0 = hi + s_off[0];
        const int64_t all = s_off[1];
        for (int64_t t0 = i_lo; t0 < i_hi; t0 += ORDG_TILE) {
            int32_t cs_[ORDG_ITEMS];
            int cnt = 0;
#pragma unroll
            for (int j = 0; j < ORDG_ITEMS; ++j) {
                const int64_t i = t0 + (int64_t)tid * ORDG_ITEMS + j;
                cs_[j] = i < i_hi ? ord_item(Q, lo, i, true) : -1;
                cnt += cs_[j] >= 0;
            }
            int64_t tile_total;
            int64_t at = at0 + block_exclusive_scan(cnt, s_scan, &tile_total);
#pragma unroll
            for (int j = 0; j < ORDG_ITEMS; ++j) {
                if (cs_[j] >= 0) {
                    Q.order[at] = cs_[j];
                    Q.pos[cs_[j]] = (int32_t)at;
                    ++at;
                }
            }
            at0 += tile_total;
            __syncthreads();
        }
        if (!Q.X.arrive(e++, G, &s_flag)) return;
        lo = hi;
        hi += all;
        ++levels;
    }
    // rows never reached, ascending: one contiguous chunk of rows per block
    const int64_t reached = hi;
    const int64_t rs = (n + G - 1) / G;
    const int64_t r_lo = min(n, b * rs), r_hi = min(n, r_lo + rs);
    int64_t mine = 0;
    for (int64_t r = r_lo + tid; r < r_hi; r += blockDim.x) mine += __ldcg(Q.pos + r) < 0;
    int64_t total;
    block_exclusive_scan(mine, s_scan, &total);
    if (tid == 0) __stcg(Q.cnt + b, total);
    if (!Q.X.arrive(e++, G, &s_flag)) return;
    if (tid == 0) {
        int64_t before = 0;
        for (unsigned q = 0; q < b; ++q) before += __ldcg(Q.cnt + q);
        s_off[0] = before;
    }
    __syncthreads();
    int64_t at0 = reached + s_off[0];
    for (int64_t t0 = r_lo; t0 < r_hi; t0 += ORDG_TILE) {
        int cnt = 0;
        bool un[ORDG_ITEMS];
#pragma unroll
        for (int j = 0; j < ORDG_ITEMS; ++j) {
            const int64_t r = t0 + (int64_t)tid * ORDG_ITEMS + j;
            un[j] = r < r_hi && __ldcg(Q.pos + r) < 0;
            cnt += un[j];
        }
        int64_t tile_total;
        int64_t at = at0 + block_exclusive_scan(cnt, s_scan, &tile_total);
        __syncthreads();   // every thread read pos for its rows before any placement below
#pragma unroll
        for (int j = 0; j < ORDG_ITEMS; ++j) {
            if (un[j]) {
                const int64_t r = t0 + (int64_t)tid * ORDG_ITEMS + j;
                Q.order[at] = (int32_t)r;
                Q.pos[r] = (int32_t)at;
                ++at;
            }
        }
        at0 += tile_total;
        __syncthreads();
    }
    if (gtid == 0) {
        Q.info[0] = levels;
        Q.info[1] = reached;
        Q.info[2] = start == ORD_NONE ? -1 : (int64_t)(start & 0xffffffffull);
    }
}

// max |pos(c) - pos(r)| over the stored entries (identity numbering when pos is null).
__global__ void ell_bandwidth_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj,
                                     const int32_t *__restrict__ pos, unsigned long long *out)
{
    unsigned long long m = 0;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (int64_t)K * ld;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx / ld, r = idx - k * ld;
        if (r >= rows) continue;
        const int32_t c = Aj[idx];
        if (c < 0) continue;
        const int64_t a = pos ? pos[r] : r, b = pos ? pos[c] : c;
        const unsigned long long d = (unsigned long long)(a > b ? a - b : b - a);
        m = d > m ? d : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_down_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// B row kk = A row order[kk] with its columns renumbered through pos and its valid slots sorted
// by the new column (one thread per row; import-time work).  ranks[kk] packs, 4 bits per
// physical slot k, the rank of that slot in A's row (its place in the reference's summation
// order); padding slots (Aj = -1) follow the valid ones.
template <typename T, int KMAX>
__global__ void ell_permute_sorted_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj,
                                          const T *__restrict__ Ax, const int32_t *__restrict__ order,
                                          const int32_t *__restrict__ pos, int32_t *__restrict__ Bj,
                                          T *__restrict__ Bx, unsigned long long *__restrict__ ranks)
{
    for (int64_t kk = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; kk < ld; kk += (int64_t)gridDim.x * blockDim.x) {
        int32_t c[KMAX];
        T a[KMAX];
        int rk[KMAX];
        int n = 0;
        if (kk < rows) {
            const int64_t r = order[kk];
            for (int k = 0; k < K; ++k) {
                const int32_t j = Aj[(int64_t)k * ld + r];
                if (j < 0) continue;
                // insertion by new column; equal columns keep their original order
                const int32_t cj = pos[j];
                const T aj = Ax[(int64_t)k * ld + r];
                int at = n;
                while (at > 0 && c[at - 1] > cj) {
                    c[at] = c[at - 1];
                    a[at] = a[at - 1];
                    rk[at] = rk[at - 1];
                    --at;
                }
                c[at] = cj;
                a[at] = aj;
                rk[at] = n;
                ++n;
            }
        }
        unsigned long long packed = 0;
        for (int k = 0; k < K; ++k) {
            const bool v = k < n;
            Bj[(int64_t)k * ld + kk] = v ? c[k] : -1;
            Bx[(int64_t)k * ld + kk] = v ? a[k] : T(0);
            packed |= (unsigned long long)(v ? rk[k] : 15) << (4 * k);
        }
        if (kk < rows) ranks[kk] = packed;
    }
}

// B row kk = A row order[kk], slots unchanged; columns renumbered through pos when given.
template <typename T>
__global__ void ell_permute_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj,
                                   const T *__restrict__ Ax, const int32_t *__restrict__ order,
                                   const int32_t *__restrict__ pos, int32_t *__restrict__ Bj, T *__restrict__ Bx)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (int64_t)K * ld;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx / ld, kk = idx - k * ld;
        int32_t c = -1;
        T a = T(0);
        if (kk < rows) {
            const int64_t src = k * ld + order[kk];
            c = Aj[src];
            a = Ax[src];
            if (pos && c >= 0) c = pos[c];
        }
        Bj[idx] = c;
        Bx[idx] = a;
    }
}

// y[order[r]] = sum over B's row r (the rows4 loop of the plain product; x gathered with B's
// column indices).
template <typename T, int KT>
__global__ void __launch_bounds__(ROWS_THREADS)
ell_spmv_rows_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj, const T *__restrict__ Ax,
                     const T *__restrict__ x, const int32_t *__restrict__ order, T *__restrict__ y)
{
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r0 = g * 4;
    if (r0 >= rows) return;
    T sum[4];
    hbd::ell_rows4<T, KT>(Aj, Ax, ld, K, r0, [&](int32_t j) { return __ldg(x + j); }, sum);
    if (r0 + 3 < rows) {
        const int4 o = __ldg(reinterpret_cast<const int4 *>(order + r0));
        y[o.x] = sum[0];
        y[o.y] = sum[1];
        y[o.z] = sum[2];
        y[o.w] = sum[3];
    } else {
        for (int i = 0; i < 4 && r0 + i < rows; ++i) y[order[r0 + i]] = sum[i];
    }
}

// The product through a sorted, ranked copy (ell_permute_sorted_kernel): one row per thread,
// the products of its slots (physical order, so a warp's gathers for one slot are neighbours)
// parked in shared memory at their ranks, then summed in rank order -- the order the
// reference sums the row in.  y[order[r]] = the sum.
constexpr int RANKED_THREADS = 256;
template <typename T, int KT>
__global__ void __launch_bounds__(RANKED_THREADS)
ell_spmv_ranked_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Aj, const T *__restrict__ Ax,
                       const unsigned long long *__restrict__ ranks, const T *__restrict__ x,
                       const int32_t *__restrict__ order, T *__restrict__ y)
{
    constexpr int KS = KT > 0 ? KT : 16;
    __shared__ T park[KS * RANKED_THREADS];
    const int K_ = KT > 0 ? KT : K;
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const unsigned long long rk = __ldg(ranks + r);
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < KS; ++k) {
        if (k >= K_) break;
        const int32_t j = __ldcs(Aj + (int64_t)k * ld + r);
        const T a = __ldcs(Ax + (int64_t)k * ld + r);
        if (j >= 0) {
            const int at = (int)((rk >> (4 * k)) & 15ull);
            park[at * RANKED_THREADS + threadIdx.x] = hbd::mul(a, __ldg(x + j));
            ++cnt;
        }
    }
    T sum = T(0);
    for (int k = 0; k < cnt; ++k) sum = hbd::add(sum, park[k * RANKED_THREADS + threadIdx.x]);
    y[__ldg(order + r)] = sum;
}

// xw[k] = x[order[k]]
template <typename T>
__global__ void gather_kernel(int64_t n, const int32_t *__restrict__ order, const T *__restrict__ x, T *__restrict__ xw)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        xw[k] = __ldg(x + __ldg(order + k));
}

// The packed form of a renumbered copy (hb_ell_permute with pos: rows in the locality order,
// columns renumbered, each row's slots in their own order): slot k of row r keeps its column as
// the 16-bit offset c - r (PACK_NONE for padding).  Bandwidths within +-32767 only.
constexpr int16_t PACK_NONE = INT16_MIN;
constexpr int PACKED_THREADS = 256;

__global__ void ell_pack_kernel(int64_t rows, int64_t ld, int K, const int32_t *__restrict__ Bj,
                                int16_t *__restrict__ Bd, unsigned long long *__restrict__ overflow)
{
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (int64_t)K * ld;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx / ld, r = idx - k * ld;
        int16_t d = PACK_NONE;
        if (r < rows) {
            const int32_t c = Bj[idx];
            if (c >= 0) {
                const int64_t off = (int64_t)c - r;
                if (off < -32767 || off > 32767) atomicAdd(overflow, 1ull);
                else d = (int16_t)off;
            }
        }
        Bd[idx] = d;
    }
}

// y[order[r]] = B's row r from the packed form, summed in slot order (the reference's order: the
// copy keeps each row's slots as they were): one row per thread, every streaming load of the
// row (offsets, values, order) issued before every gather of x, 8 blocks of 256 per SM (32
// registers).
template <typename T, int KT>
__global__ void __launch_bounds__(PACKED_THREADS, 8)
ell_spmv_packed_kernel(int64_t rows, int64_t ld, int K, const int16_t *__restrict__ Bd, const T *__restrict__ Ax,
                       const T *__restrict__ x, const int32_t *__restrict__ order, T *__restrict__ y)
{
    constexpr int KS = KT > 0 ? KT : 9;
    const int K_ = KT > 0 ? KT : K;
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    int32_t c[KS];
    T a[KS];
#pragma unroll
    for (int k = 0; k < KS; ++k) {
        c[k] = -1;
        a[k] = T(0);
        if (k < K_) {
            const int16_t d = __ldcs(Bd + (int64_t)k * ld + r);
            if (d != PACK_NONE) c[k] = (int32_t)(r + d);
            a[k] = __ldcs(Ax + (int64_t)k * ld + r);
        }
    }
    const int32_t o = __ldg(order + r);
    T v[KS];
#pragma unroll
    for (int k = 0; k < KS; ++k) v[k] = c[k] >= 0 ? __ldg(x + c[k]) : T(0);
    T sum = T(0);
#pragma unroll
    for (int k = 0; k < KS; ++k)
        if (c[k] >= 0) sum = hbd::add(sum, hbd::mul(a[k], v[k]));
    y[o] = sum;
}

template <typename T>
int spmv_packed_impl(hb_context *ctx, const hb_ell *B, int dtype, const int16_t *Bd, const int32_t *order,
                     const T *x, T *y)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = hb_check_ell(B, dtype);
    if (st) return st;
    if (B->K > 9) return HB_ERR_UNSUPPORTED;
    if (B->rows == 0) return HB_OK;
    if (!Bd || !order || !x || !y) return HB_ERR_INVALID;
    const unsigned blocks = (unsigned)((B->rows + PACKED_THREADS - 1) / PACKED_THREADS);
    const T *Bx = (const T *)B->Ax;
    if (B->K == 9)
        ell_spmv_packed_kernel<T, 9><<<blocks, PACKED_THREADS, 0, ctx->stream>>>(B->rows, B->ld, 9, Bd, Bx, x, order, y);
    else
        ell_spmv_packed_kernel<T, 0><<<blocks, PACKED_THREADS, 0, ctx->stream>>>(B->rows, B->ld, (int)B->K, Bd, Bx, x,
                                                                                 order, y);
    return hb_check_launch(ctx, "ell_spmv_packed_kernel");
}

template <typename T>
int spmv_rows_impl(hb_context *ctx, const hb_ell *B, int dtype, const int32_t *order, const T *x, T *y)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = hb_check_ell(B, dtype);
    if (st) return st;
    if (B->rows == 0) return HB_OK;
    if (!order || !x || !y || ((uintptr_t)order % 16)) return HB_ERR_INVALID;
    const int64_t groups = (B->rows + 3) / 4;
    const unsigned blocks = (unsigned)((groups + ROWS_THREADS - 1) / ROWS_THREADS);
    const T *Bx = (const T *)B->Ax;
    if (B->K == 9)
        ell_spmv_rows_kernel<T, 9><<<blocks, ROWS_THREADS, 0, ctx->stream>>>(B->rows, B->ld, 9, B->Aj, Bx, x, order, y);
    else if (B->K == 4)
        ell_spmv_rows_kernel<T, 4><<<blocks, ROWS_THREADS, 0, ctx->stream>>>(B->rows, B->ld, 4, B->Aj, Bx, x, order, y);
    else
        ell_spmv_rows_kernel<T, 0><<<blocks, ROWS_THREADS, 0, ctx->stream>>>(B->rows, B->ld, (int)B->K, B->Aj, Bx, x,
                                                                             order, y);
    return hb_check_launch(ctx, "ell_spmv_rows_kernel");
}

template <typename T>
int spmv_ranked_impl(hb_context *ctx, const hb_ell *B, int dtype, const int32_t *order,
                     const unsigned long long *ranks, const T *x, T *y)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = hb_check_ell(B, dtype);
    if (st) return st;
    if (B->K > 16) return HB_ERR_UNSUPPORTED;
    if (B->rows == 0) return HB_OK;
    if (!order || !ranks || !x || !y) return HB_ERR_INVALID;
    const unsigned blocks = (unsigned)((B->rows + RANKED_THREADS - 1) / RANKED_THREADS);
    const T *Bx = (const T *)B->Ax;
    if (B->K == 9)
        ell_spmv_ranked_kernel<T, 9><<<blocks, RANKED_THREADS, 0, ctx->stream>>>(B->rows, B->ld, 9, B->Aj, Bx, ranks, x,
                                                                                 order, y);
    else
        ell_spmv_ranked_kernel<T, 0><<<blocks, RANKED_THREADS, 0, ctx->stream>>>(B->rows, B->ld, (int)B->K, B->Aj, Bx,
                                                                                 ranks, x, order, y);
    return hb_check_launch(ctx, "ell_spmv_ranked_kernel");
}

template <typename T>
int gather_impl(hb_context *ctx, int64_t n, const int32_t *order, const T *x, T *xw)
{
    if (!ctx || n < 0) return HB_ERR_INVALID;
    if (n == 0) return HB_OK;
    if (!order || !x || !xw) return HB_ERR_INVALID;
    const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 16);
    gather_kernel<T><<<blocks, 256, 0, ctx->stream>>>(n, order, x, xw);
    return hb_check_launch(ctx, "gather_kernel");
}

}  // namespace

extern "C" {

int hb_ell_cm_order(hb_context *ctx, const hb_ell *A, int32_t *order, int32_t *pos, int64_t *info)
{
    HB_RANGE("hb_ell_cm_order");
    if (!ctx || !A || !order) return HB_ERR_INVALID;
    if (!A->Aj || A->rows < 0 || A->K < 1 || A->ld < A->rows) return HB_ERR_INVALID;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    if (A->rows > INT32_MAX) return HB_ERR_UNSUPPORTED;
    const int64_t n = A->rows;
    if (n == 0) {
        if (info) info[0] = info[1] = 0, info[2] = -1;
        return HB_OK;
    }
    // workspace: key (u64), without a caller array pos (int32), and for the grid form the start
    // candidate (u64) and one count per block (int64)
    const size_t key_bytes = (size_t)n * 8;
    const size_t pos_bytes = pos ? 0 : hb_round_up(n * 4, 256);
    int grid = 0;
    if (n >= CM_GRID_MIN_ROWS) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, cm_order_grid_kernel, ORDG_THREADS, 0) != cudaSuccess)
            cudaGetLastError();
        grid = std::min(std::max(occ, 0), 2) * ctx->num_sms;
    }
    const size_t grid_bytes = grid ? 256 + hb_round_up((int64_t)grid * 8, 256) : 0;
    int st = hb_ensure_work(ctx, key_bytes + pos_bytes + grid_bytes);
    if (st) return st;
    unsigned long long *key = (unsigned long long *)ctx->work;
    int32_t *p = pos ? pos : (int32_t *)((char *)ctx->work + key_bytes);
    int64_t *dinfo = (int64_t *)hb_scalars(ctx);
    unsigned *bar = hb_bar(ctx);
    if (grid) {
        OrdGrid Q;
        Q.n = n;
        Q.ld = A->ld;
        Q.K = (int)A->K;
        Q.Aj = A->Aj;
        Q.order = order;
        Q.pos = p;
        Q.key = key;
        Q.best = (unsigned long long *)((char *)ctx->work + key_bytes + pos_bytes);
        Q.cnt = (int64_t *)((char *)Q.best + 256);
        Q.info = dinfo;
        Q.X.count = bar;
        Q.X.status = (int *)(bar + 2);
        HB_CUDA_TRY(ctx, cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), ctx->stream));
        HB_CUDA_TRY(ctx, cudaMemsetAsync(Q.best, 0xff, sizeof(unsigned long long), ctx->stream));
        void *args[] = {&Q};
        HB_CUDA_TRY(ctx, cudaLaunchCooperativeKernel((const void *)cm_order_grid_kernel, dim3(grid), dim3(ORDG_THREADS),
                                                     args, 0, ctx->stream));
        st = hb_check_launch(ctx, "cm_order_grid_kernel");
    } else {
        cm_order_kernel<<<1, ORD_THREADS, 0, ctx->stream>>>(n, A->ld, (int)A->K, A->Aj, order, p, key, dinfo);
        st = hb_check_launch(ctx, "cm_order_kernel");
    }
    if (st) return st;
    int64_t *h = (int64_t *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, dinfo, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h + 3, bar + 2, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (grid) {
        const int dev_status = *(const int *)(h + 3);
        HB_CUDA_TRY(ctx, cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), ctx->stream));
        if (dev_status == HB_DEV_TIMEOUT) return HB_ERR_TIMEOUT;
    }
    if (info) { info[0] = h[0]; info[1] = h[1]; info[2] = h[2]; }
    return HB_OK;
}

int hb_ell_bandwidth(hb_context *ctx, const hb_ell *A, const int32_t *pos, int64_t *bandwidth)
{
    HB_RANGE("hb_ell_bandwidth");
    if (!ctx || !A || !A->Aj || !bandwidth || A->rows < 0 || A->K < 1 || A->ld < A->rows) return HB_ERR_INVALID;
    unsigned long long *d = (unsigned long long *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(d, 0, sizeof(*d), ctx->stream));
    const int64_t total = A->K * A->ld;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 16));
    ell_bandwidth_kernel<<<blocks, 256, 0, ctx->stream>>>(A->rows, A->ld, (int)A->K, A->Aj, pos, d);
    int st = hb_check_launch(ctx, "ell_bandwidth_kernel");
    if (st) return st;
    unsigned long long *h = (unsigned long long *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, d, sizeof(*h), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *bandwidth = (int64_t)*h;
    return HB_OK;
}

int hb_ell_permute(hb_context *ctx, const hb_ell *A, const int32_t *order, const int32_t *pos, hb_ell *B)
{
    HB_RANGE("hb_ell_permute");
    if (!ctx || !B || !order) return HB_ERR_INVALID;
    int st = hb_check_ell(A, A ? A->dtype : 0);
    if (st) return st;
    if (pos && A->rows != A->cols) return HB_ERR_SIZE;
    if (B->K != A->K || B->ld != A->ld || B->Aj == A->Aj || B->Ax == A->Ax) return HB_ERR_SIZE;
    B->rows = A->rows;
    B->cols = A->cols;
    B->dtype = A->dtype;
    st = hb_check_ell(B, A->dtype);
    if (st) return st;
    const int64_t total = A->K * A->ld;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32));
    if (A->dtype == HB_F64)
        ell_permute_kernel<double><<<blocks, 256, 0, ctx->stream>>>(A->rows, A->ld, (int)A->K, A->Aj,
                                                                    (const double *)A->Ax, order, pos, B->Aj,
                                                                    (double *)B->Ax);
    else
        ell_permute_kernel<float><<<blocks, 256, 0, ctx->stream>>>(A->rows, A->ld, (int)A->K, A->Aj,
                                                                   (const float *)A->Ax, order, pos, B->Aj,
                                                                   (float *)B->Ax);
    return hb_check_launch(ctx, "ell_permute_kernel");
}

int hb_ell_permute_sorted(hb_context *ctx, const hb_ell *A, const int32_t *order, const int32_t *pos, hb_ell *B,
                          uint64_t *ranks)
{
    HB_RANGE("hb_ell_permute_sorted");
    if (!ctx || !B || !order || !pos || !ranks) return HB_ERR_INVALID;
    int st = hb_check_ell(A, A ? A->dtype : 0);
    if (st) return st;
    if (A->rows != A->cols) return HB_ERR_SIZE;
    if (A->K > 16) return HB_ERR_UNSUPPORTED;
    if (B->K != A->K || B->ld != A->ld || B->Aj == A->Aj || B->Ax == A->Ax) return HB_ERR_SIZE;
    B->rows = A->rows;
    B->cols = A->cols;
    B->dtype = A->dtype;
    st = hb_check_ell(B, A->dtype);
    if (st) return st;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((A->ld + 255) / 256, (int64_t)ctx->num_sms * 32));
    unsigned long long *rk = (unsigned long long *)ranks;
    if (A->dtype == HB_F64)
        ell_permute_sorted_kernel<double, 16><<<blocks, 256, 0, ctx->stream>>>(
            A->rows, A->ld, (int)A->K, A->Aj, (const double *)A->Ax, order, pos, B->Aj, (double *)B->Ax, rk);
    else
        ell_permute_sorted_kernel<float, 16><<<blocks, 256, 0, ctx->stream>>>(
            A->rows, A->ld, (int)A->K, A->Aj, (const float *)A->Ax, order, pos, B->Aj, (float *)B->Ax, rk);
    return hb_check_launch(ctx, "ell_permute_sorted_kernel");
}

int hb_spmv_ranked_f64(hb_context *ctx, const hb_ell *B, const int32_t *order, const uint64_t *ranks, const double *x,
                       double *y)
{
    HB_RANGE("hb_spmv_ranked_f64");
    return spmv_ranked_impl<double>(ctx, B, HB_F64, order, (const unsigned long long *)ranks, x, y);
}

int hb_spmv_ranked_f32(hb_context *ctx, const hb_ell *B, const int32_t *order, const uint64_t *ranks, const float *x,
                       float *y)
{
    HB_RANGE("hb_spmv_ranked_f32");
    return spmv_ranked_impl<float>(ctx, B, HB_F32, order, (const unsigned long long *)ranks, x, y);
}

int hb_spmv_rows_f64(hb_context *ctx, const hb_ell *B, const int32_t *order, const double *x, double *y)
{
    HB_RANGE("hb_spmv_rows_f64");
    return spmv_rows_impl<double>(ctx, B, HB_F64, order, x, y);
}

int hb_spmv_rows_f32(hb_context *ctx, const hb_ell *B, const int32_t *order, const float *x, float *y)
{
    HB_RANGE("hb_spmv_rows_f32");
    return spmv_rows_impl<float>(ctx, B, HB_F32, order, x, y);
}

int hb_ell_pack_offsets(hb_context *ctx, const hb_ell *B, int16_t *Bd)
{
    HB_RANGE("hb_ell_pack_offsets");
    if (!ctx || !Bd) return HB_ERR_INVALID;
    int st = hb_check_ell(B, B ? B->dtype : 0);
    if (st) return st;
    if (B->K > 9) return HB_ERR_UNSUPPORTED;
    if (B->rows == 0) return HB_OK;
    unsigned long long *d = (unsigned long long *)hb_scalars(ctx);
    HB_CUDA_TRY(ctx, cudaMemsetAsync(d, 0, sizeof(*d), ctx->stream));
    const int64_t total = B->K * B->ld;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 32));
    ell_pack_kernel<<<blocks, 256, 0, ctx->stream>>>(B->rows, B->ld, (int)B->K, B->Aj, Bd, d);
    st = hb_check_launch(ctx, "ell_pack_kernel");
    if (st) return st;
    unsigned long long *h = (unsigned long long *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, d, sizeof(*h), cudaMemcpyDeviceToHost, ctx->stream));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return *h ? HB_ERR_UNSUPPORTED : HB_OK;
}

int hb_spmv_packed_f64(hb_context *ctx, const hb_ell *B, const int16_t *Bd, const int32_t *order, const double *x,
                       double *y)
{
    HB_RANGE("hb_spmv_packed_f64");
    return spmv_packed_impl<double>(ctx, B, HB_F64, Bd, order, x, y);
}

int hb_spmv_packed_f32(hb_context *ctx, const hb_ell *B, const int16_t *Bd, const int32_t *order, const float *x,
                       float *y)
{
    HB_RANGE("hb_spmv_packed_f32");
    return spmv_packed_impl<float>(ctx, B, HB_F32, Bd, order, x, y);
}

int hb_gather_f64(hb_context *ctx, int64_t n, const int32_t *order, const double *x, double *xw)
{
    HB_RANGE("hb_gather_f64");
    return gather_impl<double>(ctx, n, order, x, xw);
}

int hb_gather_f32(hb_context *ctx, int64_t n, const int32_t *order, const float *x, float *xw)
{
    HB_RANGE("hb_gather_f32");
    return gather_impl<float>(ctx, n, order, x, xw);
}

}  // extern "C"
