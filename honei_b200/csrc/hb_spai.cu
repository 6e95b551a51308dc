// hb_spai.cu -- SPAI2<tags::GPU::CUDA>::value(M, A) (honei/math/spai2.hh:294-298, wrapper
// honei/math/spai2-cuda.cc:180-228): the sparse approximate inverse M of a square matrix A with
// A's sparsity pattern, column by column (Grote and Huckle's least-squares SPAI restricted to
// the pattern of A), with the arithmetic of SPAI2<tags::CPU::SSE> (honei/math/spai2.hh:129-260)
// so that M is bit-identical to it:
//   J  = the rows of A's column idx (ascending), n2 of them;
//   I  = the rows of A's columns J[0], J[1], ... concatenated (each ascending), n1 of them;
//   At(k, j) = A(I[k], J[j]), et(k) = (I[k] == idx);
//   product(i, j) = sum_k At(k, i) At(k, j), pro_v(i) = sum_k At(k, i) et(k), sequential in k;
//   LUDecomposition<tags::CPU::SSE> (honei/math/ludecomposition.hh:254-320): elimination
//   without pivoting, then forward and backward substitution with sequential sums;
//   M(J[i], idx) = res[i].
// The entries of A are what SparseMatrix(const SparseMatrixELL &) takes (honei/la/sparse_matrix.hh:
// 157-185): slots whose value is not 0.  Columns with n2 == 0 or n1 == 0 keep A's values (M
// starts as a copy of A, spai2-cuda.cc:187).
//
// Device plan:
//   1. the column structure of A: per-column counts (atomics), an exclusive scan, a fill by
//      atomics and a per-column insertion sort by row -- CSC rows ascending plus, per entry, its
//      ELL slot (where M's value goes);
//   2. columns of at most 9 entries (every Q1 matrix): one thread per column with the normal
//      equations, the LU and the substitutions in registers (spai2_col_kernel);
//   3. wider columns: one warp per column (grid-stride): J's column lengths are scanned across the warp; At is
//      built 32 rows at a time in shared memory (lane k loads row I[k]'s ELL slots together and
//      places each value by a binary search in J), the n2 (n2 + 1)
//      / 2 distinct product entries (product is symmetric: the two multiplication orders give
//      the same products) and pro_v accumulate across the chunks in k order, one lane per entry;
//      the elimination runs in place on the warp's product (rows in parallel, columns in
//      parallel within a step), the two substitutions in lane 0.
// A row that stores one column twice is outside the supported input (the reference's
// conversion keeps the later slot; here both would enter the column lists).
#include "hb_internal.cuh"

#include <cub/device/device_scan.cuh>

#include <climits>

namespace {

constexpr int SPAI_MAX_WARPS = 8;
constexpr int SPAI_MAX_COLUMN = 256;   // longest column any SPAI kernel here can solve (shared memory)
constexpr int SORT_REG = 16;           // columns up to this length are sorted in registers
constexpr int SLOTS = 9;           // ELL slots of a row whose loads are in flight together (Q1: all)

template <typename T>
__device__ __forceinline__ bool spai_entry(int32_t c, T v, int64_t n)
{
    return c >= 0 && (int64_t)c < n && v != T(0);
}

template <typename T>
__global__ void spai_count_kernel(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t n, int64_t ld,
                                  int64_t K, unsigned long long *__restrict__ cnt)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < K * n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = q / n, r = q - s * n;
        const int32_t c = Aj[s * ld + r];
        if (spai_entry(c, Ax[s * ld + r], n)) atomicAdd(cnt + c, 1ull);
    }
}

template <typename T>
__global__ void spai_fill_kernel(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t n, int64_t ld,
                                 int64_t K, unsigned long long *__restrict__ cursor, int32_t *__restrict__ crow,
                                 int32_t *__restrict__ cslot)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < K * n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = q / n, r = q - s * n;
        const int32_t c = Aj[s * ld + r];
        if (!spai_entry(c, Ax[s * ld + r], n)) continue;
        const unsigned long long p = atomicAdd(cursor + c, 1ull);
        crow[p] = (int32_t)r;
        cslot[p] = (int32_t)s;
    }
}

// Sorts each column's (row, slot) pairs by row and records the longest column.  A column longer
// than SPAI_MAX_COLUMN is left unsorted (the call is refused once the longest length is known), so
// the quadratic insertion sort stays bounded for any input.
__global__ void spai_sort_kernel(int64_t n, const unsigned long long *__restrict__ cp, int32_t *__restrict__ crow,
                                 int32_t *__restrict__ cslot, unsigned *__restrict__ maxlen)
{
    unsigned longest = 0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t lo = (int64_t)cp[c], hi = (int64_t)cp[c + 1];
        const int64_t len = hi - lo;
        longest = max(longest, len > (int64_t)UINT_MAX ? UINT_MAX : (unsigned)len);
        if (len > SPAI_MAX_COLUMN) continue;
        if (len <= SORT_REG) {
            // in registers: one load and one store per entry, an odd-even transposition network
            // (rows within a column are distinct, so any correct sort gives the same order)
            int32_t rr[SORT_REG], ss[SORT_REG];
#pragma unroll
            for (int u = 0; u < SORT_REG; ++u) {
                rr[u] = u < len ? crow[lo + u] : INT_MAX;
                ss[u] = u < len ? cslot[lo + u] : 0;
            }
#pragma unroll
            for (int round = 0; round < SORT_REG; ++round)
#pragma unroll
                for (int u = round & 1; u + 1 < SORT_REG; u += 2)
                    if (rr[u] > rr[u + 1]) {
                        const int32_t tr = rr[u], ts = ss[u];
                        rr[u] = rr[u + 1];
                        ss[u] = ss[u + 1];
                        rr[u + 1] = tr;
                        ss[u + 1] = ts;
                    }
#pragma unroll
            for (int u = 0; u < SORT_REG; ++u)
                if (u < len) {
                    crow[lo + u] = rr[u];
                    cslot[lo + u] = ss[u];
                }
            continue;
        }
        for (int64_t a = lo + 1; a < hi; ++a) {
            const int32_t r = crow[a], s = cslot[a];
            int64_t b = a - 1;
            while (b >= lo && crow[b] > r) {
                crow[b + 1] = crow[b];
                cslot[b + 1] = cslot[b];
                --b;
            }
            crow[b + 1] = r;
            cslot[b + 1] = s;
        }
    }
    for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxlen, longest);
}

// Shared memory of one warp for columns of up to cap entries.
template <typename T> size_t spai_warp_bytes(int cap)
{
    const size_t b = ((size_t)32 * cap + (size_t)cap * cap + cap + 32) * sizeof(T) + (size_t)(3 * cap + 1) * sizeof(int32_t);
    return (b + 15) & ~(size_t)15;
}

template <typename T>
__global__ void __launch_bounds__(SPAI_MAX_WARPS * 32, 4) spai2_kernel(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t ld, int64_t K,
                             int64_t n, const unsigned long long *__restrict__ cp, const int32_t *__restrict__ crow,
                             const int32_t *__restrict__ cslot, T *__restrict__ Mx, int cap, unsigned warp_bytes)
{
    using hbd::add; using hbd::div; using hbd::mul; using hbd::sub;
    extern __shared__ __align__(16) unsigned char spai_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    T *At = (T *)(spai_smem + (size_t)w * warp_bytes);    // [32][cap]: chunk rows of At
    T *prod = At + 32 * cap;                               // [n2][n2]: product, then its L\U
    T *pv = prod + cap * cap;                              // [n2]: pro_v, then the solution
    T *et = pv + cap;                                      // [32]
    int32_t *J = (int32_t *)(et + 32);                     // [n2]
    int32_t *seg = J + cap;                                // [n2 + 1]: start of column J[i]'s rows in I
    int32_t *cstart = seg + cap + 1;                       // [n2]: column J[i]'s first entry (CSC)

    for (int64_t col = (int64_t)blockIdx.x * wpb + w; col < n; col += (int64_t)gridDim.x * wpb) {
        const int64_t c0 = (int64_t)cp[col];
        const int n2 = (int)((int64_t)cp[col + 1] - c0);
        if (n2 == 0) continue;
        // J, the CSC start of each column J[i], and the offsets of their row lists in I (an
        // inclusive warp scan of the column lengths, 32 columns at a time)
        int carry = 0;
        if (lane == 0) seg[0] = 0;
        for (int i0 = 0; i0 < n2; i0 += 32) {
            const int i = i0 + lane;
            int len = 0;
            if (i < n2) {
                const int32_t j = crow[c0 + i];
                const int64_t a = (int64_t)cp[j];
                len = (int)((int64_t)cp[j + 1] - a);
                J[i] = j;
                cstart[i] = (int32_t)a;
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, len, o);
                if (lane >= o) len += t;
            }
            if (i < n2) seg[i + 1] = carry + len;
            carry += __shfl_sync(0xffffffffu, len, 31);
        }
        __syncwarp();
        const int n1 = carry;
        if (n1 == 0) {
            __syncwarp();
            continue;
        }
        for (int q = lane; q < n2 * n2; q += 32) prod[q] = T(0);
        for (int i = lane; i < n2; i += 32) pv[i] = T(0);
        const int npairs = n2 * (n2 + 1) / 2;
        for (int k0 = 0; k0 < n1; k0 += 32) {
            const int kc = min(32, n1 - k0);
            if (lane < kc) {
                const int k = k0 + lane;
                int i = 0;
                while (seg[i + 1] <= k) ++i;
                const int32_t r = crow[(int64_t)cstart[i] + (k - seg[i])];
                T *row = At + lane * cap;
                for (int j = 0; j < n2; ++j) row[j] = T(0);
                // the row's slots, SLOTS at a time with all loads in flight, then placed by a
                // binary search in J (slots in order: a later slot of the same column would win)
                for (int64_t s0 = 0; s0 < K; s0 += SLOTS) {
                    int32_t cc[SLOTS];
                    T vv[SLOTS];
#pragma unroll
                    for (int u = 0; u < SLOTS; ++u) {
                        const bool in = s0 + u < K;
                        cc[u] = in ? Aj[(s0 + u) * ld + r] : -1;
                        vv[u] = in ? Ax[(s0 + u) * ld + r] : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < SLOTS; ++u) {
                        if (!spai_entry(cc[u], vv[u], n)) continue;
                        int lo = 0, hi = n2;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (J[mid] < cc[u]) lo = mid + 1; else hi = mid;
                        }
                        if (lo < n2 && J[lo] == cc[u]) row[lo] = vv[u];
                    }
                }
                et[lane] = (int64_t)r == col ? T(1) : T(0);
            }
            __syncwarp();
            for (int q = lane; q < npairs; q += 32) {
                int i = 0, rem = q;
                while (rem >= n2 - i) { rem -= n2 - i; ++i; }
                const int j = i + rem;
                T acc = prod[i * n2 + j];
                for (int kk = 0; kk < kc; ++kk) acc = add(acc, mul(At[kk * cap + i], At[kk * cap + j]));
                prod[i * n2 + j] = acc;
            }
            for (int i = lane; i < n2; i += 32) {
                T acc = pv[i];
                for (int kk = 0; kk < kc; ++kk) acc = add(acc, mul(At[kk * cap + i], et[kk]));
                pv[i] = acc;
            }
            __syncwarp();
        }
        for (int q = lane; q < n2 * n2; q += 32) {
            const int i = q / n2, j = q - i * n2;
            if (i > j) prod[q] = prod[j * n2 + i];
        }
        __syncwarp();
        // elimination step k: l(j, k) = u(j, k) / u(k, k), stored at (j, k) (u's column k below
        // the diagonal is not read again); u(j, i) -= l(j, k) u(k, i) for i > k
        for (int k = 0; k + 1 < n2; ++k) {
            const T ukk = prod[k * n2 + k];
            for (int j = k + 1 + lane; j < n2; j += 32) prod[j * n2 + k] = div(prod[j * n2 + k], ukk);
            __syncwarp();
            const int m = n2 - k - 1;
            for (int q = lane; q < m * m; q += 32) {
                const int j = k + 1 + q / m, i = k + 1 + q % m;
                prod[j * n2 + i] = sub(prod[j * n2 + i], mul(prod[j * n2 + k], prod[k * n2 + i]));
            }
            __syncwarp();
        }
        if (lane == 0) {
            // forward: x_i = 1 / l(i, i) * (b_i - sum), l(i, i) = 1 and 1 / 1 * v == v
            for (int i = 0; i < n2; ++i) {
                T s = T(0);
                for (int j = 0; j < i; ++j) s = add(s, mul(prod[i * n2 + j], pv[j]));
                pv[i] = sub(pv[i], s);
            }
            // backward: x_i = 1 / u(i, i) * (x_i - sum)
            for (int i = n2 - 1; i >= 0; --i) {
                T s = T(0);
                for (int j = i + 1; j < n2; ++j) s = add(s, mul(prod[i * n2 + j], pv[j]));
                pv[i] = mul(div(T(1), prod[i * n2 + i]), sub(pv[i], s));
            }
        }
        __syncwarp();
        for (int i = lane; i < n2; i += 32) Mx[(int64_t)cslot[c0 + i] * ld + J[i]] = pv[i];
        __syncwarp();
    }
}

// Thread per column for columns of at most N entries (N = 9 covers every Q1 matrix): J, the
// normal-equation sums (their N (N + 1) / 2 distinct entries), the LU and both substitutions in
// registers with compile-time indices.  A column with n2 < N entries is padded: J's padding
// matches no column, so its At entries are 0 and only the leading n2 x n2 block is eliminated
// and substituted (the operations on it, and their order, are the warp kernel's and the
// reference's).  Rows of I are visited in I's order: column J[0]'s rows, then J[1]'s, ...
// Launch bounds: FP64 at 3 blocks per SM (168 registers; the few spills fall in the LU, once per
// column) measured 14.0 ms against 15.2 ms at 2 blocks (223 registers) for Q1 2049^2; FP32 fits 4
// blocks per SM in 128 registers.
template <typename T, int N>
__global__ void __launch_bounds__(128, sizeof(T) == 8 ? 3 : 4) spai2_col_kernel(const int32_t *__restrict__ Aj, const T *__restrict__ Ax,
                                                         int64_t ld, int64_t K, int64_t n,
                                                         const unsigned long long *__restrict__ cp,
                                                         const int32_t *__restrict__ crow,
                                                         const int32_t *__restrict__ cslot, T *__restrict__ Mx)
{
    using hbd::add; using hbd::div; using hbd::mul; using hbd::sub;
    constexpr int NP = N * (N + 1) / 2;
    for (int64_t col = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; col < n; col += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c0 = (int64_t)cp[col];
        const int n2 = (int)((int64_t)cp[col + 1] - c0);
        if (n2 == 0) continue;
        // J in registers; the CSC start and length of each column J[i] in shared memory, so the
        // loop over the rows of I is one loop (not one copy per segment: the loop body stays
        // small in the instruction cache)
        __shared__ int64_t sh_cst[N][128];
        __shared__ int sh_len[N][128];
        const int t = threadIdx.x;
        int32_t J[N];
#pragma unroll
        for (int i = 0; i < N; ++i) J[i] = i < n2 ? crow[c0 + i] : -2;
        int n1 = 0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            int64_t a = 0;
            int l = 0;
            if (i < n2) {
                a = (int64_t)cp[J[i]];
                l = (int)((int64_t)cp[J[i] + 1] - a);
            }
            sh_cst[i][t] = a;
            sh_len[i][t] = l;
            n1 += l;
        }
        if (n1 == 0) continue;    // M keeps A's values
        T acc[NP], pv[N];
#pragma unroll
        for (int q = 0; q < NP; ++q) acc[q] = T(0);
#pragma unroll
        for (int i = 0; i < N; ++i) pv[i] = T(0);
        int seg = 0, q = 0;
        for (int k = 0; k < n1; ++k) {
            while (q == sh_len[seg][t]) { ++seg; q = 0; }
            const int32_t r = crow[sh_cst[seg][t] + q];
            ++q;
            T a[N];
#pragma unroll
            for (int j = 0; j < N; ++j) a[j] = T(0);
            for (int64_t s0 = 0; s0 < K; s0 += SLOTS) {
                int32_t cc[SLOTS];
                T vv[SLOTS];
#pragma unroll
                for (int u = 0; u < SLOTS; ++u) {
                    const bool in = s0 + u < K;
                    cc[u] = in ? Aj[(s0 + u) * ld + r] : -1;
                    vv[u] = in ? Ax[(s0 + u) * ld + r] : T(0);
                }
#pragma unroll
                for (int u = 0; u < SLOTS; ++u) {
                    if (!spai_entry(cc[u], vv[u], n)) continue;
#pragma unroll
                    for (int j = 0; j < N; ++j)
                        if (J[j] == cc[u]) a[j] = vv[u];
                }
            }
            const T e = (int64_t)r == col ? T(1) : T(0);
            int p = 0;
#pragma unroll
            for (int i2 = 0; i2 < N; ++i2)
#pragma unroll
                for (int j2 = i2; j2 < N; ++j2) {
                    acc[p] = add(acc[p], mul(a[i2], a[j2]));
                    ++p;
                }
#pragma unroll
            for (int i2 = 0; i2 < N; ++i2) pv[i2] = add(pv[i2], mul(a[i2], e));
        }
        T u[N][N];
        {
            int p = 0;
#pragma unroll
            for (int i2 = 0; i2 < N; ++i2)
#pragma unroll
                for (int j2 = i2; j2 < N; ++j2) {
                    u[i2][j2] = acc[p];
                    u[j2][i2] = acc[p];
                    ++p;
                }
        }
        // elimination without pivoting on the leading n2 x n2 block; l(j, k) kept at (j, k)
#pragma unroll
        for (int k = 0; k + 1 < N; ++k) {
#pragma unroll
            for (int j = k + 1; j < N; ++j) {
                if (j < n2) {
                    const T l = div(u[j][k], u[k][k]);
                    u[j][k] = l;
#pragma unroll
                    for (int i = k + 1; i < N; ++i)
                        if (i < n2) u[j][i] = sub(u[j][i], mul(l, u[k][i]));
                }
            }
        }
        T x[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            x[i] = T(0);
            if (i < n2) {
                T sum = T(0);
#pragma unroll
                for (int j = 0; j < i; ++j) sum = add(sum, mul(u[i][j], x[j]));
                x[i] = sub(pv[i], sum);
            }
        }
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            if (i < n2) {
                T sum = T(0);
#pragma unroll
                for (int j = i + 1; j < N; ++j)
                    if (j < n2) sum = add(sum, mul(u[i][j], x[j]));
                x[i] = mul(div(T(1), u[i][i]), sub(x[i], sum));
            }
        }
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i < n2) Mx[(int64_t)cslot[c0 + i] * ld + J[i]] = x[i];
    }
}

constexpr int SPAI_COL_N = 9;

unsigned grid_of(hb_context *ctx, int64_t work)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)ctx->num_sms * 16));
}

template <typename T>
int spai2_impl(hb_context *ctx, const hb_ell *A, hb_ell *M, int dtype)
{
    if (!ctx) return HB_ERR_INVALID;
    int st = hb_check_ell(A, dtype);
    if (st) return st;
    st = hb_check_ell(M, dtype);
    if (st) return st;
    if (A->rows != A->cols || M->rows != A->rows || M->cols != A->cols || M->K != A->K || M->ld != A->ld)
        return HB_ERR_INVALID;
    if (M->Ax == A->Ax) return HB_ERR_INVALID;
    const int64_t n = A->rows, K = A->K, ld = A->ld;
    if (n == 0) return HB_OK;
    if (K * n > INT32_MAX) return HB_ERR_UNSUPPORTED;
    cudaStream_t s = ctx->stream;
    // M = A.copy()
    if (M->Aj != A->Aj) HB_CUDA_TRY(ctx, cudaMemcpyAsync(M->Aj, A->Aj, (size_t)K * ld * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(M->Ax, A->Ax, (size_t)K * ld * sizeof(T), cudaMemcpyDeviceToDevice, s));

    // workspace: counts / cursor, column offsets, rows and slots of the column lists, scan scratch
    size_t scan_bytes = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (unsigned long long *)nullptr,
                                      (unsigned long long *)nullptr, (int)(n + 1), s) != cudaSuccess) {
        cudaGetLastError();
        return HB_ERR_CUDA;
    }
    const size_t off_cp = (size_t)(n + 1) * 8, off_rows = off_cp + (size_t)(n + 1) * 8;
    const size_t off_slots = off_rows + (((size_t)K * n * 4 + 15) & ~(size_t)15);
    const size_t off_scan = off_slots + (((size_t)K * n * 4 + 15) & ~(size_t)15);
    st = hb_ensure_work(ctx, off_scan + scan_bytes + 16);
    if (st) return st;
    char *w = (char *)ctx->work;
    auto *cnt = (unsigned long long *)w;
    auto *cp = (unsigned long long *)(w + off_cp);
    auto *crow = (int32_t *)(w + off_rows);
    auto *cslot = (int32_t *)(w + off_slots);
    unsigned *maxlen = (unsigned *)hb_scalars(ctx) + 96;

    HB_CUDA_TRY(ctx, cudaMemsetAsync(cnt, 0, (size_t)(n + 1) * 8, s));
    HB_CUDA_TRY(ctx, cudaMemsetAsync(maxlen, 0, sizeof(unsigned), s));
    spai_count_kernel<T><<<grid_of(ctx, K * n), 256, 0, s>>>(A->Aj, (const T *)A->Ax, n, ld, K, cnt);
    if ((st = hb_check_launch(ctx, "spai_count_kernel"))) return st;
    size_t sb = scan_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(w + off_scan, sb, cnt, cp, (int)(n + 1), s);
    if (e != cudaSuccess) { hb_note_error(ctx, e, "DeviceScan::ExclusiveSum"); return HB_ERR_CUDA; }
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, cp, (size_t)(n + 1) * 8, cudaMemcpyDeviceToDevice, s));
    spai_fill_kernel<T><<<grid_of(ctx, K * n), 256, 0, s>>>(A->Aj, (const T *)A->Ax, n, ld, K, cnt, crow, cslot);
    if ((st = hb_check_launch(ctx, "spai_fill_kernel"))) return st;
    spai_sort_kernel<<<grid_of(ctx, n), 256, 0, s>>>(n, cp, crow, cslot, maxlen);
    if ((st = hb_check_launch(ctx, "spai_sort_kernel"))) return st;
    unsigned *h = (unsigned *)ctx->pinned;
    HB_CUDA_TRY(ctx, cudaMemcpyAsync(h, maxlen, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    HB_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    if (*h > (unsigned)SPAI_MAX_COLUMN) return HB_ERR_UNSUPPORTED;    // column lists left unsorted
    const int cap = (int)*h;
    if (cap == 0) return HB_OK;

    if (cap <= SPAI_COL_N) {
        int occ = 0;
        HB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, spai2_col_kernel<T, SPAI_COL_N>, 128, 0));
        const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->num_sms * std::max(occ, 1), (n + 127) / 128));
        spai2_col_kernel<T, SPAI_COL_N><<<(unsigned)blocks, 128, 0, s>>>(A->Aj, (const T *)A->Ax, ld, K, n, cp, crow,
                                                                        cslot, (T *)M->Ax);
        return hb_check_launch(ctx, "spai2_col_kernel");
    }
    int dev = 0, optin = 0;
    HB_CUDA_TRY(ctx, cudaGetDevice(&dev));
    HB_CUDA_TRY(ctx, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    HB_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, spai2_kernel<T>));
    const size_t avail = (size_t)optin - fa.sharedSizeBytes;
    const size_t wb = spai_warp_bytes<T>(cap);
    const int wpb = (int)std::min<size_t>(SPAI_MAX_WARPS, avail / wb);
    if (wpb < 1) return HB_ERR_UNSUPPORTED;    // one column's least-squares system does not fit
    // the attribute is process-wide: always the largest value, so that concurrent calls with
    // other sizes never lower it under each other's launches
    HB_CUDA_TRY(ctx, cudaFuncSetAttribute(spai2_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)avail));
    int occ = 0;
    HB_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, spai2_kernel<T>, 32 * wpb, wb * wpb));
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->num_sms * std::max(occ, 1), (n + wpb - 1) / wpb));
    spai2_kernel<T><<<(unsigned)blocks, 32 * wpb, wb * wpb, s>>>(A->Aj, (const T *)A->Ax, ld, K, n, cp, crow, cslot,
                                                                 (T *)M->Ax, cap, (unsigned)wb);
    return hb_check_launch(ctx, "spai2_kernel");
}

}  // namespace

extern "C" {

int hb_spai2_f64(hb_context *ctx, const hb_ell *A, hb_ell *M)
{
    HB_RANGE("hb_spai2_f64");
    return spai2_impl<double>(ctx, A, M, HB_F64);
}

int hb_spai2_f32(hb_context *ctx, const hb_ell *A, hb_ell *M)
{
    HB_RANGE("hb_spai2_f32");
    return spai2_impl<float>(ctx, A, M, HB_F32);
}

}  // extern "C"
