// hb_internal.cuh -- shared device helpers and the context structure of libhonei_b200.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <string>
#include <mutex>

#include "../../include/honei_b200.h"

#define HB_CUDA_TRY(ctx, call)                                                   \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) { hb_note_error((ctx), e_, #call); return HB_ERR_CUDA; } \
    } while (0)

#define HB_CHECK(cond, code) do { if (!(cond)) return (code); } while (0)

// Device-side status word values (written by bounded waits and input checks).
enum { HB_DEV_OK = 0, HB_DEV_TIMEOUT = 1, HB_DEV_NONFINITE = 2 };

// Bounded wait: a grid barrier gives up after this many nanoseconds (2 s) and reports
// HB_ERR_TIMEOUT; no legitimate phase of any kernel here comes close.
static constexpr uint64_t HB_WAIT_NS = 2000000000ull;

// Scalars a solver kernel reports back (one pinned-host readback per solve).
struct hb_solve_result {
    int64_t used;
    double defect0;
    double defect;
    int32_t status;
    int32_t pad;
};

struct hb_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    // device scratch: reduction partials, barrier words, solver results
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    // device work vectors for solvers (grown on demand, or by hb_reserve)
    void *work = nullptr;
    size_t work_bytes = 0;
    // pinned host slot for scalar readback
    void *pinned = nullptr;
    uint64_t launches = 0;
    // CG on systems that fit: the resident-operator kernel (hb_cg_set_resident)
    int cg_resident = 1;
    // streaming CG: one row per thread (cg_row_kernel) or groups of four rows (hb_cg_set_layout)
    int cg_row_layout = 0;
    // threads per block chosen by the caller for a kernel family (hb_set_block_size); 0 = default
    int block[3] = {0, 0, 0};
    std::string last_error;
};

// An NVTX range around each compute entry point (named after it), for nsys / ncu
// (--nvtx --nvtx-include "hb_cg_f64/").  NVTX v3 is header-only: without a tool attached a
// push / pop is a check of one function pointer.
struct HbRange {
    explicit HbRange(const char *name) { nvtxRangePushA(name); }
    ~HbRange() { nvtxRangePop(); }
    HbRange(const HbRange &) = delete;
    HbRange &operator=(const HbRange &) = delete;
};
#define HB_RANGE(name) HbRange hb_range_guard_(name)

void hb_note_error(hb_context *ctx, cudaError_t e, const char *what);
int hb_ensure_work(hb_context *ctx, size_t bytes);
int hb_check_launch(hb_context *ctx, const char *what);

// Scratch map (bytes from ctx->scratch): partial sums, barrier words, result slots.
static constexpr size_t HB_PARTIALS = 8192;                    // doubles
static constexpr size_t HB_OFF_PARTIALS = 0;
static constexpr size_t HB_OFF_BAR = HB_PARTIALS * 8;          // 64 unsigned words
static constexpr size_t HB_OFF_RESULT = HB_OFF_BAR + 256;      // hb_solve_result[16]
static constexpr size_t HB_OFF_SCALAR = HB_OFF_RESULT + 16 * sizeof(hb_solve_result);
static constexpr size_t HB_SCRATCH_BYTES = HB_OFF_SCALAR + 4096;

inline double *hb_partials(hb_context *c) { return (double *)((char *)c->scratch + HB_OFF_PARTIALS); }
inline unsigned *hb_bar(hb_context *c) { return (unsigned *)((char *)c->scratch + HB_OFF_BAR); }
inline hb_solve_result *hb_result(hb_context *c) { return (hb_solve_result *)((char *)c->scratch + HB_OFF_RESULT); }
inline double *hb_scalars(hb_context *c) { return (double *)((char *)c->scratch + HB_OFF_SCALAR); }

inline int64_t hb_round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Output modes of the SpMV family (hb_ell.cu).
enum { HB_MODE_SPMV = 0, HB_MODE_DEFECT = 1, HB_MODE_ADD = 2, HB_MODE_JACOBI = 3 };

int hb_check_ell(const hb_ell *A, int dtype);
// y = A x | b - A x | y + A x | x + P (b - A x), asynchronous on ctx->stream.
template <typename T>
int hb_launch_spmv_mode(hb_context *ctx, const hb_ell *A, int mode, const T *x, const T *b, const T *P, T *y);
// P[i] = damping / A(i, i)
template <typename T> int hb_launch_jacobi_diag(hb_context *ctx, const hb_ell *A, T damping, T *P);
// Banded Q1 level operator in the fused ELL modes (SPMV / DEFECT / JACOBI), summed in the ELL
// row's column order, and the matrix-free PROLMAT-order transfers of a (2^k + 1)^2 grid of
// fine side Mf (y += P c; d = P^T f), all bit-identical to the ELL kernels on the same matrices.
template <typename T>
int hb_launch_band_mode(hb_context *ctx, const hb_q1band *A, int mode, const T *x, const T *b, const T *P, T *y);
template <typename T> int hb_launch_prolong_add(hb_context *ctx, int64_t Mf, T *y, const T *c);
template <typename T> int hb_launch_restrict_pt(hb_context *ctx, int64_t Mf, T *d, const T *f);
// Sum of squares / dot product into a device scalar (no host sync).
template <typename T> int hb_launch_dot(hb_context *ctx, int64_t n, const T *x, const T *y, T *out_dev);
// Plain CG (cg.hh semantics) as one persistent kernel, asynchronous: work = 5 * ld entries,
// result written to *res on the device.
template <typename T>
int hb_launch_cg(hb_context *ctx, const hb_ell *A, const T *b, T *x, int64_t max_iters, T eps, T *work,
                 hb_solve_result *res);

// MG-preconditioned CG in FP32 on the finest level of an FP32 hierarchy (hb_mg.cu).
struct hb_mg;
int hb_mg_pcg_f32(hb_mg *mg, const float *b, float *x, float eps, int64_t max_iters, float *work, int64_t *used);
int hb_mg_finest(hb_mg *mg, hb_ell *A);
int hb_mg_set_dense_coarse(hb_mg *mg, void *inv);
int hb_mg_pcg_f32_graph(hb_mg *mg, cudaStream_t capture_stream, const float *b, float *x, float eps, int64_t max_iters,
                        float *work, cudaGraphExec_t *graph, int check_every, int64_t *used);

// Device pointers of a served system (hb_q1) for kernels that run its solve themselves (the
// batched served solve): levels coarsest first, P32[l] / R32[l] transfer between levels l and
// l + 1, per-level FP32 vectors of the MG hierarchy (Jacobi diagonal, coarse solution c and
// right-hand side d, smoother ping-pong xt, defect store), the finest FP64 matrix and the
// refinement / PCG vectors.
constexpr int HB_Q1_MAXL = 16;
struct hb_q1_view {
    int L = 0;
    hb_ell A64{};
    hb_ell A32[HB_Q1_MAXL], P32[HB_Q1_MAXL], R32[HB_Q1_MAXL];
    hb_q1band B32[HB_Q1_MAXL];   // banded copies of the FP32 levels
    float *jac[HB_Q1_MAXL], *c[HB_Q1_MAXL], *d[HB_Q1_MAXL], *store[HB_Q1_MAXL], *xt[HB_Q1_MAXL];
    const float *coarse_inv = nullptr;
    double *r64 = nullptr;
    float *b32 = nullptr, *x32 = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *v = nullptr;
    int n_pre = 2, n_post = 2;
    hb_context *ctx = nullptr;
};
int hb_mg_view(const hb_mg *mg, hb_q1_view *out);
int hb_q1_view_of(const hb_q1 *q, hb_q1_view *out);
// The fused coarse cycle: levels 0..top of a served system's banded FP32 hierarchy as one
// single-cluster launch (a device descriptor built once; hb_tail_launch runs the V-cycle of
// those levels on X = z, zero on entry, and B = r, with the same arithmetic as the per-level
// kernels).  hb_mg_enable_tail switches an hb_mg's cycle to it for the levels of at most max_rows
// rows (0: per-level kernels only).
// Off by default: measured on B200, graph-replayed per-level kernels (about 1.5 us each) beat one
// 16-CTA cluster with a barrier per phase for single solves (65^2 .. 2049^2).
constexpr int64_t HB_TAIL_DEFAULT_ROWS = 0;
int hb_tail_create(hb_context *ctx, const hb_q1_view &v, int top, void **desc);
int hb_tail_launch(hb_context *ctx, const void *desc, float *z, const float *r);
int hb_mg_enable_tail(hb_mg *mg, int64_t max_rows);

// --------------------------------------------------------------------------------------
// Device helpers
// --------------------------------------------------------------------------------------
namespace hbd {

// One rounding per multiply and per add (no FMA contraction): the reference's CPU order.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }

template <typename T> struct vec4;
template <> struct vec4<double> { double2 a, b; };
template <> struct vec4<float> { float4 a; };

// Streaming (evict-first) 4-wide loads of matrix data: the matrix is touched once per
// operator application, the vectors are the reusable part of L2.
__device__ __forceinline__ void ld4_stream(const double *p, double (&v)[4])
{
    double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
    double2 b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4_stream(const float *p, float (&v)[4])
{
    float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void ld4_stream(const int32_t *p, int32_t (&v)[4])
{
    int4 a = __ldcs(reinterpret_cast<const int4 *>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
// Cached 4-wide loads / stores of padded work vectors (16-byte aligned by construction).
__device__ __forceinline__ void ld4(const double *p, double (&v)[4])
{
    double2 a = *reinterpret_cast<const double2 *>(p);
    double2 b = *(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4(const float *p, float (&v)[4])
{
    float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void st4(double *p, const double (&v)[4])
{
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void red_release_add(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Warp tree sum in a fixed order (shuffle-down halving): deterministic.
template <typename T> __device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = add(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block sum in a fixed order; result valid in thread 0.  smem: >= 32 entries.
template <typename T> __device__ __forceinline__ T block_sum(T v, T *smem)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nwarps ? smem[lane] : T(0);
        v = warp_sum(v);
    }
    return v;
}

// Grid barrier for cooperative (co-resident) launches: generation counter + arrival count.
// Every wait is bounded (HB_WAIT_NS); on timeout the status word gets HB_DEV_TIMEOUT and all
// blocks return false, so the kernel ends instead of hanging.
struct GridBarrier {
    unsigned *count;
    unsigned *gen;
    int *status;

    __device__ __forceinline__ bool sync(unsigned nblocks, int *s_flag) const
    {
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            const unsigned g = ld_acquire(gen);
            __threadfence();
            const unsigned arrived = atomicAdd(count, 1u);
            if (arrived == nblocks - 1) {
                atomicExch(count, 0u);
                __threadfence();
                st_release(gen, g + 1);
            } else {
                const uint64_t t0 = globaltimer();
                while (ld_acquire(gen) == g) {
                    if (*(volatile int *)status != HB_DEV_OK) { ok = 0; break; }
                    if (globaltimer() - t0 > HB_WAIT_NS) {
                        atomicCAS(status, HB_DEV_OK, HB_DEV_TIMEOUT);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
            if (*(volatile int *)status != HB_DEV_OK) ok = 0;
            *s_flag = ok;
        }
        __syncthreads();
        return *(volatile int *)s_flag != 0;
    }
};

// Grid-wide exchange of one partial per block, for cooperative launches, on a monotonic
// arrival counter (zero before the launch).  Exchange e: thread 0 stores the block's partial in
// slot array e & 1, adds 1 to the counter with release semantics (fire and forget) and waits
// until the counter reaches (e + 1) * blocks; every block may then read all partials of e, and
// everything the other blocks wrote before arriving.  Two slot arrays suffice: a block reaches
// exchange e + 2 only after every block arrived at e + 1, i.e. after every block read e.
// The barrier form (arrive) publishes whatever thread 0 of each block stored before it; a slot
// written at exchange e may be rewritten at e + 2 at the earliest, by the same argument.
// Waits are bounded like GridBarrier's (HB_WAIT_NS, HB_DEV_TIMEOUT in the status word; a block
// that sees another block's failure leaves too).
struct CountExchange {
    unsigned *count;
    int *status;

    template <typename T>
    __device__ __forceinline__ bool arrive_wait(T partial, T *slots, unsigned e, unsigned nblocks, int *s_flag) const
    {
        if (threadIdx.x == 0) __stcg(slots + (e & 1u) * nblocks + blockIdx.x, partial);
        return arrive(e, nblocks, s_flag);
    }

    __device__ __forceinline__ bool arrive(unsigned e, unsigned nblocks, int *s_flag) const
    {
        __syncthreads();
        return arrive_synced(e, nblocks, s_flag);
    }

    // arrive() for callers whose threads passed a __syncthreads after their last global store
    // (a block reduction ending in one): thread 0's release then covers those stores already
    __device__ __forceinline__ bool arrive_synced(unsigned e, unsigned nblocks, int *s_flag) const
    {
        if (threadIdx.x == 0) {
            int ok = 1;
            red_release_add(count, 1u);
            const unsigned target = (e + 1u) * nblocks;
            if ((int)(ld_acquire(count) - target) < 0) {
                const uint64_t t0 = globaltimer();
                unsigned n = 0;
                while ((int)(ld_acquire(count) - target) < 0) {
                    if ((++n & 31u) == 0 && *(volatile int *)status != HB_DEV_OK) { ok = 0; break; }
                    if (globaltimer() - t0 > HB_WAIT_NS) {
                        atomicCAS(status, HB_DEV_OK, HB_DEV_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
            *s_flag = ok;
        }
        __syncthreads();
        return *(volatile int *)s_flag != 0;
    }
};

}  // namespace hbd
