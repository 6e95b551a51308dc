// hb_spmv_core.cuh -- the per-row-group ELL product shared by the SpMV, CG, MG and batched
// kernels: one thread, 4 consecutive rows, slots in the reference order, 16-byte streaming
// loads of Aj/Ax, a caller-supplied gather for the vector entry of column j.
#pragma once
#include "hb_internal.cuh"

namespace hbd {

// sum[i] = sum_k Ax[k*ld + r0 + i] * gather(Aj[k*ld + r0 + i]) over valid slots (Aj >= 0),
// accumulated left to right with one rounding per multiply and add.
// KT > 0: K is a compile-time constant, all slot loads first; KT == 0: runtime K, 4 slots per
// chunk.
// CH = slots whose loads are in flight together (register budget); CH >= KT loads every slot
// before the first gather.
template <typename T, int KT, int CH = (KT > 0 ? KT : 4), typename Gather>
__device__ __forceinline__ void ell_rows4(const int32_t *__restrict__ Aj, const T *__restrict__ Ax,
                                          int64_t ld, int K, int64_t r0, Gather gather, T (&sum)[4])
{
#pragma unroll
    for (int i = 0; i < 4; ++i) sum[i] = T(0);
    if (KT > 0 && CH >= KT) {
        // every slot's Aj/Ax load issued before the first gather: one memory round trip
        int32_t j[KT > 0 ? KT : 1][4];
        T a[KT > 0 ? KT : 1][4];
#pragma unroll
        for (int k = 0; k < KT; ++k) {
            ld4_stream(Aj + (int64_t)k * ld + r0, j[k]);
            ld4_stream(Ax + (int64_t)k * ld + r0, a[k]);
        }
#pragma unroll
        for (int k = 0; k < KT; ++k)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (j[k][i] >= 0) sum[i] = add(sum[i], mul(a[k][i], gather(j[k][i])));
        return;
    }
    const int kend = KT > 0 ? KT : K;
#pragma unroll
    for (int k0 = 0; k0 < kend; k0 += CH) {
        int32_t j[CH][4];
        T a[CH][4];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            if (k0 + c < kend) {
                ld4_stream(Aj + (int64_t)(k0 + c) * ld + r0, j[c]);
                ld4_stream(Ax + (int64_t)(k0 + c) * ld + r0, a[c]);
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) { j[c][i] = -1; a[c][i] = T(0); }
            }
        }
        T xv[CH][4];
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i) xv[c][i] = j[c][i] >= 0 ? gather(j[c][i]) : T(0);
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (j[c][i] >= 0) sum[i] = add(sum[i], mul(a[c][i], xv[c][i]));
    }
}


// Lane-strided quads: quad q holds rows tile*128 + lane + w*i (i = 0..3) of its 128-row tile
// (tile = q / 32, lane = q % 32, w = quads in that tile, 32 except in a last partial tile), so a
// warp's 32 lanes read 32 consecutive rows per instruction.
__device__ __forceinline__ void quad_rows(int64_t q, int64_t groups, uint32_t (&row)[4])
{
    const int64_t tile = q >> 5;
    const int64_t left = groups - (tile << 5);
    const uint32_t w = (uint32_t)(left < 32 ? left : 32);
    const uint32_t base = (uint32_t)((tile << 7) + (q & 31));
#pragma unroll
    for (int i = 0; i < 4; ++i) row[i] = base + w * (uint32_t)i;
}

// ell_rows4 on the rows of a lane-strided quad: the loads of CH slots at a time (all of them for
// CH >= KT), then their gathers, in slot order.
template <typename T, int KT, int CH = (KT > 0 ? KT : 4), typename Gather>
__device__ __forceinline__ void ell_rows4s(const int32_t *__restrict__ Aj, const T *__restrict__ Ax, int64_t ld,
                                           int K, const uint32_t (&row)[4], Gather gather, T (&sum)[4])
{
#pragma unroll
    for (int i = 0; i < 4; ++i) sum[i] = T(0);
    const int kend = KT > 0 ? KT : K;
#pragma unroll
    for (int k0 = 0; k0 < kend; k0 += CH) {
        int32_t j[CH][4];
        T a[CH][4];
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const bool in = k0 + c < kend;
                j[c][i] = in ? __ldcs(Aj + (int64_t)(k0 + c) * ld + row[i]) : -1;
                a[c][i] = in ? __ldcs(Ax + (int64_t)(k0 + c) * ld + row[i]) : T(0);
            }
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (j[c][i] >= 0) sum[i] = add(sum[i], mul(a[c][i], gather(j[c][i])));
    }
}

}  // namespace hbd
