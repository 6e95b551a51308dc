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

}  // namespace hbd
