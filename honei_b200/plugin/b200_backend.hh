/* b200_backend.hh -- shared pieces of the HONEI plugin that puts tags::GPU::CUDA on the B200
 * backend (libhonei_b200, include/honei_b200.h).
 *
 * The plugin is compiled into HONEI in place of honei/backends/cuda/* and honei/la/*-cuda.cc:
 *   memory_backend_b200.cc  MemoryBackend<tags::GPU::CUDA> (honei/util/memory_backend.hh:131-165)
 *   operations_b200.cc      Product / Defect / DotProduct / Norm / ScaledSum / Scale / Sum /
 *                           Difference / ElementProduct <tags::GPU::CUDA> (declared unconditionally
 *                           in honei/la/*.hh and honei/math/defect.hh)
 *   solvers_b200.hh         full specialisation CGSolver<tags::GPU::CUDA, methods::NONE>: one
 *                           persistent kernel per solve instead of 7 launches per iteration
 */
#pragma once
#ifndef HONEI_B200_PLUGIN_BACKEND_HH
#define HONEI_B200_PLUGIN_BACKEND_HH 1

#include <honei/la/sparse_matrix_ell.hh>
#include <honei/util/exception.hh>

#include <honei_b200.h>

#include <cstdint>
#include <string>

namespace honei
{
    namespace b200
    {
        /// The calling thread's context on the current device (legacy default stream, so it
        /// orders with the memory backend's synchronous copies).
        hb_context * context();

        /// Throws InternalError for a non-zero hb_status.
        void check(int status, const char * what);

        /// Device pointer and upload generation of a block the memory backend holds
        /// (0 / nullptr when it holds none).
        void * device_address(void * memid, void * address);
        std::uint64_t generation(void * memid, void * address);

        /// The hb_ell mirror of a SparseMatrixELL: imported from the backend's copies of
        /// Aj/Ax/Arl on first use, re-imported whenever one of them was uploaded again.
        template <typename DT_> const hb_ell & device_mirror(const SparseMatrixELL<DT_> & a);

        /// Drops mirrors built from this memid (called when the backend frees it).
        void forget(void * memid);
    }
}

#endif
