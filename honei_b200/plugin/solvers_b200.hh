/* solvers_b200.hh -- full specialisation CGSolver<tags::GPU::CUDA, methods::NONE> on the B200
 * backend.
 *
 * HONEI's generic CGSolver<Tag_, methods::NONE> (honei/math/cg.hh:63-133) already runs on the GPU
 * tag through the operators in operations_b200.cc: 7 operator calls and 2 scalar read-backs per
 * iteration.  Including this header replaces it, for tags::GPU::CUDA only, with one persistent
 * kernel per solve (hb_cg_f64 / hb_cg_f32): same update formulas, same guarded divisions, same
 * dual stopping rule, same used_iters semantics; scalars stay on the device.  Call sites stay
 * unchanged (a full specialisation beats the partial one).  Include it in every translation
 * unit that instantiates CGSolver<tags::GPU::CUDA, methods::NONE>, before that instantiation.
 */
#pragma once
#ifndef HONEI_B200_PLUGIN_SOLVERS_HH
#define HONEI_B200_PLUGIN_SOLVERS_HH 1

#include "b200_backend.hh"

#include <honei/la/dense_vector.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/la/vector_error.hh>
#include <honei/math/cg.hh>
#include <honei/math/methods.hh>
#include <honei/util/tags.hh>

namespace honei
{
    template <> struct CGSolver<tags::GPU::CUDA, methods::NONE>
    {
        private:
            static int solve(const hb_ell & A, const double * b, double * x, unsigned long max_iters, double eps,
                    int64_t & used)
            {
                return hb_cg_f64(b200::context(), &A, b, x, (int64_t)max_iters, eps, &used, nullptr);
            }

            static int solve(const hb_ell & A, const float * b, float * x, unsigned long max_iters, float eps,
                    int64_t & used)
            {
                return hb_cg_f32(b200::context(), &A, b, x, (int64_t)max_iters, eps, &used, nullptr);
            }

        public:
            template <typename DT_, typename MatDT_, typename PreconContType_>
            static inline DenseVector<MatDT_> & value(SparseMatrixELL<MatDT_> & A, PreconContType_ & /*P*/,
                    DenseVector<MatDT_> & b, DenseVector<MatDT_> & x, unsigned long max_iters,
                    unsigned long & used_iters, DT_ eps_relative = 1e-8)
            {
                CONTEXT("When solving linear system with CG (B200 persistent kernel):");
                if (b.size() != A.rows())
                    throw VectorSizeDoesNotMatch(b.size(), A.rows());
                if (x.size() != A.columns())
                    throw VectorSizeDoesNotMatch(x.size(), A.columns());
                const hb_ell & Ad(b200::device_mirror(A));
                void * bd(b.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                void * xd(x.lock(lm_read_and_write, tags::GPU::CUDA::memory_value));
                int64_t used(0);
                const int st(solve(Ad, (const MatDT_ *)bd, (MatDT_ *)xd, max_iters, (MatDT_)eps_relative, used));
                b.unlock(lm_read_only);
                x.unlock(lm_read_and_write);
                b200::check(st, "CGSolver<GPU::CUDA, NONE>");
                // cg.hh sets used_iters only when it stops (convergence or max_iters)
                if (used > 0)
                    used_iters = (unsigned long)used;
                return x;
            }
    };
}

#endif
