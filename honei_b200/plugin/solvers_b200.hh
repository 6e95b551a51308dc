/* solvers_b200.hh -- full specialisations CGSolver<tags::GPU::CUDA, methods::NONE> and
 * CGSolver<tags::GPU::CUDA, methods::VAR> on the B200 backend.
 *
 * HONEI's generic CGSolver<Tag_, methods::NONE> (honei/math/cg.hh:63-133) already runs on the GPU
 * tag through the operators in operations_b200.cc: 7 operator calls and 2 scalar read-backs per
 * iteration.  Including this header replaces it, for tags::GPU::CUDA only, with one persistent
 * kernel per solve (hb_cg_f64 / hb_cg_f32): same update formulas, same guarded divisions, same
 * dual stopping rule, same used_iters semantics; scalars stay on the device.  Call sites stay
 * unchanged (a full specialisation beats the partial one).  Include it in every translation
 * unit that instantiates CGSolver<tags::GPU::CUDA, methods::NONE>, before that instantiation.
 *
 * CGSolver<tags::GPU::CUDA, methods::VAR> (honei/math/cg.hh:140-219) likewise becomes one
 * persistent kernel (hb_cg_var_diag_* for a DenseVector preconditioner, hb_cg_var_ell_* for a
 * SparseMatrixELL one), with the reference's sign-keeping guards and stopping tests.
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

    template <> struct CGSolver<tags::GPU::CUDA, methods::VAR>
    {
        private:
            static int solve(const hb_ell & A, const double * P, const double * b, double * x, unsigned long n,
                    double eps, int64_t & used)
            { return hb_cg_var_diag_f64(b200::context(), &A, P, b, x, (int64_t)n, eps, &used, nullptr); }
            static int solve(const hb_ell & A, const float * P, const float * b, float * x, unsigned long n,
                    float eps, int64_t & used)
            { return hb_cg_var_diag_f32(b200::context(), &A, P, b, x, (int64_t)n, eps, &used, nullptr); }
            static int solve(const hb_ell & A, const hb_ell & P, const double * b, double * x, unsigned long n,
                    double eps, int64_t & used)
            { return hb_cg_var_ell_f64(b200::context(), &A, &P, b, x, (int64_t)n, eps, &used, nullptr); }
            static int solve(const hb_ell & A, const hb_ell & P, const float * b, float * x, unsigned long n,
                    float eps, int64_t & used)
            { return hb_cg_var_ell_f32(b200::context(), &A, &P, b, x, (int64_t)n, eps, &used, nullptr); }

            template <typename MatDT_> static void check_sizes(const SparseMatrixELL<MatDT_> & A,
                    const DenseVector<MatDT_> & b, const DenseVector<MatDT_> & x)
            {
                if (b.size() != A.rows())
                    throw VectorSizeDoesNotMatch(b.size(), A.rows());
                if (x.size() != A.columns())
                    throw VectorSizeDoesNotMatch(x.size(), A.columns());
            }

            template <typename MatDT_, typename PD_> static void run(const hb_ell & Ad, const PD_ & Pd,
                    DenseVector<MatDT_> & b, DenseVector<MatDT_> & x, unsigned long max_iters,
                    unsigned long & used_iters, MatDT_ eps)
            {
                void * bd(b.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                void * xd(x.lock(lm_read_and_write, tags::GPU::CUDA::memory_value));
                int64_t used(0);
                const int st(solve(Ad, Pd, (const MatDT_ *)bd, (MatDT_ *)xd, max_iters, eps, used));
                b.unlock(lm_read_only);
                x.unlock(lm_read_and_write);
                b200::check(st, "CGSolver<GPU::CUDA, VAR>");
                if (used > 0)
                    used_iters = (unsigned long)used;
            }

        public:
            /// Vector preconditioner: z = P r elementwise (e.g. Jacobi damping / diag(A)).
            template <typename DT_, typename MatDT_>
            static inline DenseVector<MatDT_> & value(SparseMatrixELL<MatDT_> & A, DenseVector<MatDT_> & P,
                    DenseVector<MatDT_> & b, DenseVector<MatDT_> & x, unsigned long max_iters,
                    unsigned long & used_iters, DT_ eps_relative = 1e-8)
            {
                CONTEXT("When solving linear system with preconditioned CG (B200 persistent kernel):");
                check_sizes(A, b, x);
                if (P.size() != A.rows())
                    throw VectorSizeDoesNotMatch(P.size(), A.rows());
                const hb_ell & Ad(b200::device_mirror(A));
                void * pd(P.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                run(Ad, (const MatDT_ *)pd, b, x, max_iters, used_iters, (MatDT_)eps_relative);
                P.unlock(lm_read_only);
                return x;
            }

            /// Matrix preconditioner: z = P r (e.g. SPAI / SAINV approximate inverses).
            template <typename DT_, typename MatDT_>
            static inline DenseVector<MatDT_> & value(SparseMatrixELL<MatDT_> & A, SparseMatrixELL<MatDT_> & P,
                    DenseVector<MatDT_> & b, DenseVector<MatDT_> & x, unsigned long max_iters,
                    unsigned long & used_iters, DT_ eps_relative = 1e-8)
            {
                CONTEXT("When solving linear system with preconditioned CG (B200 persistent kernel):");
                check_sizes(A, b, x);
                if (P.rows() != A.rows() || P.columns() != A.columns())
                    throw VectorSizeDoesNotMatch(P.rows(), A.rows());
                const hb_ell & Ad(b200::device_mirror(A));
                const hb_ell & Pm(b200::device_mirror(P));
                run(Ad, Pm, b, x, max_iters, used_iters, (MatDT_)eps_relative);
                return x;
            }
    };
}

#endif
