/* mg_b200.hh -- HONEI's multigrid path on the B200 backend: full specialisations of
 *
 *   RISmoother<tags::GPU::CUDA>                (honei/math/ri.hh:97-133)
 *   MGCycleCreation<tags::GPU::CUDA, methods::CYCLE::V::STATIC, CGSolver<tags::GPU::CUDA, NONE>,
 *       RISmoother<tags::GPU::CUDA>, Restriction<tags::GPU::CUDA, PROLMAT>,
 *       Prolongation<tags::GPU::CUDA, PROLMAT>, DT_>   (honei/math/mg.hh:567-662)
 *   MGSolver<tags::GPU::CUDA, Norm<vnt_l_two, true, tags::GPU::CUDA> >   (honei/math/mg.hh:1094-1127)
 *
 * HONEI's generic templates already run on the GPU tag through operations_b200.cc, one operator
 * call per step of the cycle.  With this header included (before the instantiations, in every
 * translation unit that instantiates them) the same call sites run:
 *   - every smoothing step as fused sweeps x = x + P (b - A x) (hb_jacobi_sweeps_*), rounding as
 *     Defect, Product(P, .) and Sum do;
 *   - a V::STATIC cycle as one operator that drives the whole cycle through the backend's
 *     multigrid object (hb_mg_*): fused smoother / defect / prolongation-and-sum kernels, the
 *     coarse CG as one persistent kernel, the cycle replayed from a CUDA graph inside MGSolver;
 *   - MGSolver's loop as hb_mg_solve (the defect norm read back once per cycle).
 * The cycle operator takes the data's matrices, transfer matrices and smoother vectors P as they
 * are (SparseMatrixELL / DenseVector, the types MGUtil::load_data builds), and the sweep counts,
 * coarse iteration cap, eps and min_level from MGData.  Every elementwise and per-row operation
 * is bit-identical to tags::CPU; only the coarse CG's dot products are summed in another (fixed)
 * order.  IRSolver<tags::GPU::CUDA, tags::GPU::CUDA, Norm<vnt_l_two, true, tags::GPU::CUDA> >
 * (honei/math/ir.hh:30-78) needs no specialisation: its inner MGSolver call lands here.
 *
 * A cycle built for other container types, or an OperatorList assembled by hand, runs the
 * generic way (MGSolver below falls back to the reference's loop for any list that is not one
 * of these cycle operators).  The cycle operator keeps a pointer to the MGData it was built
 * from: that MGData must outlive the OperatorList (as it does when both are locals of one
 * scope, the data declared first).
 */
#pragma once
#ifndef HONEI_B200_PLUGIN_MG_HH
#define HONEI_B200_PLUGIN_MG_HH 1

#include "b200_backend.hh"
#include "solvers_b200.hh"

#include <honei/la/dense_vector.hh>
#include <honei/la/norm.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/la/sum.hh>
#include <honei/la/product.hh>
#include <honei/la/vector_error.hh>
#include <honei/math/defect.hh>
#include <honei/math/methods.hh>
#include <honei/math/mg.hh>
#include <honei/math/operator.hh>
#include <honei/math/operator_list.hh>
#include <honei/math/prolongation.hh>
#include <honei/math/restriction.hh>
#include <honei/math/ri.hh>
#include <honei/util/tags.hh>

#include <cstdint>
#include <iostream>
#include <vector>

namespace honei
{
    namespace b200
    {
        inline int jacobi_sweeps(const hb_ell & A, const double * P, const double * b, double * x, double * t,
                unsigned long n)
        { return hb_jacobi_sweeps_f64(context(), &A, P, b, x, t, (int64_t)n); }
        inline int jacobi_sweeps(const hb_ell & A, const float * P, const float * b, float * x, float * t,
                unsigned long n)
        { return hb_jacobi_sweeps_f32(context(), &A, P, b, x, t, (int64_t)n); }
        inline int mg_cycle(hb_mg * mg, const double * b, double * x) { return hb_mg_cycle_f64(mg, b, x); }
        inline int mg_cycle(hb_mg * mg, const float * b, float * x) { return hb_mg_cycle_f32(mg, b, x); }
        inline int mg_solve(hb_mg * mg, const double * b, double * x, int64_t * used, double * rn)
        { return hb_mg_solve_f64(mg, b, x, used, rn); }
        inline int mg_solve(hb_mg * mg, const float * b, float * x, int64_t * used, float * rn)
        { return hb_mg_solve_f32(mg, b, x, used, rn); }

        /// One V::STATIC cycle over an MGData of SparseMatrixELL / DenseVector containers, run by
        /// the backend's multigrid object.  Built by the MGCycleCreation specialisation below.
        template <typename DT_> class MGCycleOperator :
            public Operator
        {
            public:
                typedef MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_> Data;

            private:
                Data * _data;
                hb_mg * _mg;
                std::vector<hb_ell> _A, _prol, _res;
                std::vector<void *> _P_dev;
                std::vector<std::uint64_t> _P_gen;
                hb_mg_params _prm;

                static bool same(const hb_ell & a, const hb_ell & b)
                {
                    return a.Aj == b.Aj && a.Ax == b.Ax && a.rows == b.rows && a.cols == b.cols && a.K == b.K
                        && a.ld == b.ld;
                }

                /// The multigrid object for the data's current matrices and parameters; the
                /// smoother vectors copied in whenever the backend uploaded them anew.
                void ensure()
                {
                    Data & d(*_data);
                    const unsigned long top(d.A.size()), low(d.min_level);
                    if (low < 1 || low > top)
                        throw InternalError("B200 MG cycle: min_level outside the hierarchy");
                    std::vector<hb_ell> A, prol, res;
                    for (unsigned long level(low) ; level <= top ; ++level)
                    {
                        A.push_back(device_mirror(d.A.at(MGDataIndex::internal_index_A(level))));
                        if (level < top)
                        {
                            prol.push_back(device_mirror(d.prolmat.at(MGDataIndex::internal_index_Prol(level + 1))));
                            res.push_back(device_mirror(d.resmat.at(MGDataIndex::internal_index_Prol(level + 1))));
                        }
                    }
                    hb_mg_params prm;
                    prm.max_iters = (int64_t)d.max_iters;
                    prm.max_iters_coarse = (int64_t)d.max_iters_coarse;
                    prm.n_pre = (int64_t)d.n_pre_smooth;
                    prm.n_post = (int64_t)d.n_post_smooth;
                    prm.damping = 0.7;      // unused: the smoother vectors come from the data
                    prm.eps = (double)d.eps_relative;
                    bool rebuild(_mg == nullptr || A.size() != _A.size());
                    for (unsigned long i(0) ; ! rebuild && i < A.size() ; ++i)
                        rebuild = ! same(A[i], _A[i]);
                    for (unsigned long i(0) ; ! rebuild && i < prol.size() ; ++i)
                        rebuild = ! same(prol[i], _prol[i]) || ! same(res[i], _res[i]);
                    if (rebuild)
                    {
                        if (_mg)
                            hb_mg_destroy(_mg);
                        _mg = nullptr;
                        check(hb_mg_create(context(), (int)A.size(), A.data(), prol.empty() ? nullptr : prol.data(),
                                    res.empty() ? nullptr : res.data(), &prm, &_mg), "B200 MG cycle: hb_mg_create");
                        _A = A;
                        _prol = prol;
                        _res = res;
                        _prm = prm;
                        _P_dev.assign(A.size(), nullptr);
                        _P_gen.assign(A.size(), 0);
                    }
                    else if (prm.max_iters != _prm.max_iters || prm.max_iters_coarse != _prm.max_iters_coarse
                            || prm.n_pre != _prm.n_pre || prm.n_post != _prm.n_post || prm.eps != _prm.eps)
                    {
                        check(hb_mg_set_params(_mg, &prm), "B200 MG cycle: hb_mg_set_params");
                        _prm = prm;
                    }
                    for (unsigned long level(low), i(0) ; level <= top ; ++level, ++i)
                    {
                        DenseVector<DT_> & P(d.P.at(MGDataIndex::internal_index_A(level)));
                        if (P.size() != d.A.at(MGDataIndex::internal_index_A(level)).rows())
                            throw VectorSizeDoesNotMatch(P.size(), d.A.at(MGDataIndex::internal_index_A(level)).rows());
                        void * p(P.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                        const std::uint64_t g(generation(P.memid(), P.address()));
                        int st(HB_OK);
                        if (p != _P_dev[i] || g != _P_gen[i])
                            st = hb_mg_set_smoother(_mg, (int)i, p);
                        P.unlock(lm_read_only);
                        check(st, "B200 MG cycle: hb_mg_set_smoother");
                        _P_dev[i] = p;
                        _P_gen[i] = g;
                    }
                }

            public:
                explicit MGCycleOperator(Data & data) :
                    _data(&data),
                    _mg(nullptr)
                {
                }

                virtual ~MGCycleOperator()
                {
                    if (_mg)
                        hb_mg_destroy(_mg);
                }

                virtual std::string to_string()
                {
                    return "B200 MGCycleOperator (V::STATIC, CGSolver<NONE>, RISmoother, PROLMAT)";
                }

                const Data * data() const
                {
                    return _data;
                }

                /// One cycle on the finest level: what the generic cycle's operators do in turn.
                virtual void value()
                {
                    ensure();
                    DenseVector<DT_> & b(_data->b.back());
                    DenseVector<DT_> & x(_data->x.back());
                    void * bd(b.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                    void * xd(x.lock(lm_read_and_write, tags::GPU::CUDA::memory_value));
                    const int st(mg_cycle(_mg, (const DT_ *)bd, (DT_ *)xd));
                    b.unlock(lm_read_only);
                    x.unlock(lm_read_and_write);
                    check(st, "B200 MG cycle");
                }

                /// MGSolver's loop (honei/math/mg.hh:1098-1126) on the finest level: data.used_iters
                /// and the initial / final defect norms.
                void solve(DT_ & rnorm_initial, DT_ & rnorm_final)
                {
                    ensure();
                    DenseVector<DT_> & b(_data->b.back());
                    DenseVector<DT_> & x(_data->x.back());
                    void * bd(b.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                    void * xd(x.lock(lm_read_and_write, tags::GPU::CUDA::memory_value));
                    int64_t used(0);
                    DT_ rn[2] = {DT_(0), DT_(0)};
                    const int st(mg_solve(_mg, (const DT_ *)bd, (DT_ *)xd, &used, rn));
                    b.unlock(lm_read_only);
                    x.unlock(lm_read_and_write);
                    check(st, "B200 MGSolver");
                    _data->used_iters = (unsigned long)used;
                    rnorm_initial = rn[0];
                    rnorm_final = rn[1];
                }
        };
    }

    template <> struct RISmoother<tags::GPU::CUDA>
    {
        public:
            static const unsigned long NUM_TEMPVECS = 2;

            /// A vector preconditioner: each sweep one fused kernel (x = x + P (b - A x)).
            template <typename DT_>
            static void value(SparseMatrixELL<DT_> & A, DenseVector<DT_> & P, DenseVector<DT_> & b,
                    DenseVector<DT_> & x, std::vector<DenseVector<DT_> > & temp_vecs, unsigned long max_iters)
            {
                CONTEXT("When smoothing with Richardson (B200 fused sweeps): ");
                if (b.size() != A.rows())
                    throw VectorSizeDoesNotMatch(b.size(), A.rows());
                if (x.size() != A.columns() || x.size() != A.rows())
                    throw VectorSizeDoesNotMatch(x.size(), A.rows());
                if (P.size() != A.rows())
                    throw VectorSizeDoesNotMatch(P.size(), A.rows());
                if (temp_vecs.empty() || temp_vecs[0].size() != A.rows())
                    throw VectorSizeDoesNotMatch(temp_vecs.empty() ? 0 : temp_vecs[0].size(), A.rows());
                if (max_iters == 0)
                    return;
                const hb_ell & Ad(b200::device_mirror(A));
                void * pd(P.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                void * bd(b.lock(lm_read_only, tags::GPU::CUDA::memory_value));
                void * xd(x.lock(lm_read_and_write, tags::GPU::CUDA::memory_value));
                void * td(temp_vecs[0].lock(lm_write_only, tags::GPU::CUDA::memory_value));
                const int st(b200::jacobi_sweeps(Ad, (const DT_ *)pd, (const DT_ *)bd, (DT_ *)xd, (DT_ *)td, max_iters));
                temp_vecs[0].unlock(lm_write_only);
                x.unlock(lm_read_and_write);
                b.unlock(lm_read_only);
                P.unlock(lm_read_only);
                b200::check(st, "RISmoother<GPU::CUDA>");
            }

            /// Any other preconditioner (e.g. a SparseMatrixELL): the reference's three operators
            /// per sweep on the GPU tag.
            template <typename MatrixType_, typename VectorType_, typename PreconContType_>
            static void value(MatrixType_ & A, PreconContType_ & P, VectorType_ & b, VectorType_ & x,
                    std::vector<VectorType_> & temp_vecs, unsigned long max_iters)
            {
                CONTEXT("When smoothing with Richardson: ");
                VectorType_ temp_0(temp_vecs[0]);
                VectorType_ temp_1(temp_vecs[1]);
                for (unsigned long i(0) ; i < max_iters ; ++i)
                {
                    Defect<tags::GPU::CUDA>::value(temp_0, b, A, x);
                    Product<tags::GPU::CUDA>::value(temp_1, P, temp_0);
                    Sum<tags::GPU::CUDA>::value(x, temp_1);
                }
            }
    };

    template <typename DataType_>
    struct MGCycleCreation<tags::GPU::CUDA, methods::CYCLE::V::STATIC, CGSolver<tags::GPU::CUDA, methods::NONE>,
        RISmoother<tags::GPU::CUDA>, Restriction<tags::GPU::CUDA, methods::PROLMAT>,
        Prolongation<tags::GPU::CUDA, methods::PROLMAT>, DataType_>
    {
        public:
            /// The whole V-cycle as one operator (b200::MGCycleOperator) over the data.
            static OperatorList value(MGData<SparseMatrixELL<DataType_>, DenseVector<DataType_>,
                    SparseMatrixELL<DataType_>, DenseVector<DataType_>, DataType_> & data)
            {
                CONTEXT("When evaluating MGCycleCreation (B200):");
                OperatorList cycle;
                cycle.push_back(new b200::MGCycleOperator<DataType_>(data));
                return cycle;
            }
    };

    template <> struct MGSolver<tags::GPU::CUDA, Norm<vnt_l_two, true, tags::GPU::CUDA> >
    {
        public:
            template <typename MatrixType_, typename VectorType_, typename TransferContType_, typename PreconContType_,
                     typename DataType_>
            static void value(MGData<MatrixType_, VectorType_, TransferContType_, PreconContType_, DataType_> & data,
                    OperatorList & cycle)
            {
                CONTEXT("When solving linear system with MG (B200):");
                typedef Norm<vnt_l_two, true, tags::GPU::CUDA> NormType;
                b200::MGCycleOperator<DataType_> * op(cycle.size() == 1
                        ? dynamic_cast<b200::MGCycleOperator<DataType_> *>(cycle[0]) : nullptr);
                if (op != nullptr && (const void *)op->data() == (const void *)&data)
                {
                    DataType_ r0(0), r1(0);
                    op->solve(r0, r1);
                    std::cout << "Initial norm: " << r0 << std::endl;
                    std::cout << "Final norm: " << r1 << std::endl;
                    return;
                }
                // any other cycle: the reference's loop, operator by operator
                VectorType_ r(data.x.at(data.x.size() - 1).size());
                Defect<tags::GPU::CUDA>::value(r, data.b.at(data.b.size() - 1), data.A.at(data.A.size() - 1),
                        data.x.at(data.x.size() - 1));
                DataType_ rnorm_initial = NormType::value(r);
                std::cout << "Initial norm: " << rnorm_initial << std::endl;
                DataType_ rnorm_current(1e16);
                for (unsigned long i(0) ; i < data.max_iters ; ++i)
                {
                    cycle.value();
                    Defect<tags::GPU::CUDA>::value(r, data.b.at(data.b.size() - 1), data.A.at(data.A.size() - 1),
                            data.x.at(data.x.size() - 1));
                    rnorm_current = NormType::value(r);
                    data.used_iters = i + 1;
                    if (rnorm_current < data.eps_relative * rnorm_initial)
                        break;
                }
                std::cout << "Final norm: " << rnorm_current << std::endl;
            }
    };
}

#endif
