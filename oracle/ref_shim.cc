// ref_shim.cc -- C entry points into the reference HONEI CPU path (test infrastructure only).
//
// This file is compiled together with the unmodified HONEI sources (oracle/Makefile) into
// oracle/_ref/libhonei_ref.so.  Every function builds the reference's own containers from
// plain arrays and calls the reference's own operators, so the numbers it returns ARE the
// reference's: it is the parity pin for the plain-C restatement in honei_oracle.c and the
// timed CPU baseline.  Nothing in the product links it.
//
// Tag selector (int tag):
//   0 tags::CPU                      (sequential; the parity oracle)
//   1 tags::CPU::Generic
//   2 tags::CPU::SSE                 (best single core)
//   3 tags::CPU::MultiCore::Generic
//   4 tags::CPU::MultiCore::SSE      (all cores)
//
// Reference functions called (paths within the HONEI tree):
//   Product<Tag>::value(DV, SparseMatrixELL, DV)            honei/la/product.hh:148-204
//   Defect<Tag>::value(DV, DV, SparseMatrixELL, DV)         honei/math/defect.hh:357-383
//   DotProduct<Tag>, Norm<vnt_l_two, false/true, Tag>       honei/la/dot_product.hh:72-88, honei/la/norm.hh:290-397
//   CGSolver<Tag, methods::NONE>                            honei/math/cg.hh:63-133
//   MGUtil / MGCycleCreation<V::STATIC> / MGSolver          honei/math/mg.hh:423-662, 1093-1127
//   IRSolver<Outer, Inner, Norm>                            honei/math/ir.hh:30-78
//   FillMatrix<POISSON, DIRICHLET_0> + SparseMatrix -> ELL  honei/math/fill_matrix.hh:37-77, honei/la/sparse_matrix_ell-impl.hh:75-122
//   Transposition<Tag>                                      honei/math/transposition.hh:30-50
//   SparseMatrixCSR(SparseMatrix / SparseMatrixELL)         honei/la/sparse_matrix_csr-impl.hh:73-136
//   Product<Tag>::value(DV, SparseMatrixCSR, DV)            honei/la/product.hh:209-242 (tags::CPU)
//   Defect<Tag>::value(DV, DV, SparseMatrixCSR, DV)         honei/math/defect.hh:386-419 (tags::CPU)
//   SPAI2<tags::CPU::SSE / MultiCore::SSE>::value(SM, SM)   honei/math/spai2.hh:129-296

#include <honei/la/dense_vector.hh>
#include <honei/la/sparse_matrix.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/la/sparse_matrix_csr.hh>
#include <honei/la/banded_matrix_qx.hh>
#include <honei/la/product.hh>
#include <honei/la/dot_product.hh>
#include <honei/la/norm.hh>
#include <honei/la/scaled_sum.hh>
#include <honei/la/sum.hh>
#include <honei/la/algorithm.hh>
#include <honei/math/defect.hh>
#include <honei/math/cg.hh>
#include <honei/math/ri.hh>
#include <honei/math/mg.hh>
#include <honei/math/ir.hh>
#include <honei/math/operator.hh>
#include <honei/math/restriction.hh>
#include <honei/math/prolongation.hh>
#include <honei/math/transposition.hh>
#include <honei/math/fill_matrix.hh>
#include <honei/math/spai2.hh>
#include <honei/math/matrix_io.hh>
#include <honei/math/vector_io.hh>
#include <honei/util/configuration.hh>

#include <cstdint>
#include <cstring>
#include <ctime>
#include <vector>
#include <string>
#include <exception>
#include <iostream>
#include <sstream>
#include <algorithm>

using namespace honei;

namespace
{
    double now_s()
    {
        timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        return ts.tv_sec + 1e-9 * ts.tv_nsec;
    }

    template <typename DT_> DenseVector<DT_> dv_from(const DT_ * p, unsigned long n)
    {
        DenseVector<DT_> v(n);
        if (n) std::memcpy(v.elements(), p, n * sizeof(DT_));
        return v;
    }

    template <typename DT_> void dv_to(const DenseVector<DT_> & v, DT_ * p)
    {
        if (v.size()) std::memcpy(p, v.elements(), v.size() * sizeof(DT_));
    }

    // Builds the reference container from the raw ELL arrays; the raw constructor recomputes
    // Arl from the first zero value of every row (sparse_matrix_ell-impl.hh:186-208).
    template <typename DT_> SparseMatrixELL<DT_> ell_from(unsigned long rows, unsigned long cols,
            unsigned long stride, unsigned long ncpr, unsigned long threads,
            const uint64_t * Aj, const DT_ * Ax)
    {
        const unsigned long size(ncpr * stride);
        DenseVector<unsigned long> aj(size);
        for (unsigned long i(0) ; i < size ; ++i) aj[i] = Aj[i];
        DenseVector<DT_> ax(dv_from(Ax, size));
        return SparseMatrixELL<DT_>(rows, cols, stride, ncpr, aj, ax, threads);
    }

    template <typename DT_> void ell_export(const SparseMatrixELL<DT_> & A, unsigned long * info,
            uint64_t * Aj, DT_ * Ax, uint64_t * Arl)
    {
        info[0] = A.rows(); info[1] = A.columns(); info[2] = A.stride();
        info[3] = A.num_cols_per_row(); info[4] = A.threads(); info[5] = A.used_elements();
        if (Aj)  for (unsigned long i(0) ; i < A.Aj().size() ; ++i) Aj[i] = A.Aj()[i];
        if (Ax)  dv_to(A.Ax(), Ax);
        if (Arl) for (unsigned long i(0) ; i < A.Arl().size() ; ++i) Arl[i] = A.Arl()[i];
    }

    std::string g_last_error;

    template <typename F_> int guarded(F_ f)
    {
        try { f(); return 0; }
        catch (honei::Exception & e) { g_last_error = e.message(); return 1; }
        catch (std::exception & e) { g_last_error = e.what(); return 1; }
        catch (...) { g_last_error = "unknown exception"; return 1; }
    }

#define REF_DISPATCH(tag, CALL)                                               \
    switch (tag) {                                                            \
        case 0: { typedef tags::CPU T_; CALL; } break;                        \
        case 1: { typedef tags::CPU::Generic T_; CALL; } break;               \
        case 2: { typedef tags::CPU::SSE T_; CALL; } break;                   \
        case 3: { typedef tags::CPU::MultiCore::Generic T_; CALL; } break;    \
        case 4: { typedef tags::CPU::MultiCore::SSE T_; CALL; } break;        \
        default: throw InternalError("ref_shim: unknown tag selector");       \
    }

    template <typename T_, typename DT_> void spmv_reps(SparseMatrixELL<DT_> & A, DenseVector<DT_> & y,
            const DenseVector<DT_> & x, int reps, double * seconds)
    {
        Product<T_>::value(y, A, x);                      // warm-up
        std::vector<double> t;
        for (int r(0) ; r < reps ; ++r)
        {
            double t0(now_s());
            Product<T_>::value(y, A, x);
            t.push_back(now_s() - t0);
        }
        if (seconds)
        {
            std::sort(t.begin(), t.end());
            *seconds = t.empty() ? 0. : t[t.size() / 2];
        }
    }

    template <typename DT_> int spmv_impl(int tag, unsigned long rows, unsigned long cols, unsigned long stride,
            unsigned long ncpr, unsigned long threads, const uint64_t * Aj, const DT_ * Ax,
            const DT_ * x, DT_ * y, int reps, double * seconds)
    {
        return guarded([&]() {
            SparseMatrixELL<DT_> A(ell_from(rows, cols, stride, ncpr, threads, Aj, Ax));
            DenseVector<DT_> xv(dv_from(x, cols));
            DenseVector<DT_> yv(rows, DT_(0));
            REF_DISPATCH(tag, (spmv_reps<T_, DT_>(A, yv, xv, reps, seconds)));
            dv_to(yv, y);
        });
    }

    template <typename DT_> int defect_impl(int tag, unsigned long rows, unsigned long cols, unsigned long stride,
            unsigned long ncpr, unsigned long threads, const uint64_t * Aj, const DT_ * Ax,
            const DT_ * b, const DT_ * x, DT_ * r)
    {
        return guarded([&]() {
            SparseMatrixELL<DT_> A(ell_from(rows, cols, stride, ncpr, threads, Aj, Ax));
            DenseVector<DT_> xv(dv_from(x, cols)), bv(dv_from(b, rows)), rv(rows, DT_(0));
            REF_DISPATCH(tag, (Defect<T_>::value(rv, bv, A, xv)));
            dv_to(rv, r);
        });
    }

    template <typename DT_> int cg_impl(int tag, unsigned long rows, unsigned long cols, unsigned long stride,
            unsigned long ncpr, unsigned long threads, const uint64_t * Aj, const DT_ * Ax,
            const DT_ * b, DT_ * x, unsigned long max_iters, DT_ eps, unsigned long * used, double * seconds)
    {
        return guarded([&]() {
            SparseMatrixELL<DT_> A(ell_from(rows, cols, stride, ncpr, threads, Aj, Ax));
            DenseVector<DT_> xv(dv_from(x, cols)), bv(dv_from(b, rows));
            unsigned long u(0);
            double t0(now_s());
            REF_DISPATCH(tag, (CGSolver<T_, methods::NONE>::value(A, A, bv, xv, max_iters, u, eps)));
            if (seconds) *seconds = now_s() - t0;
            *used = u;
            dv_to(xv, x);
        });
    }

    // Levels are given finest-last (level 1 = coarsest), as MGData stores them (mg.hh:35-54).
    template <typename DT_> struct MGLevels
    {
        std::vector<SparseMatrixELL<DT_> > A, prol, res;
        std::vector<DenseVector<DT_> > P, b, x, d, c, store;
        std::vector<std::vector<DenseVector<DT_> > > smoother_temp;
    };

    // Builds MGData exactly as MGUtil::load_data (mg.hh:442-547) does from files, but from
    // arrays: A_l, Prol_l from the caller; P_l = PreconFill "jac" = damping / diag(A_l)
    // (mg.hh:255-286); Res_l = Transposition(Prol_l) (mg.hh:496), or -- when the caller passes
    // them (rinfo non-null) -- the transposes it computed already (the same entries in the same
    // row order; HONEI's Transposition of a 2049^2 prolongation takes tens of seconds).
    template <typename DT_> MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_>
    mg_data_from(int nlevels, const unsigned long * ainfo, const uint64_t * const * Aj, const DT_ * const * Ax,
            const unsigned long * pinfo, const uint64_t * const * Pj, const DT_ * const * Px,
            const DT_ * b, const DT_ * x0, DT_ damping, const unsigned long * rinfo = nullptr,
            const uint64_t * const * Rj = nullptr, const DT_ * const * Rx = nullptr)
    {
        MGLevels<DT_> L;
        for (int i(0) ; i < nlevels ; ++i)
        {
            const unsigned long * ai(ainfo + 5 * i);
            SparseMatrixELL<DT_> a(ell_from(ai[0], ai[1], ai[2], ai[3], ai[4], Aj[i], Ax[i]));
            L.A.push_back(a);
            PreconFill<DenseVector<DT_>, SparseMatrixELL<DT_>, DT_>::value(i, L.P, "", "jac", a, damping);
            if (i < nlevels - 1)
            {
                const unsigned long * pi(pinfo + 5 * i);
                SparseMatrixELL<DT_> p(ell_from(pi[0], pi[1], pi[2], pi[3], pi[4], Pj[i], Px[i]));
                L.prol.push_back(p);
                if (rinfo)
                {
                    const unsigned long * ri(rinfo + 5 * i);
                    L.res.push_back(ell_from(ri[0], ri[1], ri[2], ri[3], ri[4], Rj[i], Rx[i]));
                }
                else
                    L.res.push_back(Transposition<tags::CPU>::value(p.copy()));
            }
            const unsigned long n(ai[0]);
            DenseVector<DT_> zero(n, DT_(0));
            if (i == nlevels - 1)
            {
                L.b.push_back(dv_from(b, n));
                L.x.push_back(dv_from(x0, n));
            }
            else
            {
                L.b.push_back(zero.copy());
                L.x.push_back(zero.copy());
            }
            L.d.push_back(zero.copy());
            L.c.push_back(zero.copy());
            L.store.push_back(zero.copy());
            L.smoother_temp.push_back(std::vector<DenseVector<DT_> >());
        }
        return MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_>(
                L.A, L.res, L.prol, L.P, L.b, L.x, L.d, L.c, L.store, L.smoother_temp, 0, 0, 0, 0, 0, DT_(0));
    }

    template <typename T_, typename DT_> void mg_run(
            MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>, DenseVector<DT_>, DT_> & data)
    {
        OperatorList cycle(MGCycleCreation<T_, methods::CYCLE::V::STATIC, CGSolver<T_, methods::NONE>, RISmoother<T_>,
                Restriction<T_, methods::PROLMAT>, Prolongation<T_, methods::PROLMAT>, DT_>::value(data));
        MGSolver<T_, Norm<vnt_l_two, true, T_> >::value(data, cycle);
    }

    // IRSolver<T_, T_> (honei/math/ir.hh:30-78): FP64 outer loop around the FP32 V-cycle of data.
    template <typename T_> void ir_mg_run(SparseMatrixELL<double> & A, DenseVector<double> & b,
            DenseVector<double> & x,
            MGData<SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>, float> & data,
            double eps, unsigned long max_iters, unsigned long & used)
    {
        OperatorList cycle(MGCycleCreation<T_, methods::CYCLE::V::STATIC, CGSolver<T_, methods::NONE>, RISmoother<T_>,
                Restriction<T_, methods::PROLMAT>, Prolongation<T_, methods::PROLMAT>, float>::value(data));
        IRSolver<T_, T_, Norm<vnt_l_two, true, T_> >::value(A, b, x, data, cycle, eps, max_iters, used);
    }

    // MGSolver prints its initial and final norm to stdout (mg.hh:1107,1125); keep the
    // caller's stdout clean.
    struct MuteCout
    {
        std::streambuf * old;
        std::ostringstream sink;
        MuteCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
        ~MuteCout() { std::cout.rdbuf(old); }
    };

    // Product on BandedMatrixQx<Q1Type> for tags::CPU (product.hh:333-366), tags::CPU::SSE
    // (product-sse.cc:217-253) and tags::CPU::MultiCore::SSE (product.hh:1970-2020; the
    // MultiCore::Generic instantiation does not compile in the reference).  reps > 0 times that many products (median into *seconds).
    template <typename T_, typename DT_> void q1band_product(const BandedMatrixQx<Q1Type, DT_> & A,
            const DenseVector<DT_> & x, DT_ * y, int reps, double * seconds)
    {
        DenseVector<DT_> r(Product<T_>::value(A, x));
        std::vector<double> t;
        for (int k(0) ; k < reps ; ++k)
        {
            double t0(now_s());
            DenseVector<DT_> rr(Product<T_>::value(A, x));
            t.push_back(now_s() - t0);
        }
        if (seconds)
        {
            std::sort(t.begin(), t.end());
            *seconds = t.empty() ? 0. : t[t.size() / 2];
        }
        dv_to(r, y);
    }

    template <typename DT_> BandedMatrixQx<Q1Type, DT_> q1band_from(unsigned long n, const DT_ * const * band)
    {
        std::vector<DenseVector<DT_> > b;
        for (int k(0) ; k < 9 ; ++k)
        {
            DenseVector<DT_> v(n);
            for (unsigned long i(0) ; i < n ; ++i) v[i] = band[k][i];
            b.push_back(v);
        }
        return BandedMatrixQx<Q1Type, DT_>(n, b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8]);
    }

    template <typename DT_> int q1band_spmv_impl(int tag, unsigned long n, const DT_ * const * band, const DT_ * x,
            DT_ * y, int reps, double * seconds)
    {
        return guarded([&]() {
            BandedMatrixQx<Q1Type, DT_> A(q1band_from<DT_>(n, band));
            DenseVector<DT_> xv(n);
            for (unsigned long i(0) ; i < n ; ++i) xv[i] = x[i];
            switch (tag)
            {
                case 0: q1band_product<tags::CPU>(A, xv, y, reps, seconds); break;
                case 2: q1band_product<tags::CPU::SSE>(A, xv, y, reps, seconds); break;
                case 4: q1band_product<tags::CPU::MultiCore::SSE>(A, xv, y, reps, seconds); break;
                default: throw InternalError("ref_shim: no banded Q1 product for this tag");
            }
        });
    }
    // CGSolver<T_, methods::VAR>::value(A, P, b, x, max_iters, used, eps) (cg.hh:140-219) with a
    // vector P (Pd != NULL) or an ELL matrix P (pinfo/Pj/Px).
    template <typename DT_> int cg_var_impl(int tag, const unsigned long * ainfo, const uint64_t * Aj, const DT_ * Ax,
            const DT_ * Pd, const unsigned long * pinfo, const uint64_t * Pj, const DT_ * Px, const DT_ * b, DT_ * x,
            unsigned long max_iters, DT_ eps, unsigned long * used, double * seconds)
    {
        return guarded([&]() {
            SparseMatrixELL<DT_> A(ell_from(ainfo[0], ainfo[1], ainfo[2], ainfo[3], ainfo[4], Aj, Ax));
            DenseVector<DT_> bv(A.rows()), xv(A.rows());
            for (unsigned long i(0) ; i < A.rows() ; ++i) { bv[i] = b[i]; xv[i] = x[i]; }
            unsigned long u(0);
            double t0(now_s());
            if (Pd)
            {
                DenseVector<DT_> P(A.rows());
                for (unsigned long i(0) ; i < A.rows() ; ++i) P[i] = Pd[i];
                switch (tag)
                {
                    case 0: CGSolver<tags::CPU, methods::VAR>::value(A, P, bv, xv, max_iters, u, eps); break;
                    case 4: CGSolver<tags::CPU::MultiCore::SSE, methods::VAR>::value(A, P, bv, xv, max_iters, u, eps); break;
                    default: throw InternalError("ref_shim: CGSolver<VAR> tag not available");
                }
            }
            else
            {
                SparseMatrixELL<DT_> P(ell_from(pinfo[0], pinfo[1], pinfo[2], pinfo[3], pinfo[4], Pj, Px));
                switch (tag)
                {
                    case 0: CGSolver<tags::CPU, methods::VAR>::value(A, P, bv, xv, max_iters, u, eps); break;
                    case 4: CGSolver<tags::CPU::MultiCore::SSE, methods::VAR>::value(A, P, bv, xv, max_iters, u, eps); break;
                    default: throw InternalError("ref_shim: CGSolver<VAR> tag not available");
                }
            }
            if (seconds) *seconds = now_s() - t0;
            *used = u;
            dv_to(xv, x);
        });
    }


    // SparseMatrixCSR from plain arrays (the raw-array constructor, sparse_matrix_csr.hh)
    template <typename DT_> SparseMatrixCSR<DT_> csr_from(unsigned long rows, unsigned long cols,
            unsigned long blocksize, unsigned long used, const uint64_t * Ar, const uint64_t * Aj, const DT_ * Ax)
    {
        const unsigned long nblocks(Ar[rows]);
        DenseVector<unsigned long> ar(rows + 1), aj(nblocks ? nblocks : 1);
        for (unsigned long i(0) ; i <= rows ; ++i) ar[i] = Ar[i];
        for (unsigned long i(0) ; i < nblocks ; ++i) aj[i] = Aj[i];
        DenseVector<DT_> ax(dv_from(Ax, nblocks ? nblocks * blocksize : 1));
        return SparseMatrixCSR<DT_>(blocksize, rows, cols, aj, ax, ar, used);
    }

    // info = {rows, cols, blocksize, nblocks, used_elements}; arrays copied when non-null
    template <typename DT_> void csr_to(const SparseMatrixCSR<DT_> & A, unsigned long * info, uint64_t * Ar,
            uint64_t * Aj, DT_ * Ax)
    {
        const unsigned long nb(A.Ar()[A.rows()]);
        info[0] = A.rows(); info[1] = A.columns(); info[2] = A.blocksize(); info[3] = nb; info[4] = A.used_elements();
        if (Ar) for (unsigned long i(0) ; i <= A.rows() ; ++i) Ar[i] = A.Ar()[i];
        if (Aj) for (unsigned long i(0) ; i < nb ; ++i) Aj[i] = A.Aj()[i];
        if (Ax) for (unsigned long i(0) ; i < nb * A.blocksize() ; ++i) Ax[i] = A.Ax()[i];
    }

    struct BlocksizeScope
    {
        unsigned long old;
        explicit BlocksizeScope(unsigned long bs) : old(Configuration::instance()->get_value("csr::blocksize", 1))
        { Configuration::instance()->set_value("csr::blocksize", bs); }
        ~BlocksizeScope() { Configuration::instance()->set_value("csr::blocksize", old); }
    };

    template <typename T_, typename DT_> void csr_spmv_reps(SparseMatrixCSR<DT_> & A, DenseVector<DT_> & y,
            const DenseVector<DT_> & x, int reps, double * seconds)
    {
        Product<T_>::value(y, A, x);                      // warm-up
        std::vector<double> t;
        for (int r(0) ; r < reps ; ++r)
        {
            double t0(now_s());
            Product<T_>::value(y, A, x);
            t.push_back(now_s() - t0);
        }
        if (seconds)
        {
            std::sort(t.begin(), t.end());
            *seconds = t.empty() ? 0. : t[t.size() / 2];
        }
    }

    // SPAI2 on the SparseMatrix made of the ELL matrix (sparse_matrix.hh:157-185), M starting as
    // a copy of it (the test's and spai2-cuda.cc's M = A.copy()); Mx returns M's value at every
    // ELL slot of A that holds an entry (0 elsewhere).  tag 2: SSE, 4: MultiCore::SSE.
    template <typename DT_> int spai2_impl(int tag, const unsigned long * ainfo, const uint64_t * Aj,
            const DT_ * Ax, DT_ * Mx, double * seconds)
    {
        return guarded([&]() {
            SparseMatrixELL<DT_> A(ell_from(ainfo[0], ainfo[1], ainfo[2], ainfo[3], ainfo[4], Aj, Ax));
            SparseMatrix<DT_> sm(A);
            SparseMatrix<DT_> m(sm.copy());
            double t0(now_s());
            switch (tag)
            {
                case 2: SPAI2<tags::CPU::SSE>::value(m, sm); break;
                case 4: SPAI2<tags::CPU::MultiCore::SSE>::value(m, sm); break;
                default: throw InternalError("ref_shim: SPAI2 tag not available");
            }
            if (seconds) *seconds = now_s() - t0;
            const SparseMatrix<DT_> & cm(m);
            const unsigned long size(ainfo[2] * ainfo[3]), T(ainfo[4]), stride(ainfo[2]);
            for (unsigned long i(0) ; i < size ; ++i)
            {
                const unsigned long row((i % stride) / T);
                Mx[i] = Ax[i] != DT_(0) ? cm[row][Aj[i]] : DT_(0);
            }
        });
    }
}

extern "C"
{
    const char * ref_last_error() { return g_last_error.c_str(); }

    int ref_cg_var_f64(int tag, const unsigned long * ainfo, const uint64_t * Aj, const double * Ax, const double * Pd,
            const unsigned long * pinfo, const uint64_t * Pj, const double * Px, const double * b, double * x,
            unsigned long max_iters, double eps, unsigned long * used, double * seconds)
    { return cg_var_impl<double>(tag, ainfo, Aj, Ax, Pd, pinfo, Pj, Px, b, x, max_iters, eps, used, seconds); }

    int ref_cg_var_f32(int tag, const unsigned long * ainfo, const uint64_t * Aj, const float * Ax, const float * Pd,
            const unsigned long * pinfo, const uint64_t * Pj, const float * Px, const float * b, float * x,
            unsigned long max_iters, float eps, unsigned long * used, double * seconds)
    { return cg_var_impl<float>(tag, ainfo, Aj, Ax, Pd, pinfo, Pj, Px, b, x, max_iters, eps, used, seconds); }

    int ref_spai2_f64(int tag, const unsigned long * ainfo, const uint64_t * Aj, const double * Ax, double * Mx,
            double * seconds)
    { return spai2_impl<double>(tag, ainfo, Aj, Ax, Mx, seconds); }

    int ref_spai2_f32(int tag, const unsigned long * ainfo, const uint64_t * Aj, const float * Ax, float * Mx,
            double * seconds)
    { return spai2_impl<float>(tag, ainfo, Aj, Ax, Mx, seconds); }

    int ref_q1band_spmv_f64(int tag, unsigned long n, const double * const * band, const double * x, double * y,
            int reps, double * seconds)
    { return q1band_spmv_impl<double>(tag, n, band, x, y, reps, seconds); }

    int ref_q1band_spmv_f32(int tag, unsigned long n, const float * const * band, const float * x, float * y,
            int reps, double * seconds)
    { return q1band_spmv_impl<float>(tag, n, band, x, y, reps, seconds); }

    // Defect<tags::CPU> on BandedMatrixQx (defect.hh:194-199).
    int ref_q1band_defect_f64(unsigned long n, const double * const * band, const double * b, const double * x,
            double * r)
    {
        return guarded([&]() {
            BandedMatrixQx<Q1Type, double> A(q1band_from<double>(n, band));
            DenseVector<double> bv(n), xv(n), rv(n);
            for (unsigned long i(0) ; i < n ; ++i) { bv[i] = b[i]; xv[i] = x[i]; }
            Defect<tags::CPU>::value(rv, bv, A, xv);
            dv_to(rv, r);
        });
    }

    // FillMatrix<POISSON, DIRICHLET_0> on BandedMatrixQx (fill_matrix.hh:41-77), bands out.
    int ref_q1band_poisson_f64(unsigned long M, double * const * band)
    {
        return guarded([&]() {
            const unsigned long N(M * M);
            DenseVector<double> z(N, 0.);
            BandedMatrixQx<Q1Type, double> q1(N, z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(),
                    z.copy(), z.copy(), z.copy());
            FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(q1);
            const Q1BandIndex idx[9] = { LL, LD, LU, DL, DD, DU, UL, UD, UU };
            for (int k(0) ; k < 9 ; ++k) dv_to(q1.band(idx[k]), band[k]);
        });
    }

    // BandedMatrixQx(SparseMatrixELL&) conversion (banded_matrix_qx-impl.hh:111-167): n must be
    // (2^L + 1)^2.  ELL arrays in, bands out.
    int ref_q1band_from_ell_f64(const unsigned long * ainfo, const uint64_t * Aj, const double * Ax, double * const * band)
    {
        return guarded([&]() {
            SparseMatrixELL<double> A(ell_from(ainfo[0], ainfo[1], ainfo[2], ainfo[3], ainfo[4], Aj, Ax));
            BandedMatrixQx<Q1Type, double> q1(A);
            const Q1BandIndex idx[9] = { LL, LD, LU, DL, DD, DU, UL, UD, UU };
            for (int k(0) ; k < 9 ; ++k) dv_to(q1.band(idx[k]), band[k]);
        });
    }

    // Threads used by the MultiCore tags: mc::num_threads and every max_count key on the path.
    int ref_set_threads(int n)
    {
        return guarded([&]() {
            Configuration * c(Configuration::instance());
            c->set_value("mc::num_threads", n);
            const char * keys[] = { "mc::Product(DV,SMELL,DV)::max_count", "mc::dot_product(DVCB,DVCB)::max_count",
                "mc::ScaledSum(DVB,DVB,DT)::max_count", "mc::ScaledSum(DVCB,DVCB,DT)::max_count",
                "mc::Sum(DVCB,DVCB)::max_count", "mc::Scale(DVCB,DT)::max_count",
                "mc::Difference(DVCB,DVCB)::max_count", "mc::ElementProduct(DVCB,DVCB)::max_count",
                "mc::Defect(DV,DV,SMELL,DV)::max_count" };
            for (const char * k : keys) c->set_value(k, n);
        });
    }

    // Q1 Poisson (Dirichlet rows = identity) on an M x M node grid through the reference's own
    // construction path: FillMatrix -> BandedMatrixQx -> SparseMatrix -> SparseMatrixELL.
    // Call with Aj == NULL to receive info = {rows, cols, stride, ncpr, threads, nnz} only.
    int ref_q1_poisson_f64(unsigned long M, unsigned long * info, uint64_t * Aj, double * Ax, uint64_t * Arl)
    {
        return guarded([&]() {
            const unsigned long N(M * M);
            DenseVector<double> z(N, 0.);
            BandedMatrixQx<Q1Type, double> q1(N, z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(),
                    z.copy(), z.copy(), z.copy());
            FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(q1);
            SparseMatrix<double> sm(q1);
            SparseMatrixELL<double> A(sm);
            ell_export(A, info, Aj, Ax, Arl);
        });
    }

    // Reads a HONEI .ell file with the reference reader (matrix_io.hh:433-582).
    int ref_read_ell_f64(const char * path, unsigned long * info, uint64_t * Aj, double * Ax, uint64_t * Arl)
    {
        return guarded([&]() {
            SparseMatrixELL<double> A(MatrixIO<io_formats::ELL>::read_matrix(std::string(path), double(0)));
            ell_export(A, info, Aj, Ax, Arl);
        });
    }

    // Prolongation / Restriction<tags::CPU, methods::NONE> (prolongation.hh:42-139,
    // restriction.hh:41-170) on plain arrays; the unused matrix argument is a dummy.
    int ref_prolongate_f64(unsigned long n_fine, double * fine, const double * coarse, unsigned long n_coarse,
            const uint64_t * mask)
    {
        return guarded([&]() {
            DenseVector<double> f(n_fine, 0.), c(n_coarse);
            DenseVector<unsigned long> m(8);
            for (unsigned long i(0) ; i < n_coarse ; ++i) c[i] = coarse[i];
            for (int i(0) ; i < 8 ; ++i) m[i] = mask[i];
            int unused(0);
            Prolongation<tags::CPU, methods::NONE>::value(f, c, m, unused);
            dv_to(f, fine);
        });
    }

    int ref_restrict_f64(unsigned long n_fine, double * coarse, const double * fine, unsigned long n_coarse,
            const uint64_t * mask)
    {
        return guarded([&]() {
            DenseVector<double> f(n_fine), c(n_coarse, 0.);
            DenseVector<unsigned long> m(8);
            for (unsigned long i(0) ; i < n_fine ; ++i) f[i] = fine[i];
            for (int i(0) ; i < 8 ; ++i) m[i] = mask[i];
            int unused(0);
            Restriction<tags::CPU, methods::NONE>::value(c, f, m, unused);
            dv_to(c, coarse);
        });
    }

    int ref_prolongate_f32(unsigned long n_fine, float * fine, const float * coarse, unsigned long n_coarse,
            const uint64_t * mask)
    {
        return guarded([&]() {
            DenseVector<float> f(n_fine, 0.f), c(n_coarse);
            DenseVector<unsigned long> m(8);
            for (unsigned long i(0) ; i < n_coarse ; ++i) c[i] = coarse[i];
            for (int i(0) ; i < 8 ; ++i) m[i] = mask[i];
            int unused(0);
            Prolongation<tags::CPU, methods::NONE>::value(f, c, m, unused);
            dv_to(f, fine);
        });
    }

    int ref_restrict_f32(unsigned long n_fine, float * coarse, const float * fine, unsigned long n_coarse,
            const uint64_t * mask)
    {
        return guarded([&]() {
            DenseVector<float> f(n_fine), c(n_coarse, 0.f);
            DenseVector<unsigned long> m(8);
            for (unsigned long i(0) ; i < n_fine ; ++i) f[i] = fine[i];
            for (int i(0) ; i < 8 ; ++i) m[i] = mask[i];
            int unused(0);
            Restriction<tags::CPU, methods::NONE>::value(c, f, m, unused);
            dv_to(c, coarse);
        });
    }

    // MatrixMarket file -> SparseMatrix -> SparseMatrixELL through the reference (mtxtoell.cc).
    int ref_read_mtx_f64(const char * path, unsigned long * info, uint64_t * Aj, double * Ax, uint64_t * Arl)
    {
        return guarded([&]() {
            SparseMatrix<double> sm(MatrixIO<io_formats::MTX>::read_matrix(std::string(path), double(0)));
            SparseMatrixELL<double> A(sm);
            ell_export(A, info, Aj, Ax, Arl);
        });
    }

    // Reads an EXP vector with the reference reader (vector_io.hh:52-115). n receives the size.
    int ref_read_exp_f64(const char * path, unsigned long * n, double * out)
    {
        return guarded([&]() {
            DenseVector<double> v(VectorIO<io_formats::EXP>::read_vector(std::string(path), double(0)));
            *n = v.size();
            if (out) dv_to(v, out);
        });
    }

    // Transposition of an ELL matrix (the MG restriction matrix), raw arrays in, ELL arrays out.
    int ref_transpose_f64(const unsigned long * ainfo, const uint64_t * Aj, const double * Ax,
            unsigned long * info, uint64_t * Tj, double * Tx, uint64_t * Trl)
    {
        return guarded([&]() {
            SparseMatrixELL<double> A(ell_from(ainfo[0], ainfo[1], ainfo[2], ainfo[3], ainfo[4], Aj, Ax));
            SparseMatrixELL<double> T(Transposition<tags::CPU>::value(A));
            ell_export(T, info, Tj, Tx, Trl);
        });
    }

    int ref_spmv_f64(int tag, unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const double * Ax, const double * x, double * y,
            int reps, double * seconds)
    { return spmv_impl<double>(tag, rows, cols, stride, ncpr, threads, Aj, Ax, x, y, reps, seconds); }

    int ref_spmv_f32(int tag, unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const float * Ax, const float * x, float * y,
            int reps, double * seconds)
    { return spmv_impl<float>(tag, rows, cols, stride, ncpr, threads, Aj, Ax, x, y, reps, seconds); }

    // A reference SparseMatrixELL<double> built once and kept (the product benchmark's set-up,
    // honei/benchmark/product_ell_file_BENCHMARK.cc:57-92), then Product<tag> on it `reps`
    // times: the wall time of every product into seconds[0..reps).
    struct RefEll
    {
        SparseMatrixELL<double> A;
        DenseVector<double> x, y;
        RefEll(SparseMatrixELL<double> a, DenseVector<double> xv) : A(a), x(xv), y(a.rows(), 0.) {}
    };

    int ref_ell_create_f64(unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const double * Ax, const double * x, void ** out)
    {
        return guarded([&]() {
            *out = new RefEll(ell_from<double>(rows, cols, stride, ncpr, threads, Aj, Ax), dv_from(x, cols));
        });
    }

    int ref_ell_spmv_f64(int tag, void * h, int reps, double * seconds, double * y)
    {
        return guarded([&]() {
            RefEll & e(*static_cast<RefEll *>(h));
            for (int r(0) ; r < reps ; ++r)
            {
                double t0(now_s());
                REF_DISPATCH(tag, (Product<T_>::value(e.y, e.A, e.x)));
                if (seconds) seconds[r] = now_s() - t0;
            }
            if (y) dv_to(e.y, y);
        });
    }

    int ref_ell_destroy(void * h)
    {
        return guarded([&]() { delete static_cast<RefEll *>(h); });
    }

    int ref_defect_f64(int tag, unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const double * Ax, const double * b, const double * x, double * r)
    { return defect_impl<double>(tag, rows, cols, stride, ncpr, threads, Aj, Ax, b, x, r); }

    int ref_defect_f32(int tag, unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const float * Ax, const float * b, const float * x, float * r)
    { return defect_impl<float>(tag, rows, cols, stride, ncpr, threads, Aj, Ax, b, x, r); }

    int ref_dot_f64(int tag, unsigned long n, const double * x, const double * y, double * out)
    {
        return guarded([&]() {
            DenseVector<double> xv(dv_from(x, n)), yv(dv_from(y, n));
            REF_DISPATCH(tag, (*out = DotProduct<T_>::value(xv, yv)));
        });
    }

    int ref_dot_f32(int tag, unsigned long n, const float * x, const float * y, float * out)
    {
        return guarded([&]() {
            DenseVector<float> xv(dv_from(x, n)), yv(dv_from(y, n));
            REF_DISPATCH(tag, (*out = DotProduct<T_>::value(xv, yv)));
        });
    }

    int ref_norm2sq_f64(int tag, unsigned long n, const double * x, double * out)
    {
        return guarded([&]() {
            DenseVector<double> xv(dv_from(x, n));
            REF_DISPATCH(tag, (*out = Norm<vnt_l_two, false, T_>::value(xv)));
        });
    }

    int ref_cg_f64(int tag, unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const double * Ax, const double * b, double * x,
            unsigned long max_iters, double eps, unsigned long * used, double * seconds)
    { return cg_impl<double>(tag, rows, cols, stride, ncpr, threads, Aj, Ax, b, x, max_iters, eps, used, seconds); }

    int ref_cg_f32(int tag, unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj, const float * Ax, const float * b, float * x,
            unsigned long max_iters, float eps, unsigned long * used, double * seconds)
    { return cg_impl<float>(tag, rows, cols, stride, ncpr, threads, Aj, Ax, b, x, max_iters, eps, used, seconds); }

    // V(n_pre, n_post) MG with damped Jacobi ("jac") smoothing, PROLMAT transfers and a CG
    // coarse solver at level 1.  ainfo/pinfo hold {rows, cols, stride, ncpr, threads} per level,
    // coarsest first; x holds x0 on entry and the solution on exit.
    int ref_mg_f64(int tag, int nlevels, const unsigned long * ainfo, const uint64_t * const * Aj,
            const double * const * Ax, const unsigned long * pinfo, const uint64_t * const * Pj,
            const double * const * Px, const double * b, double * x, double damping,
            unsigned long max_iters, unsigned long max_iters_coarse, unsigned long n_pre, unsigned long n_post,
            double eps, unsigned long * used, double * seconds, const unsigned long * rinfo,
            const uint64_t * const * Rj, const double * const * Rx)
    {
        return guarded([&]() {
            MuteCout mute;
            MGData<SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>, double>
                data(mg_data_from<double>(nlevels, ainfo, Aj, Ax, pinfo, Pj, Px, b, x, damping, rinfo, Rj, Rx));
            MGUtil<tags::CPU, SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>,
                MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, double>::configure(
                        data, max_iters, max_iters_coarse, n_pre, n_post, 1, eps);
            double t0(now_s());
            REF_DISPATCH(tag, (mg_run<T_, double>(data)));
            if (seconds) *seconds = now_s() - t0;
            *used = data.used_iters;
            dv_to(data.x.back(), x);
        });
    }

    int ref_mg_f32(int tag, int nlevels, const unsigned long * ainfo, const uint64_t * const * Aj,
            const float * const * Ax, const unsigned long * pinfo, const uint64_t * const * Pj,
            const float * const * Px, const float * b, float * x, float damping,
            unsigned long max_iters, unsigned long max_iters_coarse, unsigned long n_pre, unsigned long n_post,
            float eps, unsigned long * used, double * seconds, const unsigned long * rinfo,
            const uint64_t * const * Rj, const float * const * Rx)
    {
        return guarded([&]() {
            MuteCout mute;
            MGData<SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>, float>
                data(mg_data_from<float>(nlevels, ainfo, Aj, Ax, pinfo, Pj, Px, b, x, damping, rinfo, Rj, Rx));
            MGUtil<tags::CPU, SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>,
                MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, float>::configure(
                        data, max_iters, max_iters_coarse, n_pre, n_post, 1, eps);
            double t0(now_s());
            REF_DISPATCH(tag, (mg_run<T_, float>(data)));
            if (seconds) *seconds = now_s() - t0;
            *used = data.used_iters;
            dv_to(data.x.back(), x);
        });
    }

    // IRSolver<tags::CPU, tags::CPU, Norm<l2, true>> (ir.hh:30-78): FP64 outer defect/update
    // around the FP32 MG above.  The inner data keeps its x between outer steps, as ir.hh does.
    int ref_ir_mg(int tag, int nlevels, const unsigned long * ainfo, const uint64_t * const * Aj,
            const double * const * Ax64, const float * const * Ax32, const unsigned long * pinfo,
            const uint64_t * const * Pj, const float * const * Px32, const double * b, double * x,
            float damping, unsigned long inner_max_iters, unsigned long max_iters_coarse,
            unsigned long n_pre, unsigned long n_post, float inner_eps, double eps,
            unsigned long max_iters, unsigned long * used, double * seconds, const unsigned long * rinfo,
            const uint64_t * const * Rj, const float * const * Rx32)
    {
        return guarded([&]() {
            MuteCout mute;
            const unsigned long n(ainfo[5 * (nlevels - 1)]);
            std::vector<float> zero(n, 0.f);
            MGData<SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>, float>
                data(mg_data_from<float>(nlevels, ainfo, Aj, Ax32, pinfo, Pj, Px32, zero.data(), zero.data(), damping,
                        rinfo, Rj, Rx32));
            MGUtil<tags::CPU, SparseMatrixELL<float>, DenseVector<float>, SparseMatrixELL<float>, DenseVector<float>,
                MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, float>::configure(
                        data, inner_max_iters, max_iters_coarse, n_pre, n_post, 1, inner_eps);
            const unsigned long * ai(ainfo + 5 * (nlevels - 1));
            SparseMatrixELL<double> A(ell_from(ai[0], ai[1], ai[2], ai[3], ai[4], Aj[nlevels - 1], Ax64[nlevels - 1]));
            DenseVector<double> bv(dv_from(b, n)), xv(dv_from(x, n));
            unsigned long u(0);
            double t0(now_s());
            REF_DISPATCH(tag, (ir_mg_run<T_>(A, bv, xv, data, eps, max_iters, u)));
            if (seconds) *seconds = now_s() - t0;
            *used = u;
            dv_to(xv, x);
        });
    }

    // The reference's CSR product test matrix (honei/la/product_TEST.cc:936-948) converted with
    // csr::blocksize = blocksize: info, arrays (two-phase: call with null arrays for info), x and
    // y = Product<tags::CPU>(A, x).
    int ref_csr_product_test_f64(unsigned long size, unsigned long blocksize, unsigned long * info,
            uint64_t * Ar, uint64_t * Aj, double * Ax, double * x, double * y)
    {
        return guarded([&]() {
            BlocksizeScope scope(blocksize);
            SparseMatrix<double> sms(size, size + 3);
            for (SparseMatrix<double>::ElementIterator i(sms.begin_elements()) ; i < sms.end_elements() ; ++i)
            {
                if (i.index() % 5 == 0)
                    *i = double(i.index()) / 1.234;
            }
            SparseMatrixCSR<double> A(sms);
            csr_to(A, info, Ar, Aj, Ax);
            if (x && y)
            {
                DenseVector<double> dv1(size + 3, double(4));
                dv1[0] = 1;
                dv1[1] = 2;
                DenseVector<double> prod(size, double(4711));
                Product<tags::CPU>::value(prod, A, dv1);
                dv_to(dv1, x);
                dv_to(prod, y);
            }
        });
    }

    // SparseMatrixCSR(SparseMatrixELL) with csr::blocksize = blocksize (two-phase like above).
    int ref_csr_from_ell_f64(unsigned long rows, unsigned long cols, unsigned long stride, unsigned long ncpr,
            unsigned long threads, const uint64_t * Aj_ell, const double * Ax_ell, unsigned long blocksize,
            unsigned long * info, uint64_t * Ar, uint64_t * Aj, double * Ax)
    {
        return guarded([&]() {
            BlocksizeScope scope(blocksize);
            SparseMatrixELL<double> E(ell_from(rows, cols, stride, ncpr, threads, Aj_ell, Ax_ell));
            SparseMatrixCSR<double> A(E);
            csr_to(A, info, Ar, Aj, Ax);
        });
    }

    int ref_csr_spmv_f64(int tag, unsigned long rows, unsigned long cols, unsigned long blocksize, unsigned long used,
            const uint64_t * Ar, const uint64_t * Aj, const double * Ax, const double * x, double * y,
            int reps, double * seconds)
    {
        return guarded([&]() {
            SparseMatrixCSR<double> A(csr_from(rows, cols, blocksize, used, Ar, Aj, Ax));
            DenseVector<double> xv(dv_from(x, cols)), yv(rows, 0.);
            REF_DISPATCH(tag, (csr_spmv_reps<T_, double>(A, yv, xv, reps, seconds)));
            dv_to(yv, y);
        });
    }

    int ref_csr_spmv_f32(int tag, unsigned long rows, unsigned long cols, unsigned long blocksize, unsigned long used,
            const uint64_t * Ar, const uint64_t * Aj, const float * Ax, const float * x, float * y,
            int reps, double * seconds)
    {
        return guarded([&]() {
            SparseMatrixCSR<float> A(csr_from(rows, cols, blocksize, used, Ar, Aj, Ax));
            DenseVector<float> xv(dv_from(x, cols)), yv(rows, 0.f);
            REF_DISPATCH(tag, (csr_spmv_reps<T_, float>(A, yv, xv, reps, seconds)));
            dv_to(yv, y);
        });
    }

    int ref_csr_defect_f64(int tag, unsigned long rows, unsigned long cols, unsigned long blocksize, unsigned long used,
            const uint64_t * Ar, const uint64_t * Aj, const double * Ax, const double * b, const double * x, double * r)
    {
        return guarded([&]() {
            SparseMatrixCSR<double> A(csr_from(rows, cols, blocksize, used, Ar, Aj, Ax));
            DenseVector<double> xv(dv_from(x, cols)), bv(dv_from(b, rows)), rv(rows, 0.);
            REF_DISPATCH(tag, (Defect<T_>::value(rv, bv, A, xv)));
            dv_to(rv, r);
        });
    }

    int ref_csr_defect_f32(int tag, unsigned long rows, unsigned long cols, unsigned long blocksize, unsigned long used,
            const uint64_t * Ar, const uint64_t * Aj, const float * Ax, const float * b, const float * x, float * r)
    {
        return guarded([&]() {
            SparseMatrixCSR<float> A(csr_from(rows, cols, blocksize, used, Ar, Aj, Ax));
            DenseVector<float> xv(dv_from(x, cols)), bv(dv_from(b, rows)), rv(rows, 0.f);
            REF_DISPATCH(tag, (Defect<T_>::value(rv, bv, A, xv)));
            dv_to(rv, r);
        });
    }
}
