// HONEI's own operators and generic solver templates on tags::GPU::CUDA, provided by the B200
// plugin (honei_b200/plugin), checked against tags::CPU on the same inputs.
//   plugin_ops_test [mg_dir]
// mg_dir holds A_1..A_L.ell, prol_2..prol_L.ell, rhs_L, init_L (HONEI file formats); it is
// loaded with MGUtil::load_data exactly as honei/math/mg_TEST.cc loads FEATFLOW data.
// This translation unit does NOT include solvers_b200.hh: CGSolver<tags::GPU::CUDA, NONE> here
// is HONEI's generic template (honei/math/cg.hh:63-133) running on the plugin's operators.
#include "plugin_common.hh"
#include "honei_b200/plugin/b200_backend.hh"

#include <honei/la/difference.hh>
#include <honei/la/dot_product.hh>
#include <honei/la/element_product.hh>
#include <honei/la/norm.hh>
#include <honei/la/product.hh>
#include <honei/la/scale.hh>
#include <honei/la/scaled_sum.hh>
#include <honei/la/sparse_matrix_csr.hh>
#include <honei/la/sum.hh>
#include <honei/util/configuration.hh>
#include <honei/math/cg.hh>
#include <honei/math/defect.hh>
#include <honei/math/matrix_io.hh>
#include <honei/math/mg.hh>
#include <honei/math/operator.hh>
#include <honei/math/prolongation.hh>
#include <honei/math/restriction.hh>
#include <honei/math/ri.hh>
#include <honei/math/spai2.hh>
#include <honei/math/vector_io.hh>

#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>

using namespace honei;
using namespace plugin_test;

template <typename DT_> bool equal(const DenseVector<DT_> & a, const DenseVector<DT_> & b)
{
    a.lock(lm_read_only);
    b.lock(lm_read_only);
    bool ok(a.size() == b.size());
    for (unsigned long i(0) ; ok && i < a.size() ; ++i)
        ok = (a[i] == b[i]);
    a.unlock(lm_read_only);
    b.unlock(lm_read_only);
    return ok;
}

template <typename DT_> void operators(unsigned long M, const std::string & tag)
{
    SparseMatrixELL<DT_> A(q1<DT_>(M));
    const unsigned long n(A.rows());
    DenseVector<DT_> x(seeded<DT_>(n, 1)), y(seeded<DT_>(n, 2)), b(seeded<DT_>(n, 3));

    DenseVector<DT_> ycpu(n), ygpu(n);
    Product<tags::CPU>::value(ycpu, A, x);
    Product<tags::GPU::CUDA>::value(ygpu, A, x);
    report(equal(ycpu, ygpu), "Product<GPU::CUDA> ELL bit-exact " + tag);

    DenseVector<DT_> rcpu(n), rgpu(n);
    Defect<tags::CPU>::value(rcpu, b, A, x);
    Defect<tags::GPU::CUDA>::value(rgpu, b, A, x);
    report(equal(rcpu, rgpu), "Defect<GPU::CUDA> ELL bit-exact " + tag);

    const DT_ dc(DotProduct<tags::CPU>::value(x, y)), dg(DotProduct<tags::GPU::CUDA>::value(x, y));
    DT_ scale(0);
    for (unsigned long i(0) ; i < n ; ++i) scale += std::abs(x[i] * y[i]);
    const double tol(sizeof(DT_) == 8 ? 1e-13 : 1e-5);
    report(std::abs(dc - dg) <= tol * scale, "DotProduct<GPU::CUDA> " + tag);
    const DT_ nc(Norm<vnt_l_two, true, tags::CPU>::value(x)), ng(Norm<vnt_l_two, true, tags::GPU::CUDA>::value(x));
    report(std::abs(nc - ng) <= tol * nc, "Norm<l2, true, GPU::CUDA> " + tag);
    const DT_ nsc(Norm<vnt_l_two, false, tags::CPU>::value(x)), nsg(Norm<vnt_l_two, false, tags::GPU::CUDA>::value(x));
    report(std::abs(nsc - nsg) <= tol * nsc, "Norm<l2, false, GPU::CUDA> " + tag);

    DenseVector<DT_> a1(x.copy()), a2(x.copy());
    ScaledSum<tags::CPU>::value(a1, y, DT_(0.37));
    ScaledSum<tags::GPU::CUDA>::value(a2, y, DT_(0.37));
    report(equal(a1, a2), "ScaledSum<GPU::CUDA>(x, y, b) bit-exact " + tag);
    DenseVector<DT_> s1(n), s2(n);
    ScaledSum<tags::CPU>::value(s1, x, y, DT_(-1.25));
    ScaledSum<tags::GPU::CUDA>::value(s2, x, y, DT_(-1.25));
    report(equal(s1, s2), "ScaledSum<GPU::CUDA>(r, x, y, b) bit-exact " + tag);
    DenseVector<DT_> c1(x.copy()), c2(x.copy());
    Scale<tags::CPU>::value(c1, DT_(3.1));
    Scale<tags::GPU::CUDA>::value(c2, DT_(3.1));
    report(equal(c1, c2), "Scale<GPU::CUDA> bit-exact " + tag);
    DenseVector<DT_> u1(x.copy()), u2(x.copy());
    Sum<tags::CPU>::value(u1, y);
    Sum<tags::GPU::CUDA>::value(u2, y);
    report(equal(u1, u2), "Sum<GPU::CUDA> bit-exact " + tag);
    DenseVector<DT_> d1(x.copy()), d2(x.copy());
    Difference<tags::CPU>::value(d1, y);
    Difference<tags::GPU::CUDA>::value(d2, y);
    report(equal(d1, d2), "Difference<GPU::CUDA> bit-exact " + tag);
    DenseVector<DT_> e1(x.copy()), e2(x.copy());
    ElementProduct<tags::CPU>::value(e1, y);
    ElementProduct<tags::GPU::CUDA>::value(e2, y);
    report(equal(e1, e2), "ElementProduct<GPU::CUDA> bit-exact " + tag);

    // coherence: change x on the host after a GPU use; the next GPU product must see it
    x.lock(lm_read_and_write);
    x[n / 2] += DT_(1);
    x.unlock(lm_read_and_write);
    Product<tags::CPU>::value(ycpu, A, x);
    Product<tags::GPU::CUDA>::value(ygpu, A, x);
    report(equal(ycpu, ygpu), "host write of x is seen by the next GPU product " + tag);

    // a host change of the matrix values invalidates the device mirror
    A.Ax().lock(lm_read_and_write);
    A.Ax()[A.stride() * 4 + M + 1] *= DT_(2);
    A.Ax().unlock(lm_read_and_write);
    Product<tags::CPU>::value(ycpu, A, x);
    Product<tags::GPU::CUDA>::value(ygpu, A, x);
    report(equal(ycpu, ygpu), "host write of A is seen by the next GPU product " + tag);

    bool threw(false);
    try
    {
        DenseVector<DT_> wrong(n + 1);
        Product<tags::GPU::CUDA>::value(wrong, A, x);
    }
    catch (VectorSizeDoesNotMatch &)
    {
        threw = true;
    }
    report(threw, "VectorSizeDoesNotMatch before launch " + tag);
}

void generic_cg()
{
    // HONEI's generic CGSolver template on the GPU tag (operator by operator)
    SparseMatrixELL<double> A(q1<double>(65));
    const unsigned long n(A.rows());
    DenseVector<double> xt(seeded<double>(n, 7)), b(n);
    Product<tags::CPU>::value(b, A, xt);
    DenseVector<double> xc(n, 0.), xg(n, 0.);
    unsigned long uc(0), ug(0);
    CGSolver<tags::CPU, methods::NONE>::value(A, A, b, xc, 10000ul, uc, 1e-8);
    CGSolver<tags::GPU::CUDA, methods::NONE>::value(A, A, b, xg, 10000ul, ug, 1e-8);
    std::ostringstream d;
    d << "iterations cpu " << uc << " gpu " << ug;
    // tags::CPU's product reads elements() without locking: bring the GPU result home first
    xg.lock(lm_read_only);
    xg.unlock(lm_read_only);
    DenseVector<double> r(n);
    Defect<tags::CPU>::value(r, b, A, xg);
    const double rel(Norm<vnt_l_two, true, tags::CPU>::value(r) / Norm<vnt_l_two, true, tags::CPU>::value(b));
    d << ", relres " << rel;
    report((uc > ug ? uc - ug : ug - uc) <= 1 && rel < 1.5e-8, "generic CGSolver<GPU::CUDA, NONE> vs tags::CPU", d.str());
}

template <typename Tag_> double run_mg(const std::string & dir, unsigned long L, DenseVector<double> & x_out,
        unsigned long & cycles)
{
    typedef MGUtil<Tag_, SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>,
            MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, double> Util;
    MGData<SparseMatrixELL<double>, DenseVector<double>, SparseMatrixELL<double>, DenseVector<double>, double>
        data(Util::load_data(dir + "/", L, 0.7, "jac"));
    Util::configure(data, 100, 1000, 2, 2, 1, 1e-8);
    OperatorList ol(MGCycleCreation<Tag_, methods::CYCLE::V::STATIC, CGSolver<Tag_, methods::NONE>, RISmoother<Tag_>,
            Restriction<Tag_, methods::PROLMAT>, Prolongation<Tag_, methods::PROLMAT>, double>::value(data));
    const auto t0(std::chrono::steady_clock::now());
    MGSolver<Tag_, Norm<vnt_l_two, true, Tag_> >::value(data, ol);
    data.x.back().lock(lm_read_only);
    data.x.back().unlock(lm_read_only);
    const double ms(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    cycles = data.used_iters;
    x_out = data.x.back().copy();
    return ms;
}

void generic_mg(const std::string & dir, unsigned long L)
{
    DenseVector<double> xc(1), xg(1);
    unsigned long cc(0), cg(0);
    const double msc(run_mg<tags::CPU>(dir, L, xc, cc));
    run_mg<tags::GPU::CUDA>(dir, L, xg, cg);                 // first solve: uploads and mirrors
    const double msg(run_mg<tags::GPU::CUDA>(dir, L, xg, cg));
    double err(0), nrm(0);
    xc.lock(lm_read_only);
    xg.lock(lm_read_only);
    for (unsigned long i(0) ; i < xc.size() ; ++i)
    {
        err = std::max(err, std::abs(xc[i] - xg[i]));
        nrm = std::max(nrm, std::abs(xc[i]));
    }
    xc.unlock(lm_read_only);
    xg.unlock(lm_read_only);
    std::ostringstream d;
    d << "cycles cpu " << cc << " gpu " << cg << ", max |x_gpu - x_cpu| / max |x| = " << err / nrm << ", ms cpu "
      << msc << " gpu " << msg;
    report((cc > cg ? cc - cg : cg - cc) <= 1 && err <= 1e-6 * nrm, "MGSolver<GPU::CUDA> (MGUtil::load_data, V(2,2), jac)",
            d.str());
}

// BandedMatrixQx<Q1Type>: the reference's own banded Poisson fill, plus a banded matrix with
// seeded values on every band; product and defect on tags::GPU::CUDA against tags::CPU.
template <typename DT_> void banded(unsigned long M, const std::string & tag)
{
    const unsigned long n(M * M);
    DenseVector<DT_> z(n, DT_(0));
    BandedMatrixQx<Q1Type, DT_> P(n, z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(),
            z.copy(), z.copy());
    FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(P);
    BandedMatrixQx<Q1Type, DT_> R(n, seeded<DT_>(n, 11), seeded<DT_>(n, 12), seeded<DT_>(n, 13), seeded<DT_>(n, 14),
            seeded<DT_>(n, 15), seeded<DT_>(n, 16), seeded<DT_>(n, 17), seeded<DT_>(n, 18), seeded<DT_>(n, 19));
    DenseVector<DT_> x(seeded<DT_>(n, 4)), b(seeded<DT_>(n, 5));
    for (int k(0) ; k < 2 ; ++k)
    {
        const BandedMatrixQx<Q1Type, DT_> & A(k == 0 ? P : R);
        const std::string what(k == 0 ? " Poisson " : " seeded ");
        DenseVector<DT_> ycpu(n), ygpu(n);
        Product<tags::CPU>::value(ycpu, A, x);
        Product<tags::GPU::CUDA>::value(ygpu, A, x);
        report(equal(ycpu, ygpu), "Product<GPU::CUDA> BandedMatrixQx bit-exact" + what + tag);
        DenseVector<DT_> yret(Product<tags::GPU::CUDA>::value(A, x));
        report(equal(ycpu, yret), "Product<GPU::CUDA> BandedMatrixQx (value-returning) bit-exact" + what + tag);
        DenseVector<DT_> rcpu(n), rgpu(n);
        Defect<tags::CPU>::value(rcpu, b, A, x);
        Defect<tags::GPU::CUDA>::value(rgpu, b, A, x);
        report(equal(rcpu, rgpu), "Defect<GPU::CUDA> BandedMatrixQx bit-exact" + what + tag);
    }
    bool threw(false);
    try
    {
        DenseVector<DT_> wrong(n + 1);
        Product<tags::GPU::CUDA>::value(P, wrong);
    }
    catch (VectorSizeDoesNotMatch &)
    {
        threw = true;
    }
    report(threw, "BandedMatrixQx VectorSizeDoesNotMatch before launch " + tag);
}

// SparseMatrixCSR (csr::blocksize 1 and 4) built from the reference's Q1 ELL matrix, and the
// reference's own CSR product test matrix (rectangular, ragged last blocks): product and defect
// on tags::GPU::CUDA against tags::CPU.
template <typename DT_> void csr(unsigned long M, const std::string & tag)
{
    SparseMatrixELL<DT_> E(q1<DT_>(M));
    const unsigned long n(E.rows());
    DenseVector<DT_> x(seeded<DT_>(n, 21)), b(seeded<DT_>(n, 22));
    const unsigned long old(Configuration::instance()->get_value("csr::blocksize", 1));
    for (unsigned long bs(1) ; bs <= 4 ; bs *= 4)
    {
        Configuration::instance()->set_value("csr::blocksize", bs);
        SparseMatrixCSR<DT_> A(E);
        const std::string what(" blocksize " + std::to_string(bs) + " " + tag);
        DenseVector<DT_> ycpu(n), ygpu(n);
        Product<tags::CPU>::value(ycpu, A, x);
        Product<tags::GPU::CUDA>::value(ygpu, A, x);
        report(equal(ycpu, ygpu), "Product<GPU::CUDA> SparseMatrixCSR bit-exact" + what);
        DenseVector<DT_> rcpu(n), rgpu(n);
        Defect<tags::CPU>::value(rcpu, b, A, x);
        Defect<tags::GPU::CUDA>::value(rgpu, b, A, x);
        report(equal(rcpu, rgpu), "Defect<GPU::CUDA> SparseMatrixCSR bit-exact" + what);
        // the matrix of the reference's CSR product test (honei/la/product_TEST.cc:936-947)
        const unsigned long size(176);
        SparseMatrix<DT_> sms(size, size + 3);
        for (typename SparseMatrix<DT_>::ElementIterator i(sms.begin_elements()) ; i < sms.end_elements() ; ++i)
            if (i.index() % 5 == 0)
                *i = DT_(i.index()) / 1.234;
        SparseMatrixCSR<DT_> T(sms);
        DenseVector<DT_> dv1(size + 3, DT_(4));
        dv1[0] = 1;
        dv1[1] = 2;
        DenseVector<DT_> pc(size, DT_(4711)), pg(size, DT_(4711));
        Product<tags::CPU>::value(pc, T, dv1);
        Product<tags::GPU::CUDA>::value(pg, T, dv1);
        report(equal(pc, pg), "Product<GPU::CUDA> SparseMatrixCSR (reference test matrix) bit-exact" + what);
    }
    Configuration::instance()->set_value("csr::blocksize", old);
    bool threw(false);
    try
    {
        SparseMatrixCSR<DT_> A(E);
        DenseVector<DT_> wrong(n + 1), y(n);
        Product<tags::GPU::CUDA>::value(y, A, wrong);
    }
    catch (VectorSizeDoesNotMatch &)
    {
        threw = true;
    }
    report(threw, "SparseMatrixCSR VectorSizeDoesNotMatch before launch " + tag);
}

// SPAI2<tags::GPU::CUDA> against SPAI2<tags::CPU::SSE> (the tag honei/math/spai2_TEST.cc runs):
// every entry of M bit-identical, the pattern that of A.
template <typename DT_> void spai(unsigned long M, const std::string & tag)
{
    SparseMatrix<DT_> A(q1<DT_>(M));
    SparseMatrix<DT_> mc(A.copy()), mg(A.rows(), A.columns());
    SPAI2<tags::CPU::SSE>::value(mc, A);
    SPAI2<tags::GPU::CUDA>::value(mg, A);
    bool ok(true);
    for (unsigned long r(0) ; ok && r < A.rows() ; ++r)
    {
        const SparseVector<DT_> & c(mc[r]), & g(mg[r]), & a(A[r]);
        ok = c.used_elements() == g.used_elements() && g.used_elements() == a.used_elements();
        for (unsigned long i(0) ; ok && i < c.used_elements() ; ++i)
            ok = c.indices()[i] == g.indices()[i] && g.indices()[i] == a.indices()[i] &&
                std::memcmp(c.elements() + i, g.elements() + i, sizeof(DT_)) == 0;
    }
    report(ok, "SPAI2<GPU::CUDA> bit-exact to SPAI2<CPU::SSE> " + tag);
    bool threw(false);
    try
    {
        SparseMatrix<DT_> R(4, 6), out(4, 6);
        R(0, 0, DT_(1));
        SPAI2<tags::GPU::CUDA>::value(out, R);
    }
    catch (MatrixIsNotSquare &)
    {
        threw = true;
    }
    report(threw, "SPAI2<GPU::CUDA> MatrixIsNotSquare " + tag);
}

// The honeirc block-size keys (honei/honeirc: cuda::product_smell_dv_*, cuda::product_bmdv_q1_*,
// cuda::scaled_sum_two_*): each value set through Configuration reaches the plugin's context
// (clamped to the kernel's range, a multiple of 32), and the results stay bit-exact to tags::CPU.
template <typename DT_> void honeirc_blocks(unsigned long M, const std::string & tag)
{
    const bool dbl(sizeof(DT_) == 8);
    const std::string ell(dbl ? "cuda::product_smell_dv_double" : "cuda::product_smell_dv_float");
    const std::string band(dbl ? "cuda::product_bmdv_q1_double" : "cuda::product_bmdv_q1_float");
    const std::string axpy(dbl ? "cuda::scaled_sum_two_double" : "cuda::scaled_sum_two_float");
    SparseMatrixELL<DT_> A(q1<DT_>(M));
    const unsigned long n(A.rows());
    DenseVector<DT_> z(n, DT_(0));
    BandedMatrixQx<Q1Type, DT_> Q(n, z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(),
            z.copy(), z.copy());
    FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(Q);
    DenseVector<DT_> x(seeded<DT_>(n, 31)), w(seeded<DT_>(n, 32));
    DenseVector<DT_> ycpu(n), qcpu(n), acpu(x.copy());
    Product<tags::CPU>::value(ycpu, A, x);
    Product<tags::CPU>::value(qcpu, Q, x);
    ScaledSum<tags::CPU>::value(acpu, w, DT_(0.5));
    const int sizes[] = {32, 96, 128, 200, 256, 1000};
    for (int bs : sizes)
    {
        Configuration::instance()->set_value(ell, bs);
        Configuration::instance()->set_value(band, bs);
        Configuration::instance()->set_value(axpy, bs);
        DenseVector<DT_> y(n), q(n), a(x.copy());
        Product<tags::GPU::CUDA>::value(y, A, x);
        const int got_ell(hb_set_block_size(b200::context(), HB_BLOCK_ELL, 0));
        Product<tags::GPU::CUDA>::value(q, Q, x);
        const int got_band(hb_set_block_size(b200::context(), HB_BLOCK_Q1BAND, 0));
        ScaledSum<tags::GPU::CUDA>::value(a, w, DT_(0.5));
        const int got_vec(hb_set_block_size(b200::context(), HB_BLOCK_VECTOR, 0));
        const int want(bs > 256 ? 256 : bs - bs % 32), want_vec(bs - bs % 32);
        std::ostringstream d;
        d << "context blocks " << got_ell << " / " << got_band << " / " << got_vec;
        report(got_ell == want && got_band == want && got_vec == want_vec && equal(ycpu, y) && equal(qcpu, q)
                && equal(acpu, a), "honeirc block size " + std::to_string(bs) + " applied, results bit-exact " + tag,
                d.str());
    }
    Configuration::instance()->set_value(ell, 128);
    Configuration::instance()->set_value(band, 128);
    Configuration::instance()->set_value(axpy, 128);
}

int main(int argc, char ** argv)
{
    honeirc_blocks<double>(33, "f64 33^2");
    honeirc_blocks<float>(65, "f32 65^2");
    spai<double>(33, "f64 33^2");
    spai<float>(65, "f32 65^2");
    csr<double>(33, "f64 33^2");
    csr<float>(65, "f32 65^2");
    banded<double>(33, "f64 33^2");
    banded<float>(129, "f32 129^2");
    operators<double>(33, "f64 33^2");
    operators<double>(129, "f64 129^2");
    operators<float>(65, "f32 65^2");
    generic_cg();
    if (argc > 2)
        generic_mg(argv[1], std::stoul(argv[2]));
    std::printf("%d failure(s)\n", failures());
    return failures() ? 1 : 0;
}
