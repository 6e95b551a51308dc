// CGSolver<tags::GPU::CUDA, methods::NONE> and <.., methods::VAR> with the plugin's full
// specialisations (honei_b200/plugin/solvers_b200.hh: one persistent kernel per solve) against
// tags::CPU.
#include "plugin_common.hh"

#include <honei_b200/plugin/solvers_b200.hh>

#include <honei/la/norm.hh>
#include <honei/la/product.hh>
#include <honei/la/sparse_matrix.hh>
#include <honei/math/cg.hh>
#include <honei/math/defect.hh>

#include <sstream>

using namespace honei;
using namespace plugin_test;

template <typename DT_> void check_cg(unsigned long M, double eps, const std::string & tag)
{
    SparseMatrixELL<DT_> A(q1<DT_>(M));
    const unsigned long n(A.rows());
    DenseVector<DT_> xt(seeded<DT_>(n, 11)), b(n);
    Product<tags::CPU>::value(b, A, xt);
    DenseVector<DT_> xc(n, DT_(0)), xg(n, DT_(0));
    unsigned long uc(0), ug(0);
    CGSolver<tags::CPU, methods::NONE>::value(A, A, b, xc, 20000ul, uc, DT_(eps));
    CGSolver<tags::GPU::CUDA, methods::NONE>::value(A, A, b, xg, 20000ul, ug, DT_(eps));
    DenseVector<double> r(n), bd(n), xd(n);
    xg.lock(lm_read_only);
    for (unsigned long i(0) ; i < n ; ++i) { xd[i] = xg[i]; bd[i] = b[i]; }
    xg.unlock(lm_read_only);
    SparseMatrixELL<double> A64(q1<double>(M));
    Defect<tags::CPU>::value(r, bd, A64, xd);
    const double rel(Norm<vnt_l_two, true, tags::CPU>::value(r) / Norm<vnt_l_two, true, tags::CPU>::value(bd));
    std::ostringstream d;
    d << "iterations cpu " << uc << " gpu " << ug << ", relres " << rel;
    const unsigned long slack(1);
    report((uc > ug ? uc - ug : ug - uc) <= slack && rel < (sizeof(DT_) == 8 ? 1.5e-8 : 1e-4),
            "CGSolver<GPU::CUDA, NONE> specialisation " + tag, d.str());
}

// CGSolver<VAR> with a Jacobi vector (0.7 / diag, as honei/math/cg_TEST.cc builds it) and the
// same preconditioner as a diagonal SparseMatrixELL.
template <typename DT_> void check_cg_var(unsigned long M, double eps, const std::string & tag)
{
    SparseMatrixELL<DT_> A(q1<DT_>(M));
    const unsigned long n(A.rows());
    DenseVector<DT_> xt(seeded<DT_>(n, 12)), b(n), P(n);
    Product<tags::CPU>::value(b, A, xt);
    for (unsigned long i(0) ; i < n ; ++i) P[i] = DT_(0.7) / A(i, i);
    SparseMatrix<DT_> Ps(n, n);
    for (unsigned long i(0) ; i < n ; ++i) Ps(i, i) = P[i];
    SparseMatrixELL<DT_> Pm(Ps);
    for (int k(0) ; k < 2 ; ++k)
    {
        DenseVector<DT_> xc(n, DT_(0)), xg(n, DT_(0));
        unsigned long uc(0), ug(0);
        if (k == 0)
        {
            CGSolver<tags::CPU, methods::VAR>::value(A, P, b, xc, 5000ul, uc, DT_(eps));
            CGSolver<tags::GPU::CUDA, methods::VAR>::value(A, P, b, xg, 5000ul, ug, DT_(eps));
        }
        else
        {
            CGSolver<tags::CPU, methods::VAR>::value(A, Pm, b, xc, 5000ul, uc, DT_(eps));
            CGSolver<tags::GPU::CUDA, methods::VAR>::value(A, Pm, b, xg, 5000ul, ug, DT_(eps));
        }
        xg.lock(lm_read_only);
        double err(0), nrm(0);
        for (unsigned long i(0) ; i < n ; ++i)
        {
            err = std::max(err, std::abs(double(xg[i]) - double(xc[i])));
            nrm = std::max(nrm, std::abs(double(xc[i])));
        }
        xg.unlock(lm_read_only);
        std::ostringstream d;
        d << "iterations cpu " << uc << " gpu " << ug << ", max |x_gpu - x_cpu| / |x| " << err / nrm;
        const unsigned long slack(1);
        report((uc > ug ? uc - ug : ug - uc) <= slack && err <= (sizeof(DT_) == 8 ? 1e-7 : 1e-3) * nrm,
                std::string("CGSolver<GPU::CUDA, VAR> ") + (k == 0 ? "vector P " : "matrix P ") + tag, d.str());
    }
}

int main()
{
    check_cg_var<double>(65, 1e-8, "f64 65^2");
    check_cg_var<float>(33, 1e-5, "f32 33^2");
    check_cg<double>(33, 1e-8, "f64 33^2");
    check_cg<double>(257, 1e-8, "f64 257^2");
    check_cg<float>(65, 1e-5, "f32 65^2");
    // used_iters is left untouched when max_iters == 0, as cg.hh leaves it
    SparseMatrixELL<double> A(q1<double>(9));
    DenseVector<double> b(seeded<double>(81, 3)), x(81, 0.);
    unsigned long used(42);
    CGSolver<tags::GPU::CUDA, methods::NONE>::value(A, A, b, x, 0ul, used, 1e-8);
    report(used == 42, "max_iters = 0 leaves used_iters");
    std::printf("%d failure(s)\n", failures());
    return failures() ? 1 : 0;
}
