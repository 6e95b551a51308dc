// HONEI's multigrid path on tags::GPU::CUDA with the plugin's specialisations
// (honei_b200/plugin/mg_b200.hh: fused RISmoother sweeps, the V::STATIC cycle as one backend
// operator, MGSolver's loop as hb_mg_solve), against tags::CPU on the same MGData, plus
// IRSolver<GPU::CUDA, GPU::CUDA> (whose inner MGSolver takes the fast path) against
// IRSolver<CPU, CPU>.
//   plugin_mg_test mg_dir L
// mg_dir holds A_1..A_L.ell, prol_2..prol_L.ell, rhs_L, init_L (HONEI file formats), loaded with
// MGUtil::load_data as honei/math/mg_TEST.cc loads FEATFLOW data.
#include "plugin_common.hh"

#include <honei_b200/plugin/mg_b200.hh>

#include <honei/la/norm.hh>
#include <honei/la/product.hh>
#include <honei/math/defect.hh>
#include <honei/math/ir.hh>
#include <honei/math/matrix_io.hh>
#include <honei/math/mg.hh>
#include <honei/math/vector_io.hh>

#include <chrono>
#include <cmath>
#include <sstream>

using namespace honei;
using namespace plugin_test;

template <typename DT_> using Data = MGData<SparseMatrixELL<DT_>, DenseVector<DT_>, SparseMatrixELL<DT_>,
      DenseVector<DT_>, DT_>;
template <typename Tag_, typename DT_> using Util = MGUtil<Tag_, SparseMatrixELL<DT_>, DenseVector<DT_>,
      SparseMatrixELL<DT_>, DenseVector<DT_>, MatrixIO<io_formats::ELL>, VectorIO<io_formats::EXP>, DT_>;

template <typename Tag_, typename DT_> OperatorList vcycle(Data<DT_> & data)
{
    return MGCycleCreation<Tag_, methods::CYCLE::V::STATIC, CGSolver<Tag_, methods::NONE>, RISmoother<Tag_>,
           Restriction<Tag_, methods::PROLMAT>, Prolongation<Tag_, methods::PROLMAT>, DT_>::value(data);
}

template <typename DT_> void host(const DenseVector<DT_> & v)
{
    v.lock(lm_read_only);
    v.unlock(lm_read_only);
}

template <typename DT_> bool equal(const DenseVector<DT_> & a, const DenseVector<DT_> & b)
{
    host(a);
    host(b);
    bool ok(a.size() == b.size());
    for (unsigned long i(0) ; ok && i < a.size() ; ++i)
        ok = (a[i] == b[i]);
    return ok;
}

double relres(SparseMatrixELL<double> & A, DenseVector<double> & b, DenseVector<double> & x)
{
    host(x);
    DenseVector<double> r(b.size());
    Defect<tags::CPU>::value(r, b, A, x);
    return Norm<vnt_l_two, true, tags::CPU>::value(r) / Norm<vnt_l_two, true, tags::CPU>::value(b);
}

template <typename Tag_> double run_mg(const std::string & dir, unsigned long L, unsigned long max_iters,
        unsigned long max_coarse, DenseVector<double> & x_out, unsigned long & cycles)
{
    Data<double> data(Util<Tag_, double>::load_data(dir + "/", L, 0.7, "jac"));
    Util<Tag_, double>::configure(data, max_iters, max_coarse, 2, 2, 1, 1e-8);
    OperatorList ol(vcycle<Tag_, double>(data));
    const auto t0(std::chrono::steady_clock::now());
    MGSolver<Tag_, Norm<vnt_l_two, true, Tag_> >::value(data, ol);
    host(data.x.back());
    const double ms(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    cycles = data.used_iters;
    x_out = data.x.back().copy();
    return ms;
}

void mg_solver(const std::string & dir, unsigned long L)
{
    DenseVector<double> xc(1), xg(1);
    unsigned long cc(0), cg(0);
    const double msc(run_mg<tags::CPU>(dir, L, 100, 1000, xc, cc));
    run_mg<tags::GPU::CUDA>(dir, L, 100, 1000, xg, cg);                 // first solve: set-up, graph capture
    const double msg(run_mg<tags::GPU::CUDA>(dir, L, 100, 1000, xg, cg));
    double err(0), nrm(0);
    host(xc);
    host(xg);
    for (unsigned long i(0) ; i < xc.size() ; ++i)
    {
        err = std::max(err, std::abs(xc[i] - xg[i]));
        nrm = std::max(nrm, std::abs(xc[i]));
    }
    Data<double> d(Util<tags::CPU, double>::load_data(dir + "/", L, 0.7, "jac"));
    const double rg(relres(d.A.back(), d.b.back(), xg)), rc(relres(d.A.back(), d.b.back(), xc));
    std::ostringstream s;
    s << "cycles cpu " << cc << " gpu " << cg << ", relres cpu " << rc << " gpu " << rg
      << ", max |x_gpu - x_cpu| / max |x| = " << err / nrm << ", ms cpu " << msc << " gpu " << msg;
    report((cc > cg ? cc - cg : cg - cc) <= 1 && std::abs(rg - rc) <= 1e-10 && err <= 1e-6 * nrm,
            "MGSolver<GPU::CUDA> fast path vs tags::CPU (V(2,2), jac)", s.str());
}

// One cycle with no coarse iterations: smoothing, defects and transfers only, which round
// exactly as tags::CPU: the same x bit for bit.
void one_cycle_bit_exact(const std::string & dir, unsigned long L)
{
    DenseVector<double> xc(1), xg(1);
    unsigned long cc(0), cg(0);
    run_mg<tags::CPU>(dir, L, 1, 0, xc, cc);
    run_mg<tags::GPU::CUDA>(dir, L, 1, 0, xg, cg);
    report(cc == 1 && cg == 1 && equal(xc, xg), "MG cycle<GPU::CUDA> without coarse iterations bit-exact");
    // the cycle operator driven by OperatorList::value() (not MGSolver): two cycles
    Data<double> dc(Util<tags::CPU, double>::load_data(dir + "/", L, 0.7, "jac"));
    Data<double> dg(Util<tags::GPU::CUDA, double>::load_data(dir + "/", L, 0.7, "jac"));
    Util<tags::CPU, double>::configure(dc, 1, 0, 2, 2, 1, 1e-8);
    Util<tags::GPU::CUDA, double>::configure(dg, 1, 0, 2, 2, 1, 1e-8);
    OperatorList oc(vcycle<tags::CPU, double>(dc)), og(vcycle<tags::GPU::CUDA, double>(dg));
    for (int k(0) ; k < 2 ; ++k)
    {
        oc.value();
        og.value();
    }
    report(og.size() == 1 && equal(dc.x.back(), dg.x.back()), "OperatorList::value() of the B200 cycle bit-exact");
}

// RISmoother<GPU::CUDA> on the finest level of the data: three sweeps, bit for bit.
void smoother(const std::string & dir, unsigned long L)
{
    Data<double> d(Util<tags::CPU, double>::load_data(dir + "/", L, 0.7, "jac"));
    SparseMatrixELL<double> & A(d.A.back());
    DenseVector<double> & P(d.P.back());
    DenseVector<double> b(seeded<double>(A.rows(), 21)), xc(seeded<double>(A.rows(), 22)), xg(xc.copy());
    std::vector<DenseVector<double> > tc, tg;
    for (int k(0) ; k < 2 ; ++k)
    {
        tc.push_back(DenseVector<double>(A.rows(), 0.));
        tg.push_back(DenseVector<double>(A.rows(), 0.));
    }
    RISmoother<tags::CPU>::value(A, P, b, xc, tc, 3ul);
    RISmoother<tags::GPU::CUDA>::value(A, P, b, xg, tg, 3ul);
    report(equal(xc, xg), "RISmoother<GPU::CUDA> (fused sweeps) bit-exact");
}

// IRSolver (honei/math/ir.hh:30-78): FP64 outer loop, FP32 inner MG (V(2,2), coarse CG), warm
// inner start; tags::CPU against tags::GPU::CUDA.
template <typename Tag_> double run_ir(const std::string & dir, unsigned long L, DenseVector<double> & x,
        unsigned long & used)
{
    Data<float> data(Util<Tag_, float>::load_data(dir + "/", L, 0.7f, "jac"));
    Util<Tag_, float>::configure(data, 100, 100, 2, 2, 1, 1e-3f);
    OperatorList ol(vcycle<Tag_, float>(data));
    SparseMatrixELL<double> A(MatrixIO<io_formats::ELL>::read_matrix(dir + "/A_" + std::to_string(L) + ".ell", double(0)));
    DenseVector<double> b(VectorIO<io_formats::EXP>::read_vector(dir + "/rhs_" + std::to_string(L), double(0)));
    x = DenseVector<double>(b.size(), 0.);
    used = 0;
    const auto t0(std::chrono::steady_clock::now());
    IRSolver<Tag_, Tag_, Norm<vnt_l_two, true, Tag_> >::value(A, b, x, data, ol, 1e-10, 100ul, used);
    host(x);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void ir_solver(const std::string & dir, unsigned long L)
{
    DenseVector<double> xc(1), xg(1);
    unsigned long uc(0), ug(0);
    const double msc(run_ir<tags::CPU>(dir, L, xc, uc));
    run_ir<tags::GPU::CUDA>(dir, L, xg, ug);
    const double msg(run_ir<tags::GPU::CUDA>(dir, L, xg, ug));
    SparseMatrixELL<double> A(MatrixIO<io_formats::ELL>::read_matrix(dir + "/A_" + std::to_string(L) + ".ell", double(0)));
    DenseVector<double> b(VectorIO<io_formats::EXP>::read_vector(dir + "/rhs_" + std::to_string(L), double(0)));
    const double rc(relres(A, b, xc)), rg(relres(A, b, xg));
    std::ostringstream s;
    s << "outer cpu " << uc << " gpu " << ug << ", relres cpu " << rc << " gpu " << rg << ", ms cpu " << msc
      << " gpu " << msg;
    report((uc > ug ? uc - ug : ug - uc) <= 1 && rc < 1e-10 && rg < 1e-10,
            "IRSolver<GPU::CUDA, GPU::CUDA> (inner MGSolver fast path) vs tags::CPU", s.str());
}

int main(int argc, char ** argv)
{
    if (argc < 3)
    {
        std::printf("usage: plugin_mg_test mg_dir L\n");
        return 2;
    }
    const std::string dir(argv[1]);
    const unsigned long L(std::stoul(argv[2]));
    smoother(dir, L);
    one_cycle_bit_exact(dir, L);
    mg_solver(dir, L);
    ir_solver(dir, L);
    std::printf("%d failure(s)\n", failures());
    return failures() ? 1 : 0;
}
