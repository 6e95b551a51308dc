// Shared helpers of the HONEI plugin tests (tests/plugin): tiny PASS/FAIL reporting and the
// reference's own Q1 Poisson construction.
#pragma once
#include <honei/la/banded_matrix_qx.hh>
#include <honei/la/dense_vector.hh>
#include <honei/la/sparse_matrix.hh>
#include <honei/la/sparse_matrix_ell.hh>
#include <honei/math/fill_matrix.hh>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace plugin_test
{
    inline int & failures() { static int f = 0; return f; }

    inline void report(bool ok, const std::string & name, const std::string & detail = "")
    {
        std::printf("%s %s%s%s\n", ok ? "PASS" : "FAIL", name.c_str(), detail.empty() ? "" : " : ", detail.c_str());
        if (! ok) ++failures();
    }

    // FillMatrix<POISSON, DIRICHLET_0> -> SparseMatrix -> SparseMatrixELL (the reference path).
    template <typename DT_> honei::SparseMatrixELL<DT_> q1(unsigned long M)
    {
        using namespace honei;
        const unsigned long N(M * M);
        DenseVector<DT_> z(N, DT_(0));
        BandedMatrixQx<Q1Type, DT_> q(N, z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(),
                z.copy(), z.copy());
        FillMatrix<tags::CPU, applications::POISSON, boundary_types::DIRICHLET::DIRICHLET_0>::value(q);
        SparseMatrix<DT_> s(q);
        return SparseMatrixELL<DT_>(s);
    }

    template <typename DT_> honei::DenseVector<DT_> seeded(unsigned long n, unsigned seed)
    {
        honei::DenseVector<DT_> v(n);
        std::srand(seed);
        for (unsigned long i(0) ; i < n ; ++i)
            v[i] = DT_(2.0 * std::rand() / double(RAND_MAX) - 1.0);
        return v;
    }
}
