// End-to-end timing of the product through HONEI's own API on the B200 plugin: host DenseVectors
// and a host SparseMatrixELL, Product<tags::GPU::CUDA>::value(y, A, x) as a HONEI caller writes
// it.  Each step the caller rewrites x on the host (so MemoryArbiter uploads it again through
// MemoryBackend<tags::GPU::CUDA>, honei/util/memory_arbiter-impl.hh:599-640,
// honei/util/memory_backend.hh:131-165), runs K products on the GPU tag and reads y on the host
// (the arbiter downloads it).  K = 1 is one product per upload; K = 10 the benchmark's step.
//   plugin_product_bench [M=2049] [steps=20]
// Prints one JSON line.  The matrix is the Q1 Poisson stencil of an M x M grid (Dirichlet rows
// identity), built with the reference's raw SparseMatrixELL constructor.
#include "plugin_common.hh"

#include <honei/la/product.hh>
#include <honei/util/configuration.hh>
#include <honei/util/memory_arbiter.hh>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <vector>

using namespace honei;

namespace
{
    SparseMatrixELL<double> q1_raw(unsigned long M)
    {
        const unsigned long n(M * M), stride((n + 31) / 32 * 32), ncpr(9);
        DenseVector<unsigned long> Aj(ncpr * stride, 0ul);
        DenseVector<double> Ax(ncpr * stride, 0.);
        const long offs[9] = {-(long)M - 1, -(long)M, -(long)M + 1, -1, 0, 1, (long)M - 1, (long)M, (long)M + 1};
        for (unsigned long r(0) ; r < n ; ++r)
        {
            const unsigned long i(r / M), j(r % M);
            if (i == 0 || j == 0 || i == M - 1 || j == M - 1)
            {
                Aj[r] = r;
                Ax[r] = 1.;
                continue;
            }
            for (unsigned long k(0) ; k < 9 ; ++k)
            {
                Aj[r + k * stride] = (unsigned long)((long)r + offs[k]);
                Ax[r + k * stride] = k == 4 ? 8. / 3. : -1. / 3.;
            }
        }
        return SparseMatrixELL<double>(n, n, stride, ncpr, Aj, Ax, 1);
    }

    double median(std::vector<double> v)
    {
        std::sort(v.begin(), v.end());
        return v[v.size() / 2];
    }
}

int main(int argc, char ** argv)
{
    const unsigned long M(argc > 1 ? std::stoul(argv[1]) : 2049), steps(argc > 2 ? std::stoul(argv[2]) : 20);
    SparseMatrixELL<double> A(q1_raw(M));
    const unsigned long n(A.rows()), nnz(A.used_elements());
    const double bytes(double(nnz) * 12. + 2. * double(n) * 8.);
    DenseVector<double> x(plugin_test::seeded<double>(n, 1)), y(n, 0.), yc(n, 0.);
    Product<tags::CPU>::value(yc, A, x);
    Product<tags::GPU::CUDA>::value(y, A, x);          // first use: matrix upload and device mirror
    y.lock(lm_read_only);
    bool same(true);
    for (unsigned long i(0) ; i < n ; i += 997)
        same = same && y[i] == yc[i];
    y.unlock(lm_read_only);
    double out[2] = {0., 0.}, ms[2] = {0., 0.};
    const unsigned long ks[2] = {1, 10};
    // the product kernel's block size, as honeirc gives it (cuda::product_smell_dv_double)
    const int configured(Configuration::instance()->get_value("cuda::product_smell_dv_double", 128));
    for (int c(0) ; c < 2 ; ++c)
    {
        std::vector<double> t;
        for (unsigned long s(0) ; s < steps + 2 ; ++s)
        {
            const auto t0(std::chrono::steady_clock::now());
            x.lock(lm_write_only);                       // the caller writes its next x on the host
            x[s % n] = x[s % n];
            x.unlock(lm_write_only);
            for (unsigned long k(0) ; k < ks[c] ; ++k)
                Product<tags::GPU::CUDA>::value(y, A, x);
            y.lock(lm_read_only);                        // and reads y on the host
            volatile double sink(y[n / 2]);
            (void)sink;
            y.unlock(lm_read_only);
            const double dt(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
            if (s >= 2)
                t.push_back(dt);
        }
        ms[c] = 1e3 * median(t);
        out[c] = double(ks[c]) * bytes / (ms[c] * 1e-3) / 1e9;
    }
    std::printf("{\"api\": \"Product<tags::GPU::CUDA>::value(DenseVector&, const SparseMatrixELL&, const DenseVector&)"
            " with host DenseVectors through MemoryArbiter / MemoryBackend<tags::GPU::CUDA>\", \"rows\": %lu, \"nnz\": %lu, "
            "\"bytes_per_product\": %.0f, \"one_product_per_upload_gbs\": %.2f, \"ms_per_product_one_per_upload\": %.4f, "
            "\"ten_products_per_upload_gbs\": %.2f, \"ms_per_step_ten_products\": %.4f, \"h2d_bytes_per_step\": %lu, "
            "\"d2h_bytes_per_step\": %lu, \"steps\": %lu, \"y_equals_tags_cpu\": %s, \"honeirc_block\": %d}\n",
            n, nnz, bytes, out[0], ms[0], out[1], ms[1], n * 8, n * 8, steps, same ? "true" : "false", configured);
    return same ? 0 : 1;
}
