/* operations_b200.cc -- HONEI's tags::GPU::CUDA operators on the B200 backend.
 *
 * Defines the static members HONEI declares unconditionally for the GPU tag:
 *   Product<tags::GPU::CUDA>         honei/la/product.hh:1728-1794   (ELL and CSR SpMV, banded
 *                                                                     Q1 product, Jacobi apply)
 *   Defect<tags::GPU::CUDA>          honei/math/defect.hh:645-692    (ELL, CSR and banded Q1 defect)
 *   DotProduct<tags::GPU::CUDA>      honei/la/dot_product.hh:343-368
 *   Norm<vnt_l_two, {false,true}, tags::GPU::CUDA>  honei/la/norm.hh:538-580
 *   ScaledSum<tags::GPU::CUDA>       honei/la/scaled_sum.hh:444-488
 *   Scale, Sum, Difference, ElementProduct <tags::GPU::CUDA>
 *   SPAI2<tags::GPU::CUDA>           honei/math/spai2.hh:294-298     (SparseMatrix in and out)
 * Every operator checks sizes first and throws VectorSizeDoesNotMatch as the CPU tags do, locks
 * its vectors for tags::GPU::CUDA (the MemoryArbiter uploads lazily through
 * MemoryBackend<tags::GPU::CUDA>), calls one entry point of the C ABI, and unlocks.  Results
 * stay on the device until a host lock reads them back.
 *
 * Block sizes come from HONEI's Configuration, as the reference's CUDA wrappers take them (e.g.
 * honei/la/product-cuda.cc:594-625, honei/la/scaled_sum-cuda.cc:210-236): before each call the
 * operator reads its honeirc key (cuda::product_smell_dv_{float,double} for the ELL product and
 * defect, cuda::product_bmdv_q1_* for the banded ones, cuda::scaled_sum_two_*,
 * cuda::scaled_sum_three_*, cuda::scale_one_*, cuda::sum_two_*, cuda::difference_two_*,
 * cuda::element_product_two_* for the vector operators; default 128 as there) and sets it on
 * the context (hb_set_block_size), clamped to the kernel's range and rounded down to a multiple
 * of 32.  The results do not depend on it.  The dot-product and norm keys are not used: those
 * kernels keep one fixed reduction tree.  ell::threads is honoured by the matrices themselves:
 * a SparseMatrixELL built with T lanes per row is imported with its T.
 */
#include "b200_backend.hh"

#include <honei/la/dense_vector.hh>
#include <honei/la/dot_product.hh>
#include <honei/la/difference.hh>
#include <honei/la/element_product.hh>
#include <honei/la/norm.hh>
#include <honei/la/product.hh>
#include <honei/la/scale.hh>
#include <honei/la/scaled_sum.hh>
#include <honei/la/sparse_matrix_csr.hh>
#include <honei/la/sum.hh>
#include <honei/la/vector_error.hh>
#include <honei/la/matrix_error.hh>
#include <honei/math/defect.hh>
#include <honei/math/spai2.hh>
#include <honei/util/configuration.hh>
#include <honei/util/memory_arbiter.hh>

#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>
#include <vector>

namespace honei
{
    namespace b200
    {
        hb_context * context()
        {
            struct Holder
            {
                hb_context * ctx = nullptr;
                ~Holder() { if (ctx) hb_destroy(ctx); }
            };
            thread_local Holder h;
            if (! h.ctx)
            {
                int dev(0);
                cudaGetDevice(&dev);
                check(hb_create(&h.ctx, dev), "hb_create");
            }
            return h.ctx;
        }

        void check(int status, const char * what)
        {
            if (status != HB_OK)
            {
                std::string msg(std::string(what) + ": " + hb_status_string(status));
                throw InternalError(msg);
            }
        }

        namespace
        {
            struct Mirror
            {
                hb_ell ell;
                std::uint64_t gen[3];
                void * Aj_dev[3];
            };

            struct CsrMirror
            {
                hb_csr csr;
                std::uint64_t gen[3];
                void * dev[3];
            };

            std::mutex g_mirror_mutex;
            std::map<void *, Mirror> g_mirrors;        // keyed by the Ax memid
            std::map<void *, CsrMirror> g_csr_mirrors; // keyed by the Ax memid

            void free_csr(hb_csr & c)
            {
                cudaFree(c.Ar);
                cudaFree(c.Aj);
                cudaFree(c.Ax);
                c.Ar = nullptr;
                c.Aj = nullptr;
                c.Ax = nullptr;
            }

            template <typename DT_> int dtype_of();
            template <> int dtype_of<double>() { return HB_F64; }
            template <> int dtype_of<float>() { return HB_F32; }

            int import(const SparseMatrixELL<double> & a, const void * aj, const void * ax, const void * arl, hb_ell & out)
            {
                return hb_ell_import_f64(context(), a.rows(), a.columns(), a.stride(), a.num_cols_per_row(), a.threads(),
                        (const uint64_t *)aj, (const double *)ax, (const uint64_t *)arl, &out);
            }

            int import(const SparseMatrixELL<float> & a, const void * aj, const void * ax, const void * arl, hb_ell & out)
            {
                return hb_ell_import_f32(context(), a.rows(), a.columns(), a.stride(), a.num_cols_per_row(), a.threads(),
                        (const uint64_t *)aj, (const float *)ax, (const uint64_t *)arl, &out);
            }
        }

        void forget(void * memid)
        {
            std::lock_guard<std::mutex> l(g_mirror_mutex);
            auto i(g_mirrors.find(memid));
            if (i != g_mirrors.end())
            {
                cudaFree(i->second.ell.Aj);
                cudaFree(i->second.ell.Ax);
                g_mirrors.erase(i);
            }
            auto c(g_csr_mirrors.find(memid));
            if (c != g_csr_mirrors.end())
            {
                free_csr(c->second.csr);
                g_csr_mirrors.erase(c);
            }
        }

        /// The hb_csr mirror of a SparseMatrixCSR: imported from the backend's copies of
        /// Ar / Aj / Ax on first use, again whenever one of them was uploaded again.
        template <typename DT_> const hb_csr & device_mirror(const SparseMatrixCSR<DT_> & a)
        {
            // the stored blocks (Aj may be allocated longer: the reference sizes it by entries)
            const std::int64_t nb((std::int64_t)a.Ar()[a.rows()]);
            void * ar(a.Ar().lock(lm_read_only, tags::GPU::CUDA::memory_value));
            void * aj(a.Aj().lock(lm_read_only, tags::GPU::CUDA::memory_value));
            void * ax(a.Ax().lock(lm_read_only, tags::GPU::CUDA::memory_value));
            const std::uint64_t g0(generation(a.Ar().memid(), a.Ar().address()));
            const std::uint64_t g1(generation(a.Aj().memid(), a.Aj().address()));
            const std::uint64_t g2(generation(a.Ax().memid(), a.Ax().address()));
            std::lock_guard<std::mutex> l(g_mirror_mutex);
            CsrMirror & m(g_csr_mirrors[a.Ax().memid()]);
            int st(HB_OK);
            if (! m.csr.Ar || m.gen[0] != g0 || m.gen[1] != g1 || m.gen[2] != g2 || m.dev[0] != ar
                    || m.dev[1] != aj || m.dev[2] != ax)
            {
                const std::int64_t bs((std::int64_t)a.blocksize());
                if (! m.csr.Ar || m.csr.rows != (std::int64_t)a.rows() || m.csr.nblocks != nb || m.csr.blocksize != bs)
                {
                    free_csr(m.csr);
                    if (cudaMalloc((void **)&m.csr.Ar, (a.rows() + 1) * sizeof(std::int64_t)) != cudaSuccess ||
                            cudaMalloc((void **)&m.csr.Aj, (nb > 0 ? nb : 1) * sizeof(std::int32_t)) != cudaSuccess ||
                            cudaMalloc(&m.csr.Ax, (nb > 0 ? nb * bs : 1) * sizeof(DT_)) != cudaSuccess)
                    {
                        cudaGetLastError();
                        free_csr(m.csr);
                        st = HB_ERR_ALLOC;
                    }
                }
                if (! st)
                {
                    m.csr.rows = a.rows();
                    m.csr.cols = a.columns();
                    m.csr.blocksize = bs;
                    m.csr.nblocks = nb;
                    m.csr.dtype = dtype_of<DT_>();
                    m.csr.pad_ = 0;
                    st = sizeof(DT_) == 8
                        ? hb_csr_import_f64(context(), (const uint64_t *)ar, (const uint64_t *)aj, (const double *)ax, &m.csr)
                        : hb_csr_import_f32(context(), (const uint64_t *)ar, (const uint64_t *)aj, (const float *)ax, &m.csr);
                }
                m.gen[0] = g0; m.gen[1] = g1; m.gen[2] = g2;
                m.dev[0] = ar; m.dev[1] = aj; m.dev[2] = ax;
                if (st) m.gen[0] = 0;
            }
            a.Ar().unlock(lm_read_only);
            a.Aj().unlock(lm_read_only);
            a.Ax().unlock(lm_read_only);
            check(st, "SparseMatrixCSR device mirror");
            return m.csr;
        }

        template <typename DT_> const hb_ell & device_mirror(const SparseMatrixELL<DT_> & a)
        {
            // The backend's copies of the three reference arrays (uploaded on first lock).
            void * aj(a.Aj().lock(lm_read_only, tags::GPU::CUDA::memory_value));
            void * ax(a.Ax().lock(lm_read_only, tags::GPU::CUDA::memory_value));
            void * arl(a.Arl().lock(lm_read_only, tags::GPU::CUDA::memory_value));
            const std::uint64_t g0(generation(a.Aj().memid(), a.Aj().address()));
            const std::uint64_t g1(generation(a.Ax().memid(), a.Ax().address()));
            const std::uint64_t g2(generation(a.Arl().memid(), a.Arl().address()));
            std::lock_guard<std::mutex> l(g_mirror_mutex);
            Mirror & m(g_mirrors[a.Ax().memid()]);
            int st(HB_OK);
            if (! m.ell.Aj || m.gen[0] != g0 || m.gen[1] != g1 || m.gen[2] != g2 || m.Aj_dev[0] != aj
                    || m.Aj_dev[1] != ax || m.Aj_dev[2] != arl)
            {
                int64_t K, ld;
                st = hb_ell_layout(a.rows(), a.num_cols_per_row(), a.threads(), &K, &ld);
                if (! st && (! m.ell.Aj || m.ell.K != K || m.ell.ld != ld))
                {
                    cudaFree(m.ell.Aj);
                    cudaFree(m.ell.Ax);
                    m.ell.Aj = nullptr;
                    m.ell.Ax = nullptr;
                    if (cudaMalloc((void **)&m.ell.Aj, K * ld * sizeof(int32_t)) != cudaSuccess ||
                            cudaMalloc(&m.ell.Ax, K * ld * sizeof(DT_)) != cudaSuccess)
                    {
                        cudaGetLastError();
                        st = HB_ERR_ALLOC;
                    }
                }
                if (! st)
                {
                    m.ell.K = K;
                    m.ell.ld = ld;
                    m.ell.dtype = dtype_of<DT_>();
                    st = import(a, aj, ax, arl, m.ell);
                }
                m.gen[0] = g0; m.gen[1] = g1; m.gen[2] = g2;
                m.Aj_dev[0] = aj; m.Aj_dev[1] = ax; m.Aj_dev[2] = arl;
                if (st) m.gen[0] = 0;
            }
            a.Aj().unlock(lm_read_only);
            a.Ax().unlock(lm_read_only);
            a.Arl().unlock(lm_read_only);
            check(st, "SparseMatrixELL device mirror");
            return m.ell;
        }

        template const hb_ell & device_mirror<double>(const SparseMatrixELL<double> &);
        template const hb_ell & device_mirror<float>(const SparseMatrixELL<float> &);

        // RAII lock of a vector for the GPU tag.
        template <typename V_> struct DeviceLock
        {
            const V_ & v;
            LockMode mode;
            void * ptr;
            DeviceLock(const V_ & vv, LockMode m) : v(vv), mode(m), ptr(vv.lock(m, tags::GPU::CUDA::memory_value)) {}
            ~DeviceLock() { v.unlock(mode); }
        };

        template <typename DT_> void same_size(const DenseVectorContinuousBase<DT_> & a, const DenseVectorContinuousBase<DT_> & b)
        {
            if (a.size() != b.size())
                throw VectorSizeDoesNotMatch(b.size(), a.size());
        }

        /// Sets the block size of a kernel family on this thread's context from a honeirc key.
        hb_context * configured(int family, const char * key)
        {
            hb_context * ctx(context());
            int v(Configuration::instance()->get_value(key, 128));
            const int max(family == HB_BLOCK_VECTOR ? 1024 : 256);
            v = v < 32 ? 32 : (v > max ? max : v);
            hb_set_block_size(ctx, family, v - v % 32);
            return ctx;
        }

        int spmv(const hb_ell & A, const double * x, double * y)
        { return hb_spmv_f64(configured(HB_BLOCK_ELL, "cuda::product_smell_dv_double"), &A, x, y); }
        int spmv(const hb_ell & A, const float * x, float * y)
        { return hb_spmv_f32(configured(HB_BLOCK_ELL, "cuda::product_smell_dv_float"), &A, x, y); }
        int defect(const hb_ell & A, const double * b, const double * x, double * r)
        { return hb_defect_f64(configured(HB_BLOCK_ELL, "cuda::product_smell_dv_double"), &A, b, x, r); }
        int defect(const hb_ell & A, const float * b, const float * x, float * r)
        { return hb_defect_f32(configured(HB_BLOCK_ELL, "cuda::product_smell_dv_float"), &A, b, x, r); }
        int dot(int64_t n, const double * x, const double * y, double * out) { return hb_dot_f64(context(), n, x, y, out); }
        int dot(int64_t n, const float * x, const float * y, float * out) { return hb_dot_f32(context(), n, x, y, out); }
        int norm(int64_t n, const double * x, int root, double * out) { return hb_norm_l2_f64(context(), n, x, root, out); }
        int norm(int64_t n, const float * x, int root, float * out) { return hb_norm_l2_f32(context(), n, x, root, out); }
        int axpy(int64_t n, double * x, const double * y, double b) { return hb_scaled_sum_f64(configured(HB_BLOCK_VECTOR, "cuda::scaled_sum_two_double"), n, x, y, b); }
        int axpy(int64_t n, float * x, const float * y, float b) { return hb_scaled_sum_f32(configured(HB_BLOCK_VECTOR, "cuda::scaled_sum_two_float"), n, x, y, b); }
        int axpy3(int64_t n, double * r, const double * x, const double * y, double b) { return hb_scaled_sum3_f64(configured(HB_BLOCK_VECTOR, "cuda::scaled_sum_three_double"), n, r, x, y, b); }
        int axpy3(int64_t n, float * r, const float * x, const float * y, float b) { return hb_scaled_sum3_f32(configured(HB_BLOCK_VECTOR, "cuda::scaled_sum_three_float"), n, r, x, y, b); }
        int scale(int64_t n, double * x, double a) { return hb_scale_f64(configured(HB_BLOCK_VECTOR, "cuda::scale_one_double"), n, x, a); }
        int scale(int64_t n, float * x, float a) { return hb_scale_f32(configured(HB_BLOCK_VECTOR, "cuda::scale_one_float"), n, x, a); }
        int sum(int64_t n, double * x, const double * y) { return hb_sum_f64(configured(HB_BLOCK_VECTOR, "cuda::sum_two_double"), n, x, y); }
        int sum(int64_t n, float * x, const float * y) { return hb_sum_f32(configured(HB_BLOCK_VECTOR, "cuda::sum_two_float"), n, x, y); }
        int diff(int64_t n, double * r, const double * x, const double * y) { return hb_difference_f64(configured(HB_BLOCK_VECTOR, "cuda::difference_two_double"), n, r, x, y); }
        int diff(int64_t n, float * r, const float * x, const float * y) { return hb_difference_f32(configured(HB_BLOCK_VECTOR, "cuda::difference_two_float"), n, r, x, y); }
        int eprod(int64_t n, double * r, const double * x, const double * y) { return hb_element_product_f64(configured(HB_BLOCK_VECTOR, "cuda::element_product_two_double"), n, r, x, y); }
        int eprod(int64_t n, float * r, const float * x, const float * y) { return hb_element_product_f32(configured(HB_BLOCK_VECTOR, "cuda::element_product_two_float"), n, r, x, y); }

        int q1_spmv(const hb_q1band & A, const double * x, double * y) { return hb_q1band_spmv_f64(configured(HB_BLOCK_Q1BAND, "cuda::product_bmdv_q1_double"), &A, x, y); }
        int q1_spmv(const hb_q1band & A, const float * x, float * y) { return hb_q1band_spmv_f32(configured(HB_BLOCK_Q1BAND, "cuda::product_bmdv_q1_float"), &A, x, y); }
        int q1_defect(const hb_q1band & A, const double * b, const double * x, double * r)
        { return hb_q1band_defect_f64(configured(HB_BLOCK_Q1BAND, "cuda::product_bmdv_q1_double"), &A, b, x, r); }
        int q1_defect(const hb_q1band & A, const float * b, const float * x, float * r)
        { return hb_q1band_defect_f32(configured(HB_BLOCK_Q1BAND, "cuda::product_bmdv_q1_float"), &A, b, x, r); }

        /// The nine bands of a BandedMatrixQx locked for the GPU tag (the MemoryArbiter uploads
        /// them on first use and keeps them resident), as an hb_q1band.
        template <typename DT_> struct BandLocks
        {
            const BandedMatrixQx<Q1Type, DT_> & a;
            hb_q1band s;
            BandLocks(const BandedMatrixQx<Q1Type, DT_> & aa) : a(aa)
            {
                s.n = (int64_t)a.size();
                s.root = hb_q1band_root(s.n);
                s.dtype = sizeof(DT_) == 8 ? HB_F64 : HB_F32;
                s.pad_ = 0;
                for (unsigned long k(0) ; k < 9 ; ++k)
                    s.band[k] = a.band(k).lock(lm_read_only, tags::GPU::CUDA::memory_value);
            }
            ~BandLocks()
            {
                for (unsigned long k(0) ; k < 9 ; ++k) a.band(k).unlock(lm_read_only);
            }
        };

        template <typename DT_>
        void product(DenseVectorContinuousBase<DT_> & result, const BandedMatrixQx<Q1Type, DT_> & a,
                const DenseVectorContinuousBase<DT_> & b)
        {
            if (b.size() != a.columns())
                throw VectorSizeDoesNotMatch(b.size(), a.columns());
            if (a.rows() != result.size())
                throw VectorSizeDoesNotMatch(a.rows(), result.size());
            BandLocks<DT_> A(a);
            DeviceLock<DenseVectorContinuousBase<DT_> > x(b, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > y(result, lm_write_only);
            check(q1_spmv(A.s, (const DT_ *)x.ptr, (DT_ *)y.ptr), "Product<GPU::CUDA> (BandedMatrixQx)");
        }

        template <typename DT_>
        void defect(DenseVectorContinuousBase<DT_> & result, const DenseVectorContinuousBase<DT_> & rhs,
                const BandedMatrixQx<Q1Type, DT_> & a, const DenseVectorContinuousBase<DT_> & x)
        {
            if (x.size() != a.columns())
                throw VectorSizeDoesNotMatch(x.size(), a.columns());
            if (rhs.size() != a.columns())
                throw VectorSizeDoesNotMatch(rhs.size(), a.columns());
            if (result.size() != a.rows())
                throw VectorSizeDoesNotMatch(result.size(), a.rows());
            BandLocks<DT_> A(a);
            DeviceLock<DenseVectorContinuousBase<DT_> > xl(x, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > bl(rhs, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > rl(result, lm_write_only);
            check(q1_defect(A.s, (const DT_ *)bl.ptr, (const DT_ *)xl.ptr, (DT_ *)rl.ptr),
                    "Defect<GPU::CUDA> (BandedMatrixQx)");
        }

        int csr_spmv(const hb_csr & A, const double * x, double * y) { return hb_csr_spmv_f64(context(), &A, x, y); }
        int csr_spmv(const hb_csr & A, const float * x, float * y) { return hb_csr_spmv_f32(context(), &A, x, y); }
        int csr_defect(const hb_csr & A, const double * b, const double * x, double * r)
        { return hb_csr_defect_f64(context(), &A, b, x, r); }
        int csr_defect(const hb_csr & A, const float * b, const float * x, float * r)
        { return hb_csr_defect_f32(context(), &A, b, x, r); }

        template <typename DT_>
        void product(DenseVectorContinuousBase<DT_> & result, const SparseMatrixCSR<DT_> & a, const DenseVectorContinuousBase<DT_> & b)
        {
            if (b.size() != a.columns())
                throw VectorSizeDoesNotMatch(b.size(), a.columns());
            if (a.rows() != result.size())
                throw VectorSizeDoesNotMatch(a.rows(), result.size());
            const hb_csr & A(device_mirror(a));
            DeviceLock<DenseVectorContinuousBase<DT_> > x(b, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > y(result, lm_write_only);
            check(csr_spmv(A, (const DT_ *)x.ptr, (DT_ *)y.ptr), "Product<GPU::CUDA> (CSR)");
        }

        template <typename DT_>
        void defect(DenseVectorContinuousBase<DT_> & result, const DenseVectorContinuousBase<DT_> & rhs,
                const SparseMatrixCSR<DT_> & a, const DenseVectorContinuousBase<DT_> & x)
        {
            if (x.size() != a.columns())
                throw VectorSizeDoesNotMatch(x.size(), a.columns());
            if (rhs.size() != a.rows())
                throw VectorSizeDoesNotMatch(rhs.size(), a.rows());
            if (result.size() != a.rows())
                throw VectorSizeDoesNotMatch(result.size(), a.rows());
            const hb_csr & A(device_mirror(a));
            DeviceLock<DenseVectorContinuousBase<DT_> > xl(x, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > bl(rhs, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > rl(result, lm_write_only);
            check(csr_defect(A, (const DT_ *)bl.ptr, (const DT_ *)xl.ptr, (DT_ *)rl.ptr), "Defect<GPU::CUDA> (CSR)");
        }

        template <typename DT_>
        void product(DenseVectorContinuousBase<DT_> & result, const SparseMatrixELL<DT_> & a, const DenseVectorContinuousBase<DT_> & b)
        {
            if (b.size() != a.columns())
                throw VectorSizeDoesNotMatch(b.size(), a.columns());
            if (a.rows() != result.size())
                throw VectorSizeDoesNotMatch(a.rows(), result.size());
            const hb_ell & A(device_mirror(a));
            DeviceLock<DenseVectorContinuousBase<DT_> > x(b, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > y(result, lm_write_only);
            check(spmv(A, (const DT_ *)x.ptr, (DT_ *)y.ptr), "Product<GPU::CUDA> (ELL)");
        }

        template <typename DT_>
        void defect(DenseVectorContinuousBase<DT_> & result, const DenseVectorContinuousBase<DT_> & rhs,
                const SparseMatrixELL<DT_> & a, const DenseVectorContinuousBase<DT_> & x)
        {
            if (x.size() != a.columns())
                throw VectorSizeDoesNotMatch(x.size(), a.columns());
            if (rhs.size() != a.columns())
                throw VectorSizeDoesNotMatch(rhs.size(), a.columns());
            if (result.size() != a.rows())
                throw VectorSizeDoesNotMatch(result.size(), a.rows());
            const hb_ell & A(device_mirror(a));
            DeviceLock<DenseVectorContinuousBase<DT_> > xl(x, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > bl(rhs, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > rl(result, lm_write_only);
            check(b200::defect(A, (const DT_ *)bl.ptr, (const DT_ *)xl.ptr, (DT_ *)rl.ptr), "Defect<GPU::CUDA> (ELL)");
        }
        int spai2_call(const hb_ell & A, hb_ell & M, double) { return hb_spai2_f64(context(), &A, &M); }
        int spai2_call(const hb_ell & A, hb_ell & M, float) { return hb_spai2_f32(context(), &A, &M); }

        /// SPAI2<tags::GPU::CUDA> on host SparseMatrix containers, as the reference's wrapper
        /// (honei/math/spai2-cuda.cc:180-228): M = A.copy(), the values computed on the device
        /// from A's ELL form (SparseMatrixELL(SparseMatrix), whose device mirror the arbiter
        /// uploads), then written into M entry by entry.
        template <typename DT_> SparseMatrix<DT_> & spai2(SparseMatrix<DT_> & M, const SparseMatrix<DT_> & a)
        {
            if (a.rows() != a.columns())
                throw MatrixIsNotSquare(a.rows(), a.columns());
            M = a.copy();
            SparseMatrixELL<DT_> e(a);
            const hb_ell & A(device_mirror(e));
            const std::size_t slots(A.K * A.ld);
            hb_ell Md(A);
            Md.Aj = nullptr;
            Md.Ax = nullptr;
            std::vector<int32_t> aj(slots);
            std::vector<DT_> ax(slots);
            int st(HB_OK);
            if (cudaMalloc((void **)&Md.Aj, slots * sizeof(int32_t)) != cudaSuccess ||
                    cudaMalloc(&Md.Ax, slots * sizeof(DT_)) != cudaSuccess)
            {
                cudaGetLastError();
                st = HB_ERR_ALLOC;
            }
            if (! st)
                st = spai2_call(A, Md, DT_(0));
            if (! st)
                st = hb_synchronize(context());
            if (! st && (cudaMemcpy(aj.data(), Md.Aj, slots * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(ax.data(), Md.Ax, slots * sizeof(DT_), cudaMemcpyDeviceToHost) != cudaSuccess))
            {
                cudaGetLastError();
                st = HB_ERR_CUDA;
            }
            cudaFree(Md.Aj);
            cudaFree(Md.Ax);
            check(st, "SPAI2<GPU::CUDA>");
            for (int64_t r(0) ; r < A.rows ; ++r)
                for (int64_t k(0) ; k < A.K ; ++k)
                {
                    const int32_t c(aj[k * A.ld + r]);
                    if (c >= 0)
                        M(r, c, ax[k * A.ld + r]);
                }
            return M;
        }
    }

    using namespace b200;

    // ---- Product ------------------------------------------------------------------------
    DenseVector<float> & Product<tags::GPU::CUDA>::value(DenseVector<float> & result, const SparseMatrixELL<float> & a,
            const DenseVector<float> & b)
    {
        CONTEXT("When multiplying SparseMatrixELL<float> with DenseVector<float> (B200):");
        b200::product<float>(result, a, b);
        return result;
    }

    DenseVector<double> & Product<tags::GPU::CUDA>::value(DenseVector<double> & result, const SparseMatrixELL<double> & a,
            const DenseVector<double> & b)
    {
        CONTEXT("When multiplying SparseMatrixELL<double> with DenseVector<double> (B200):");
        b200::product<double>(result, a, b);
        return result;
    }

    DenseVector<float> & Product<tags::GPU::CUDA>::value(DenseVector<float> & result, const SparseMatrixCSR<float> & a,
            const DenseVector<float> & b)
    {
        CONTEXT("When multiplying SparseMatrixCSR<float> with DenseVector<float> (B200):");
        b200::product<float>(result, a, b);
        return result;
    }

    DenseVector<double> & Product<tags::GPU::CUDA>::value(DenseVector<double> & result, const SparseMatrixCSR<double> & a,
            const DenseVector<double> & b)
    {
        CONTEXT("When multiplying SparseMatrixCSR<double> with DenseVector<double> (B200):");
        b200::product<double>(result, a, b);
        return result;
    }

    DenseVector<float> Product<tags::GPU::CUDA>::value(const BandedMatrixQx<Q1Type, float> & a,
            const DenseVectorContinuousBase<float> & b)
    {
        CONTEXT("When multiplying BandedMatrixQx<Q1Type, float> with DenseVector<float> (B200):");
        DenseVector<float> result(a.rows());
        b200::product<float>(result, a, b);
        return result;
    }

    DenseVector<double> Product<tags::GPU::CUDA>::value(const BandedMatrixQx<Q1Type, double> & a,
            const DenseVectorContinuousBase<double> & b)
    {
        CONTEXT("When multiplying BandedMatrixQx<Q1Type, double> with DenseVector<double> (B200):");
        DenseVector<double> result(a.rows());
        b200::product<double>(result, a, b);
        return result;
    }

    DenseVector<float> & Product<tags::GPU::CUDA>::value(DenseVector<float> & result,
            const BandedMatrixQx<Q1Type, float> & a, const DenseVectorContinuousBase<float> & b)
    {
        CONTEXT("When multiplying BandedMatrixQx<Q1Type, float> with DenseVector<float> (B200):");
        b200::product<float>(result, a, b);
        return result;
    }

    DenseVector<double> & Product<tags::GPU::CUDA>::value(DenseVector<double> & result,
            const BandedMatrixQx<Q1Type, double> & a, const DenseVectorContinuousBase<double> & b)
    {
        CONTEXT("When multiplying BandedMatrixQx<Q1Type, double> with DenseVector<double> (B200):");
        b200::product<double>(result, a, b);
        return result;
    }

    // ---- Defect -------------------------------------------------------------------------
    DenseVector<float> Defect<tags::GPU::CUDA>::value(const DenseVectorContinuousBase<float> & rhs,
            const BandedMatrixQx<Q1Type, float> & system, const DenseVectorContinuousBase<float> & x)
    {
        DenseVector<float> result(system.rows());
        b200::defect<float>(result, rhs, system, x);
        return result;
    }

    DenseVector<double> Defect<tags::GPU::CUDA>::value(const DenseVectorContinuousBase<double> & rhs,
            const BandedMatrixQx<Q1Type, double> & system, const DenseVectorContinuousBase<double> & x)
    {
        DenseVector<double> result(system.rows());
        b200::defect<double>(result, rhs, system, x);
        return result;
    }

    DenseVector<float> & Defect<tags::GPU::CUDA>::value(DenseVector<float> & result,
            const DenseVectorContinuousBase<float> & rhs, const BandedMatrixQx<Q1Type, float> & system,
            const DenseVectorContinuousBase<float> & x)
    {
        b200::defect<float>(result, rhs, system, x);
        return result;
    }

    DenseVector<double> & Defect<tags::GPU::CUDA>::value(DenseVector<double> & result,
            const DenseVectorContinuousBase<double> & rhs, const BandedMatrixQx<Q1Type, double> & system,
            const DenseVectorContinuousBase<double> & x)
    {
        b200::defect<double>(result, rhs, system, x);
        return result;
    }

    DenseVector<float> Defect<tags::GPU::CUDA>::value(const DenseVectorContinuousBase<float> & rhs,
            const SparseMatrixELL<float> & system, const DenseVectorContinuousBase<float> & x)
    {
        DenseVector<float> result(system.rows());
        b200::defect<float>(result, rhs, system, x);
        return result;
    }

    DenseVector<double> Defect<tags::GPU::CUDA>::value(const DenseVectorContinuousBase<double> & rhs,
            const SparseMatrixELL<double> & system, const DenseVectorContinuousBase<double> & x)
    {
        DenseVector<double> result(system.rows());
        b200::defect<double>(result, rhs, system, x);
        return result;
    }

    DenseVectorContinuousBase<float> & Defect<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & result,
            const DenseVectorContinuousBase<float> & rhs, const SparseMatrixELL<float> & system,
            const DenseVectorContinuousBase<float> & x)
    {
        b200::defect<float>(result, rhs, system, x);
        return result;
    }

    DenseVectorContinuousBase<double> & Defect<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & result,
            const DenseVectorContinuousBase<double> & rhs, const SparseMatrixELL<double> & system,
            const DenseVectorContinuousBase<double> & x)
    {
        b200::defect<double>(result, rhs, system, x);
        return result;
    }

    DenseVectorContinuousBase<float> & Defect<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & result,
            const DenseVectorContinuousBase<float> & rhs, const SparseMatrixCSR<float> & system,
            const DenseVectorContinuousBase<float> & x)
    {
        b200::defect<float>(result, rhs, system, x);
        return result;
    }

    DenseVectorContinuousBase<double> & Defect<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & result,
            const DenseVectorContinuousBase<double> & rhs, const SparseMatrixCSR<double> & system,
            const DenseVectorContinuousBase<double> & x)
    {
        b200::defect<double>(result, rhs, system, x);
        return result;
    }

    // ---- DotProduct / Norm ----------------------------------------------------------------
    template <typename DT_> static DT_ b200_dot(const DenseVectorContinuousBase<DT_> & a, const DenseVectorContinuousBase<DT_> & b)
    {
        same_size(a, b);
        DeviceLock<DenseVectorContinuousBase<DT_> > x(a, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > y(b, lm_read_only);
        DT_ out(0);
        check(dot((int64_t)a.size(), (const DT_ *)x.ptr, (const DT_ *)y.ptr, &out), "DotProduct<GPU::CUDA>");
        return out;
    }

    float DotProduct<tags::GPU::CUDA>::value(const DenseVectorContinuousBase<float> & a, const DenseVectorContinuousBase<float> & b)
    { return b200_dot<float>(a, b); }
    double DotProduct<tags::GPU::CUDA>::value(const DenseVectorContinuousBase<double> & a, const DenseVectorContinuousBase<double> & b)
    { return b200_dot<double>(a, b); }

    template <typename DT_> static DT_ b200_norm(const DenseVectorContinuousBase<DT_> & a, int root)
    {
        DeviceLock<DenseVectorContinuousBase<DT_> > x(a, lm_read_only);
        DT_ out(0);
        check(norm((int64_t)a.size(), (const DT_ *)x.ptr, root, &out), "Norm<vnt_l_two, GPU::CUDA>");
        return out;
    }

    float Norm<vnt_l_two, false, tags::GPU::CUDA>::value(const DenseVectorContinuousBase<float> & x) { return b200_norm<float>(x, 0); }
    double Norm<vnt_l_two, false, tags::GPU::CUDA>::value(const DenseVectorContinuousBase<double> & x) { return b200_norm<double>(x, 0); }
    float Norm<vnt_l_two, true, tags::GPU::CUDA>::value(const DenseVectorContinuousBase<float> & x) { return b200_norm<float>(x, 1); }
    double Norm<vnt_l_two, true, tags::GPU::CUDA>::value(const DenseVectorContinuousBase<double> & x) { return b200_norm<double>(x, 1); }

    // ---- ScaledSum ------------------------------------------------------------------------
    template <typename DT_> static void b200_axpy(DenseVectorContinuousBase<DT_> & x, const DenseVectorContinuousBase<DT_> & y, DT_ b)
    {
        same_size(x, y);
        DeviceLock<DenseVectorContinuousBase<DT_> > yl(y, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > xl(x, lm_read_and_write);
        check(axpy((int64_t)x.size(), (DT_ *)xl.ptr, (const DT_ *)yl.ptr, b), "ScaledSum<GPU::CUDA>");
    }

    template <typename DT_> static void b200_axpy3(DenseVectorContinuousBase<DT_> & r, const DenseVectorContinuousBase<DT_> & x,
            const DenseVectorContinuousBase<DT_> & y, DT_ b)
    {
        same_size(x, y);
        same_size(x, r);
        DeviceLock<DenseVectorContinuousBase<DT_> > xl(x, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > yl(y, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > rl(r, lm_write_only);
        check(axpy3((int64_t)x.size(), (DT_ *)rl.ptr, (const DT_ *)xl.ptr, (const DT_ *)yl.ptr, b), "ScaledSum<GPU::CUDA>");
    }

    DenseVectorContinuousBase<float> & ScaledSum<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & x,
            const DenseVectorContinuousBase<float> & y, float b)
    { b200_axpy<float>(x, y, b); return x; }
    DenseVectorContinuousBase<double> & ScaledSum<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & x,
            const DenseVectorContinuousBase<double> & y, double b)
    { b200_axpy<double>(x, y, b); return x; }
    DenseVectorContinuousBase<float> & ScaledSum<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & r,
            const DenseVectorContinuousBase<float> & x, const DenseVectorContinuousBase<float> & y, float b)
    { b200_axpy3<float>(r, x, y, b); return r; }
    DenseVectorContinuousBase<double> & ScaledSum<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & r,
            const DenseVectorContinuousBase<double> & x, const DenseVectorContinuousBase<double> & y, double b)
    { b200_axpy3<double>(r, x, y, b); return r; }

    // ---- Scale / Sum / Difference / ElementProduct ------------------------------------------
    DenseVectorContinuousBase<float> & Scale<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & x, const float a)
    {
        DeviceLock<DenseVectorContinuousBase<float> > xl(x, lm_read_and_write);
        check(scale((int64_t)x.size(), (float *)xl.ptr, a), "Scale<GPU::CUDA>");
        return x;
    }

    DenseVectorContinuousBase<double> & Scale<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & x, const double a)
    {
        DeviceLock<DenseVectorContinuousBase<double> > xl(x, lm_read_and_write);
        check(scale((int64_t)x.size(), (double *)xl.ptr, a), "Scale<GPU::CUDA>");
        return x;
    }

    template <typename DT_> static void b200_sum(DenseVectorContinuousBase<DT_> & a, const DenseVectorContinuousBase<DT_> & b)
    {
        same_size(a, b);
        DeviceLock<DenseVectorContinuousBase<DT_> > bl(b, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > al(a, lm_read_and_write);
        check(sum((int64_t)a.size(), (DT_ *)al.ptr, (const DT_ *)bl.ptr), "Sum<GPU::CUDA>");
    }

    DenseVectorContinuousBase<float> & Sum<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & a,
            const DenseVectorContinuousBase<float> & b)
    { b200_sum<float>(a, b); return a; }
    DenseVectorContinuousBase<double> & Sum<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & a,
            const DenseVectorContinuousBase<double> & b)
    { b200_sum<double>(a, b); return a; }

    template <typename DT_> static void b200_diff(DenseVectorContinuousBase<DT_> & r, const DenseVectorContinuousBase<DT_> & a,
            const DenseVectorContinuousBase<DT_> & b)
    {
        same_size(a, b);
        same_size(a, r);
        if (&r == &a)
        {
            DeviceLock<DenseVectorContinuousBase<DT_> > bl(b, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > al(a, lm_read_and_write);
            check(diff((int64_t)a.size(), (DT_ *)al.ptr, (const DT_ *)al.ptr, (const DT_ *)bl.ptr), "Difference<GPU::CUDA>");
            return;
        }
        DeviceLock<DenseVectorContinuousBase<DT_> > al(a, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > bl(b, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > rl(r, lm_write_only);
        check(diff((int64_t)a.size(), (DT_ *)rl.ptr, (const DT_ *)al.ptr, (const DT_ *)bl.ptr), "Difference<GPU::CUDA>");
    }

    DenseVectorContinuousBase<float> & Difference<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & a,
            const DenseVectorContinuousBase<float> & b)
    { b200_diff<float>(a, a, b); return a; }
    DenseVectorContinuousBase<double> & Difference<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & a,
            const DenseVectorContinuousBase<double> & b)
    { b200_diff<double>(a, a, b); return a; }
    DenseVectorContinuousBase<float> & Difference<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & r,
            const DenseVectorContinuousBase<float> & a, const DenseVectorContinuousBase<float> & b)
    { b200_diff<float>(r, a, b); return r; }
    DenseVectorContinuousBase<double> & Difference<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & r,
            const DenseVectorContinuousBase<double> & a, const DenseVectorContinuousBase<double> & b)
    { b200_diff<double>(r, a, b); return r; }

    template <typename DT_> static void b200_eprod(DenseVectorContinuousBase<DT_> & r, const DenseVectorContinuousBase<DT_> & a,
            const DenseVectorContinuousBase<DT_> & b)
    {
        same_size(a, b);
        same_size(a, r);
        if (&r == &a)
        {
            DeviceLock<DenseVectorContinuousBase<DT_> > bl(b, lm_read_only);
            DeviceLock<DenseVectorContinuousBase<DT_> > al(a, lm_read_and_write);
            check(eprod((int64_t)a.size(), (DT_ *)al.ptr, (const DT_ *)al.ptr, (const DT_ *)bl.ptr), "ElementProduct<GPU::CUDA>");
            return;
        }
        DeviceLock<DenseVectorContinuousBase<DT_> > al(a, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > bl(b, lm_read_only);
        DeviceLock<DenseVectorContinuousBase<DT_> > rl(r, lm_write_only);
        check(eprod((int64_t)a.size(), (DT_ *)rl.ptr, (const DT_ *)al.ptr, (const DT_ *)bl.ptr), "ElementProduct<GPU::CUDA>");
    }

    DenseVectorContinuousBase<float> & ElementProduct<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & a,
            const DenseVectorContinuousBase<float> & b)
    { b200_eprod<float>(a, a, b); return a; }
    DenseVectorContinuousBase<double> & ElementProduct<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & a,
            const DenseVectorContinuousBase<double> & b)
    { b200_eprod<double>(a, a, b); return a; }
    DenseVectorContinuousBase<float> & ElementProduct<tags::GPU::CUDA>::value(DenseVectorContinuousBase<float> & r,
            const DenseVectorContinuousBase<float> & a, const DenseVectorContinuousBase<float> & b)
    { b200_eprod<float>(r, a, b); return r; }
    DenseVectorContinuousBase<double> & ElementProduct<tags::GPU::CUDA>::value(DenseVectorContinuousBase<double> & r,
            const DenseVectorContinuousBase<double> & a, const DenseVectorContinuousBase<double> & b)
    { b200_eprod<double>(r, a, b); return r; }
}

namespace honei
{
    // ---- SPAI2 ---------------------------------------------------------------------------
    SparseMatrix<float> & SPAI2<tags::GPU::CUDA>::value(SparseMatrix<float> & M, const SparseMatrix<float> & A)
    {
        CONTEXT("When calculating SPAI2<float> (B200):");
        return b200::spai2<float>(M, A);
    }

    SparseMatrix<double> & SPAI2<tags::GPU::CUDA>::value(SparseMatrix<double> & M, const SparseMatrix<double> & A)
    {
        CONTEXT("When calculating SPAI2<double> (B200):");
        return b200::spai2<double>(M, A);
    }
}
