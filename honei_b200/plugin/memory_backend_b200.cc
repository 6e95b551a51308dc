/* memory_backend_b200.cc -- MemoryBackend<tags::GPU::CUDA> for the B200 backend.
 *
 * Implements the interface HONEI declares in honei/util/memory_backend.hh:131-165 (and the
 * contract MemoryArbiter relies on, honei/util/memory_arbiter-impl.hh:404-512): upload returns
 * the device copy of a block, creating and filling it only when this backend holds none (the
 * arbiter frees stale copies itself before it asks for a writable one); alloc creates without
 * copying; download copies back; copy / convert / fill work device-side through the C ABI.
 * Blocks are keyed by (memid, address) so ranges of one vector get their own device copies.
 * Every (re)upload bumps a generation counter, which the SparseMatrixELL mirror cache uses to
 * notice that a matrix changed on the host.
 */
#include "b200_backend.hh"

#include <honei/util/instantiation_policy-impl.hh>
#include <honei/util/memory_arbiter.hh>
#include <honei/util/memory_backend.hh>
#include <honei/util/private_implementation_pattern-impl.hh>

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace honei
{
    template <> struct Implementation<MemoryBackend<tags::GPU::CUDA> >
    {
        struct Block
        {
            void * device;
            unsigned long bytes;
            std::uint64_t generation;
        };

        std::map<std::pair<void *, void *>, Block> blocks;
        std::recursive_mutex mutex;
        std::uint64_t next_generation = 1;

        Block * find(void * memid, void * address)
        {
            auto i(blocks.find(std::make_pair(memid, address)));
            return i == blocks.end() ? nullptr : &i->second;
        }

        Block & get(void * memid, void * address, unsigned long bytes)
        {
            Block * b(find(memid, address));
            if (b && b->bytes >= bytes)
                return *b;
            if (b)
            {
                cudaFree(b->device);
                blocks.erase(std::make_pair(memid, address));
            }
            void * d(nullptr);
            if (cudaMalloc(&d, bytes ? bytes : 1) != cudaSuccess)
            {
                cudaGetLastError();
                throw InternalError("MemoryBackend<GPU::CUDA>: cudaMalloc of " + std::to_string(bytes) + " bytes failed");
            }
            Block & nb(blocks[std::make_pair(memid, address)]);
            nb.device = d;
            nb.bytes = bytes;
            nb.generation = next_generation++;
            return nb;
        }
    };

    template class InstantiationPolicy<MemoryBackend<tags::GPU::CUDA>, Singleton>;

    namespace
    {
        // The singleton's implementation, for the b200:: queries below (_imp is protected).
        Implementation<MemoryBackend<tags::GPU::CUDA> > * g_backend_imp = nullptr;
    }

    MemoryBackend<tags::GPU::CUDA>::MemoryBackend() :
        PrivateImplementationPattern<MemoryBackend<tags::GPU::CUDA>, Single>(new Implementation<MemoryBackend<tags::GPU::CUDA> >)
    {
        g_backend_imp = _imp;
    }

    MemoryBackend<tags::GPU::CUDA>::~MemoryBackend()
    {
        for (auto & kv : _imp->blocks)
            cudaFree(kv.second.device);
        g_backend_imp = nullptr;
    }

    void * MemoryBackend<tags::GPU::CUDA>::upload(void * memid, void * address, unsigned long bytes)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        Implementation<MemoryBackend<tags::GPU::CUDA> >::Block * b(_imp->find(memid, address));
        if (b && b->bytes >= bytes)
            return b->device;
        Implementation<MemoryBackend<tags::GPU::CUDA> >::Block & nb(_imp->get(memid, address, bytes));
        if (bytes && cudaMemcpy(nb.device, address, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        {
            cudaGetLastError();
            throw InternalError("MemoryBackend<GPU::CUDA>::upload: cudaMemcpy failed");
        }
        nb.generation = _imp->next_generation++;
        return nb.device;
    }

    void MemoryBackend<tags::GPU::CUDA>::download(void * memid, void * address, unsigned long bytes)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        Implementation<MemoryBackend<tags::GPU::CUDA> >::Block * b(_imp->find(memid, address));
        if (! b)
            throw InternalError("MemoryBackend<GPU::CUDA>::download: unknown memory block");
        if (bytes && cudaMemcpy(address, b->device, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        {
            cudaGetLastError();
            throw InternalError("MemoryBackend<GPU::CUDA>::download: cudaMemcpy failed");
        }
    }

    void * MemoryBackend<tags::GPU::CUDA>::alloc(void * memid, void * address, unsigned long bytes)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        Implementation<MemoryBackend<tags::GPU::CUDA> >::Block & b(_imp->get(memid, address, bytes));
        b.generation = _imp->next_generation++;
        return b.device;
    }

    void MemoryBackend<tags::GPU::CUDA>::free(void * memid)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        b200::forget(memid);
        for (auto i(_imp->blocks.begin()) ; i != _imp->blocks.end() ; )
        {
            if (i->first.first == memid)
            {
                cudaFree(i->second.device);
                i = _imp->blocks.erase(i);
            }
            else
                ++i;
        }
    }

    void MemoryBackend<tags::GPU::CUDA>::copy(void * src_id, void * src_address, void * dest_id,
            void * dest_address, unsigned long bytes)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        void * src(upload(src_id, src_address, bytes));
        void * dst(alloc(dest_id, dest_address, bytes));
        b200::check(hb_copy(b200::context(), dst, src, (int64_t)bytes), "MemoryBackend<GPU::CUDA>::copy");
    }

    void MemoryBackend<tags::GPU::CUDA>::convert_float_double(void * src_id, void * src_address, void * dest_id,
            void * dest_address, unsigned long bytes)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        void * src(upload(src_id, src_address, bytes));
        void * dst(alloc(dest_id, dest_address, bytes * 2));
        b200::check(hb_convert_f32_f64(b200::context(), (int64_t)(bytes / sizeof(float)), (double *)dst,
                    (const float *)src), "MemoryBackend<GPU::CUDA>::convert_float_double");
    }

    void MemoryBackend<tags::GPU::CUDA>::convert_double_float(void * src_id, void * src_address, void * dest_id,
            void * dest_address, unsigned long bytes)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        void * src(upload(src_id, src_address, bytes));
        void * dst(alloc(dest_id, dest_address, bytes / 2));
        b200::check(hb_convert_f64_f32(b200::context(), (int64_t)(bytes / sizeof(double)), (float *)dst,
                    (const double *)src), "MemoryBackend<GPU::CUDA>::convert_double_float");
    }

    void MemoryBackend<tags::GPU::CUDA>::fill(void * memid, void * address, unsigned long bytes, float proto)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        void * d(alloc(memid, address, bytes));
        b200::check(hb_fill_f32(b200::context(), (int64_t)(bytes / sizeof(float)), (float *)d, proto),
                "MemoryBackend<GPU::CUDA>::fill");
    }

    void MemoryBackend<tags::GPU::CUDA>::fill(void * memid, void * address, unsigned long bytes, double proto)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        void * d(alloc(memid, address, bytes));
        b200::check(hb_fill_f64(b200::context(), (int64_t)(bytes / sizeof(double)), (double *)d, proto),
                "MemoryBackend<GPU::CUDA>::fill");
    }

    bool MemoryBackend<tags::GPU::CUDA>::knows(void * memid, void * address)
    {
        std::lock_guard<std::recursive_mutex> l(_imp->mutex);
        return _imp->find(memid, address) != nullptr;
    }

    namespace b200
    {
        void * device_address(void * memid, void * address)
        {
            MemoryBackend<tags::GPU::CUDA>::instance();
            Implementation<MemoryBackend<tags::GPU::CUDA> > & imp(*g_backend_imp);
            std::lock_guard<std::recursive_mutex> l(imp.mutex);
            Implementation<MemoryBackend<tags::GPU::CUDA> >::Block * b(imp.find(memid, address));
            return b ? b->device : nullptr;
        }

        std::uint64_t generation(void * memid, void * address)
        {
            MemoryBackend<tags::GPU::CUDA>::instance();
            Implementation<MemoryBackend<tags::GPU::CUDA> > & imp(*g_backend_imp);
            std::lock_guard<std::recursive_mutex> l(imp.mutex);
            Implementation<MemoryBackend<tags::GPU::CUDA> >::Block * b(imp.find(memid, address));
            return b ? b->generation : 0;
        }
    }
}

using namespace honei;

static MemoryBackendRegistrator b200_gpu_cuda_registrator(tags::GPU::CUDA::memory_value,
        MemoryBackend<tags::GPU::CUDA>::instance());
