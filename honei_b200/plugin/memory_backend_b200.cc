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
 *
 * Device buffers are recycled: free() (which the arbiter calls whenever the host writes a vector,
 * so every step of a host-side loop) returns a block's buffer to a size-keyed cache instead of
 * cudaFree, and the next block of a fitting size takes it instead of cudaMalloc.  cudaFree
 * synchronises the whole device and a large cudaMalloc costs milliseconds, once per step each.
 * The cache holds at most a quarter of the device's memory; a cudaMalloc that fails empties it
 * and tries again.  Reuse is ordered: every kernel of this backend runs on the legacy default
 * stream, as do the synchronous copies that refill a recycled buffer.
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
        std::multimap<unsigned long, void *> cache;     // recycled buffers by size
        unsigned long cached_bytes = 0;
        unsigned long cache_limit = 0;
        std::recursive_mutex mutex;
        std::uint64_t next_generation = 1;

        Block * find(void * memid, void * address)
        {
            auto i(blocks.find(std::make_pair(memid, address)));
            return i == blocks.end() ? nullptr : &i->second;
        }

        void release(void * device, unsigned long bytes)
        {
            if (! cache_limit)
            {
                std::size_t free_b(0), total_b(0);
                cudaMemGetInfo(&free_b, &total_b);
                cache_limit = total_b / 4 ? total_b / 4 : 1;
            }
            if (cached_bytes + bytes <= cache_limit)
            {
                cache.insert(std::make_pair(bytes, device));
                cached_bytes += bytes;
            }
            else
                cudaFree(device);
        }

        void drop_cache()
        {
            for (auto & kv : cache)
                cudaFree(kv.second);
            cache.clear();
            cached_bytes = 0;
        }

        /// A buffer of at least bytes: a recycled one of up to 5/4 of the size, else a new one.
        std::pair<void *, unsigned long> take(unsigned long bytes)
        {
            const unsigned long want(bytes ? bytes : 1);
            auto i(cache.lower_bound(want));
            if (i != cache.end() && i->first <= want + want / 4)
            {
                std::pair<void *, unsigned long> r(i->second, i->first);
                cached_bytes -= i->first;
                cache.erase(i);
                return r;
            }
            void * d(nullptr);
            if (cudaMalloc(&d, want) != cudaSuccess)
            {
                cudaGetLastError();
                drop_cache();
                if (cudaMalloc(&d, want) != cudaSuccess)
                {
                    cudaGetLastError();
                    throw InternalError("MemoryBackend<GPU::CUDA>: cudaMalloc of " + std::to_string(bytes) + " bytes failed");
                }
            }
            return std::make_pair(d, want);
        }

        Block & get(void * memid, void * address, unsigned long bytes)
        {
            Block * b(find(memid, address));
            if (b && b->bytes >= bytes)
                return *b;
            if (b)
            {
                release(b->device, b->bytes);
                blocks.erase(std::make_pair(memid, address));
            }
            const std::pair<void *, unsigned long> d(take(bytes));
            Block & nb(blocks[std::make_pair(memid, address)]);
            nb.device = d.first;
            nb.bytes = d.second;
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
        _imp->drop_cache();
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
                _imp->release(i->second.device, i->second.bytes);
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
