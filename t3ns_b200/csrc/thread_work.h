// Per-host-thread workspace of the synchronous host-array entry points (the
// decomposition's factorisations and the renormalised-operator updates): the
// thread's own stream, a device buffer and a pinned host staging buffer, kept
// between calls and grown (to at least twice their size) when a call needs
// more, so a call costs one upload, its launches, one download and one
// synchronisation instead of an allocation and a pageable copy per array.
// The buffers hold the largest call the thread has made; they are freed when
// the thread exits.  A call finishes (synchronises its stream) before it
// returns, so consecutive calls of one thread may share the buffers.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>

#include "common.h"

namespace t3ns {

struct ThreadWork {
        int device = -1;
        cudaStream_t st = nullptr;
        char *dev = nullptr, *host = nullptr;
        size_t dev_bytes = 0, host_bytes = 0;
        bool svd_smem_set = false;   // large dynamic shared memory enabled for the SVD kernel

        void release()
        {
                if (st) cudaStreamSynchronize(st);
                if (dev) cudaFree(dev);
                if (host) cudaFreeHost(host);
                if (st) cudaStreamDestroy(st);
                dev = host = nullptr;
                dev_bytes = host_bytes = 0;
                st = nullptr;
                svd_smem_set = false;
        }
        ~ThreadWork() { release(); }

        // the thread's stream, dbytes on the device and hbytes pinned on the host
        int reserve(size_t dbytes, size_t hbytes)
        {
                int d = 0;
                T3NS_CUDA_TRY(cudaGetDevice(&d));
                if (d != device) {
                        release();
                        device = d;
                }
                if (!st && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
                        st = nullptr;
                        return set_error(T3NS_E_CUDA, "workspace: stream creation failed");
                }
                // a previous call that returned early on an error may have left
                // copies in flight that still read or write the buffers: drain
                // the stream before the caller touches them again
                T3NS_CUDA_TRY(cudaStreamSynchronize(st));
                if (dbytes > dev_bytes) {
                        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
                        const size_t want = std::max(dbytes, 2 * dev_bytes);
                        if (dev) cudaFree(dev);
                        dev = nullptr;
                        dev_bytes = 0;
                        if (cudaMalloc(&dev, want) != cudaSuccess) {
                                cudaGetLastError();
                                dev = nullptr;
                                return set_error(T3NS_E_NOMEM, "workspace: device buffer");
                        }
                        dev_bytes = want;
                }
                if (hbytes > host_bytes) {
                        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
                        const size_t want = std::max(hbytes, 2 * host_bytes);
                        if (host) cudaFreeHost(host);
                        host = nullptr;
                        host_bytes = 0;
                        if (cudaMallocHost(&host, want) != cudaSuccess) {
                                cudaGetLastError();
                                host = nullptr;
                                return set_error(T3NS_E_NOMEM, "workspace: pinned staging buffer");
                        }
                        host_bytes = want;
                }
                return T3NS_OK;
        }
};

inline ThreadWork &thread_work()
{
        thread_local ThreadWork w;
        return w;
}

// Byte offsets of consecutive arrays in a buffer, each 256-byte aligned (an
// empty array still takes one element, so every array has its own address).
struct Carve {
        size_t off = 0;
        template <class T>
        size_t take(size_t n)
        {
                const size_t at = off;
                off += (sizeof(T) * std::max<size_t>(n, 1) + 255) & ~(size_t) 255;
                return at;
        }
};

}  // namespace t3ns
