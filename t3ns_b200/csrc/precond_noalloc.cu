// Allocation-free variant of the Davidson diagonal preconditioner.
//
// Some callers of this library cannot allocate device memory at the point
// where they need the preconditioner: code running inside a memory pool or
// arena that owns all of the GPU's memory, code that must not synchronise the
// device (cudaMalloc/cudaFree can), and real-time or embedded drivers that
// forbid allocation after start-up.  For them this file provides
// t3ns_precondition_device_noalloc: the caller passes device buffers for the
// inputs and the output, and the only scratch the computation needs -- the
// per-chunk partial sums of the two reductions and the resulting Olsen
// coefficient -- lives in a fixed array in this library's device image.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library keeps it (about 1 MiB) until the process exits.  Host code cannot
// use the array's name as a device address; the first call on each device
// looks its address up with cudaGetSymbolAddress while that device is current
// and caches it.  Because that first call does this set-up, it should be made
// before any stream capture.  All calls share the one array: calls whose work
// overlaps on the GPU (different streams, or different host threads on the
// same device) race on it and must be serialised by the caller.  Every slot a
// call reads is written earlier by the same call, so the contents left by a
// previous call never leak into a result.
#include <mutex>

#include "common.h"

namespace t3ns {
namespace {

constexpr int kChunk = 256;                          // elements per partial sum
constexpr int kMaxChunks = 65536;                    // T3NS_NOALLOC_MAX_SIZE / kChunk
constexpr double kCutoff = 1e-12;                    // as davidson.c's DIAG_CUTOFF
static_assert((int64_t) kMaxChunks * kChunk == T3NS_NOALLOC_MAX_SIZE, "size limit");

// [2 * chunk + {0, 1}]: partial sums of uK*t and uK*r per chunk;
// [2 * kMaxChunks]: the Olsen coefficient alpha = -uKr / uKu.
static __device__ __align__(256) double g_noalloc_scratch[2 * kMaxChunks + 32];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
double *g_scratch_ptr[kMaxDevices] = {};

__device__ __forceinline__ double inv_shift(double r, double diff)
{
        return fabs(diff) > kCutoff ? r / diff : (diff < 0 ? -1 : 1) * r / kCutoff;
}

// One block per chunk of 256 elements: uK = result / (diag - theta) (with
// the cutoff), partial sums of uK * vec_t and uK * result.
__global__ void __launch_bounds__(kChunk)
noalloc_partials_kernel(const double *__restrict__ result, const double *__restrict__ vec_t,
                        const double *__restrict__ diag, double theta, int64_t n,
                        double *__restrict__ scratch)
{
        __shared__ double sh[2][kChunk / 32];
        const int64_t i = (int64_t) blockIdx.x * kChunk + threadIdx.x;
        double a = 0, b = 0;
        if (i < n) {
                const double r = result[i];
                const double uK = inv_shift(r, diag[i] - theta);
                a = uK * vec_t[i];
                b = uK * r;
        }
        for (int o = 16; o > 0; o >>= 1) {
                a += __shfl_down_sync(0xffffffffu, a, o);
                b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if ((threadIdx.x & 31) == 0) {
                sh[0][threadIdx.x >> 5] = a;
                sh[1][threadIdx.x >> 5] = b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
                double sa = 0, sb = 0;
                for (int w = 0; w < kChunk / 32; ++w) {
                        sa += sh[0][w];
                        sb += sh[1][w];
                }
                scratch[2 * blockIdx.x] = sa;
                scratch[2 * blockIdx.x + 1] = sb;
        }
}

// One block: sums the partials in a fixed order, stores alpha.
__global__ void __launch_bounds__(256) noalloc_alpha_kernel(double *__restrict__ scratch, int nchunks)
{
        __shared__ double sh[2][256];
        double a = 0, b = 0;
        for (int c = threadIdx.x; c < nchunks; c += 256) {
                a += scratch[2 * c];
                b += scratch[2 * c + 1];
        }
        sh[0][threadIdx.x] = a;
        sh[1][threadIdx.x] = b;
        __syncthreads();
        for (int s = 128; s > 0; s >>= 1) {
                if (threadIdx.x < s) {
                        sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
                        sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
                }
                __syncthreads();
        }
        if (threadIdx.x == 0) scratch[2 * kMaxChunks] = -sh[0][0] / sh[1][0];
}

// vec_t = -(vec_t + alpha * result) / (diag - theta), with the cutoff.
__global__ void __launch_bounds__(kChunk)
noalloc_update_kernel(const double *__restrict__ result, double *__restrict__ vec_t,
                      const double *__restrict__ diag, double theta, int64_t n,
                      const double *__restrict__ scratch)
{
        const int64_t i = (int64_t) blockIdx.x * kChunk + threadIdx.x;
        if (i >= n) return;
        const double alpha = scratch[2 * kMaxChunks];
        const double v = fma(alpha, result[i], vec_t[i]);
        vec_t[i] = -inv_shift(v, diag[i] - theta);
}

// Device address of the scratch array for the current device (looked up once
// per device, with that device current).
int scratch_for_current_device(double **out)
{
        int dev = 0;
        T3NS_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices)
                return set_error(T3NS_E_LIMIT, "precondition_noalloc: device ordinal beyond 63");
        std::lock_guard<std::mutex> g(g_lock);
        if (!g_scratch_ptr[dev]) {
                void *p = nullptr;
                const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
                if (e != cudaSuccess || p == nullptr)
                        return set_error(T3NS_E_CUDA, std::string("precondition_noalloc: "
                                                                  "cudaGetSymbolAddress: ") +
                                                              cudaGetErrorString(e));
                g_scratch_ptr[dev] = static_cast<double *>(p);
        }
        *out = g_scratch_ptr[dev];
        return T3NS_OK;
}

}  // namespace
}  // namespace t3ns

using namespace t3ns;

extern "C" int t3ns_precondition_device_noalloc(int64_t size, const double *result, double theta,
                                                const double *diagonal, double *vec_t,
                                                void *stream)
{
        if (!result || !diagonal || !vec_t || size <= 0)
                return set_error(T3NS_E_ARG, "precondition_noalloc: null buffer or empty vector");
        if (size > T3NS_NOALLOC_MAX_SIZE)
                return set_error(T3NS_E_LIMIT,
                                 "precondition_noalloc: size " + std::to_string(size) +
                                         " exceeds the fixed scratch limit of " +
                                         std::to_string((long long) T3NS_NOALLOC_MAX_SIZE) +
                                         " elements; use t3ns_precondition_host");
        double *scratch = nullptr;
        T3NS_TRY(scratch_for_current_device(&scratch));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int nchunks = (int) ((size + kChunk - 1) / kChunk);
        noalloc_partials_kernel<<<nchunks, kChunk, 0, s>>>(result, vec_t, diagonal, theta, size,
                                                          scratch);
        noalloc_alpha_kernel<<<1, 256, 0, s>>>(scratch, nchunks);
        noalloc_update_kernel<<<nchunks, kChunk, 0, s>>>(result, vec_t, diagonal, theta, size,
                                                        scratch);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}
