// cldenseDdotNoAlloc: the FP64 dot product <x, y> for callers that must not
// allocate device memory.
//
// Who needs it: code that calls into the library from a place where a
// cudaMalloc is not allowed or not safe -- a real-time loop that forbids
// allocation after start-up, an application that routes every device
// allocation through its own pool and budget, or code enqueuing work into a
// stream it does not own while another thread records it into a graph.
// cudaMalloc can also synchronise the whole device. The regular cldenseDdot
// needs a clsparseControl, whose creation allocates its reduction scratch;
// this entry point needs neither: it takes the stream directly and keeps its
// scratch in a fixed, file-scope device array.
//
// Scratch: kSlots per-CTA partial sums plus an arrival ticket, about 16 KB,
// held by every GPU that loads the library until the process exits. Each CTA
// sums a fixed chunk of kChunk elements, so vectors are limited to
// kSlots * kChunk = 33,554,432 elements; longer ones are rejected with
// clsparseInvalidSize. The result depends only on n (fixed chunking and a
// fixed summation order), not on the GPU or the launch.
//
// All calls share the one array: calls that overlap on the GPU (different
// streams, or different host threads, running at the same time) race on it
// and must be serialised by the caller. The first call on each device looks
// up the array's device address (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture is begun. Only a
// successful lookup is kept: a call whose lookup fails returns
// clsparseInvalidDevice and the next call tries again. The address is kept
// for the life of the process, so resetting a device (cudaDeviceReset) after
// the first call on it is not supported: the array may be reloaded elsewhere.
#include <atomic>
#include <mutex>

#include "device_common.cuh"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSlots = 2048;
constexpr uint32_t kChunk = 16384;
constexpr uint64_t kMaxElements = static_cast<uint64_t>(kSlots) * kChunk;

// [0, kSlots): partial sums; word kSlots: arrival ticket (as uint32).
static __device__ __align__(256) double g_dot_scratch[kSlots + 32];

// Device addresses of g_dot_scratch, one per device: null until a lookup
// with that device current has succeeded.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex[kMaxDevices];
std::atomic<double*> g_addr[kMaxDevices];

double* scratch_address(int dev) {
    double* p = g_addr[dev].load(std::memory_order_acquire);
    if (p) return p;
    std::lock_guard<std::mutex> lock(g_addr_mutex[dev]);
    p = g_addr[dev].load(std::memory_order_relaxed);
    if (p) return p;
    void* q = nullptr;
    if (cudaGetSymbolAddress(&q, g_dot_scratch) != cudaSuccess || q == nullptr) {
        cudaGetLastError();  // not sticky: leave no error behind for the caller's next call
        return nullptr;
    }
    p = static_cast<double*>(q);
    g_addr[dev].store(p, std::memory_order_release);
    return p;
}

__global__ void __launch_bounds__(kThreads)
    dot_noalloc_kernel(const double* __restrict__ x, const double* __restrict__ y, uint64_t n,
                       double* scratch, double* out) {
    const uint64_t begin = static_cast<uint64_t>(blockIdx.x) * kChunk;
    const uint64_t end = begin + kChunk < n ? begin + kChunk : n;
    double acc[1] = {0.0};
    for (uint64_t i = begin + threadIdx.x; i < end; i += kThreads) acc[0] += x[i] * y[i];
    double tot[1];
    uint32_t* ticket = reinterpret_cast<uint32_t*>(scratch + kSlots);
    if (dev::grid_reduce_last<1>(acc, scratch, ticket, tot) && threadIdx.x == 0) *out = tot[0];
}

}  // namespace
}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus cldenseDdotNoAlloc(clsparseScalar* r, const cldenseVector* x, const cldenseVector* y,
                                  cl_command_queue queue) {
    if (g_initialized.load() == 0) return clsparseNotInitialized;
    if (!r || !x || !y || !r->value) return clsparseInvalidValue;
    if (x->num_values != y->num_values) return clsparseInvalidSize;
    const uint64_t n = x->num_values;
    if (n > kMaxElements) return clsparseInvalidSize;
    if (n > 0 && (!x->values || !y->values)) return clsparseInvalidMemObject;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return clsparseInvalidDevice;
    // Set-up on this device (first successful call): the host-side symbol is
    // only a stand-in, the kernel needs the array's device address.
    double* scratch = scratch_address(dev);
    if (scratch == nullptr) return clsparseInvalidDevice;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(queue);
    // the ticket must start at zero; a call cut short earlier may have left it set
    if (cudaMemsetAsync(scratch + kSlots, 0, sizeof(double), s) != cudaSuccess)
        return clsparseInvalidKernelExecution;
    const uint32_t grid = n == 0 ? 1u : static_cast<uint32_t>((n + kChunk - 1) / kChunk);
    dot_noalloc_kernel<<<grid, kThreads, 0, s>>>(dev_ptr<const double>(x->values, x->off_values),
                                                 dev_ptr<const double>(y->values, y->off_values), n,
                                                 scratch, dev_ptr<double>(r->value, r->off_value));
    return cudaGetLastError() == cudaSuccess ? clsparseSuccess : clsparseInvalidKernelExecution;
}

}  // extern "C"
