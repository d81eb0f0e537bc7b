// lbm_flux_noalloc: the boundary mass-flux reduction for callers that cannot
// allocate device memory.
//
// Who needs it: code that must not call cudaMalloc once it runs — a host
// framework that owns all device memory through its own pool and hands this
// library only pointers into it, a process that is forbidden to allocate after
// start-up (real-time or memory-capped jobs), or a post-processing step that
// holds populations in someone else's buffers and wants the inlet/outlet flux
// without creating an engine (lbm_create allocates the whole lattice).
//
// How: the same two-stage FP64 reduction as lbm_get_flux (reduce.cuh: warp
// shuffles, one partial sum per block, one block summing the partials), but
// the partial sums go to g_flux_partials, a fixed array in this file's device
// memory, instead of engine-allocated scratch. The array exists on
// every device that loads the library, until the process exits. Its size
// bounds the list length: LBM_FLUX_NOALLOC_MAX_NODES entries (4096 blocks of
// 256, 32 KiB). The caller passes the populations, the node list and the
// result location, all in device memory.
//
// Host code never dereferences g_flux_partials: on the host its name is only a
// stand-in for the symbol. The first call on each device resolves the array's
// device address with cudaGetSymbolAddress (with that device current) and
// caches it; make that first call outside any stream capture.
//
// Shared state: every call on a device uses the same array, which keeps the
// previous call's partial sums. Nothing needs clearing — each call writes one
// partial per block it launches before reading them — but two calls that
// overlap on the GPU (different streams, no ordering) race on the array.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "errors.h"
#include "lattice.cuh"
#include "lbm_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = (int)(LBM_FLUX_NOALLOC_MAX_NODES / kThreads);
static_assert((long long)kMaxBlocks * kThreads == LBM_FLUX_NOALLOC_MAX_NODES,
              "the list limit must be a whole number of blocks");

static __device__ __align__(256) double g_flux_partials[kMaxBlocks];

std::mutex g_mu;
std::vector<double*> g_partials_ptr;  // device address of g_flux_partials per device ordinal

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// One partial sum per block of the caller's list, populations laid out
// [node][q]; entries outside [0, n_nodes) contribute nothing (the list lives
// in device memory the host cannot check).
template <int Q>
__global__ void __launch_bounds__(kThreads) flux_partial_noalloc_kernel(
    const double* __restrict__ f, long long n_nodes, const long long* __restrict__ nodes, long long n_list,
    double nx, double ny, double nz, double* partials) {
    using L = lbm::Lat<Q>;
    __shared__ double warp_part[kThreads / 32];
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    double v = 0.0;
    if (i < n_list) {
        const long long node = nodes[i];
        if (node >= 0 && node < n_nodes) {
            const double* p = f + node * Q;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const double cn = L::cx(q) * nx + L::cy(q) * ny + L::cz(q) * nz;
                if (L::cx(q) || L::cy(q) || L::cz(q)) v += cn * p[q];
            }
        }
    }
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < kThreads / 32 ? warp_part[threadIdx.x] : 0.0;
        w = warp_sum(w);
        if (threadIdx.x == 0) partials[blockIdx.x] = w;
    }
}

// Sum of the first n_partials partial sums into *out.
__global__ void __launch_bounds__(kThreads) flux_final_noalloc_kernel(const double* __restrict__ partials,
                                                                      int n_partials, double* out) {
    __shared__ double warp_part[kThreads / 32];
    double v = 0.0;
    for (int i = threadIdx.x; i < n_partials; i += kThreads) v += partials[i];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < kThreads / 32 ? warp_part[threadIdx.x] : 0.0;
        w = warp_sum(w);
        if (threadIdx.x == 0) *out = w;
    }
}

int fail(int code, const std::string& msg) {
    lbm::set_global_error("lbm_flux_noalloc: " + msg);
    return code;
}

// Device address of this device's partial-sum array (set-up on first use).
int partials_for_current_device(double** out) {
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return fail(LBM_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    std::lock_guard<std::mutex> lock(g_mu);
    if ((int)g_partials_ptr.size() <= dev) g_partials_ptr.resize(dev + 1, nullptr);
    if (!g_partials_ptr[dev]) {
        void* p = nullptr;
        ce = cudaGetSymbolAddress(&p, g_flux_partials);
        if (ce != cudaSuccess)
            return fail(LBM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
        g_partials_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_partials_ptr[dev];
    return LBM_OK;
}

}  // namespace

extern "C" int lbm_flux_noalloc(const double* f, int64_t n_nodes, int32_t q, const int64_t* nodes,
                                int64_t n_list, const double normal[3], double* flux, void* stream) {
    if (q != 19 && q != 27) return fail(LBM_ERR_ARGUMENT, "q must be 19 or 27");
    if (!f || !flux || !normal || (n_list > 0 && !nodes)) return fail(LBM_ERR_ARGUMENT, "null pointer");
    if (n_nodes < 0 || n_list < 0) return fail(LBM_ERR_ARGUMENT, "negative size");
    if (n_list > LBM_FLUX_NOALLOC_MAX_NODES)
        return fail(LBM_ERR_ARGUMENT, "list of " + std::to_string(n_list) + " nodes exceeds the maximum of " +
                                          std::to_string((long long)LBM_FLUX_NOALLOC_MAX_NODES) +
                                          " (LBM_FLUX_NOALLOC_MAX_NODES)");
    double* partials = nullptr;
    if (int rc = partials_for_current_device(&partials)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = (int)((n_list + kThreads - 1) / kThreads);
    const long long* nl = reinterpret_cast<const long long*>(nodes);
    if (blocks > 0) {
        if (q == 19)
            flux_partial_noalloc_kernel<19><<<blocks, kThreads, 0, st>>>(f, n_nodes, nl, n_list, normal[0],
                                                                         normal[1], normal[2], partials);
        else
            flux_partial_noalloc_kernel<27><<<blocks, kThreads, 0, st>>>(f, n_nodes, nl, n_list, normal[0],
                                                                         normal[1], normal[2], partials);
    }
    flux_final_noalloc_kernel<<<1, kThreads, 0, st>>>(partials, blocks, flux);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(ce));
    return LBM_OK;
}
