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
// How: the kernels of lbm_get_flux itself (reduce.cuh: warp shuffles, one
// partial sum per block, one block summing the partials, so both entry points
// sum in the same order), reading the caller's [node][q] populations through
// strides, with the partial sums in g_flux_partials, a fixed array in this
// file's device memory, instead of engine-allocated scratch. Its size bounds
// the list length: LBM_FLUX_NOALLOC_MAX_NODES entries (4096 blocks of 256,
// 32 KiB). The caller passes the populations, the node list and the result
// location, all in device memory.
//
// The array is part of the library's device code. Under lazy module loading
// (the CUDA default) the driver loads that code, and allocates the array with
// it, on the first call on each device; a caller that may not allocate later
// makes that first call (n_list = 0 is enough) at start-up, outside any stream
// capture. The array then stays on that device until the process exits.
//
// Host code never dereferences g_flux_partials: on the host its name is only a
// stand-in for the symbol. Every call looks the array's device address up with
// cudaGetSymbolAddress, with the caller's device current: the lookup allocates
// nothing, and a cached address could outlive the context it belongs to (after
// cudaDeviceReset).
//
// Shared state: every call on a device uses the same array, which keeps the
// previous call's partial sums. Nothing needs clearing — each call writes one
// partial per block it launches before reading them — but two calls that
// overlap on the GPU (different streams, no ordering) race on the array.
#include <cuda_runtime.h>

#include <string>

#include "errors.h"
#include "lbm_b200.h"
#include "reduce.cuh"

namespace {

constexpr int kMaxBlocks = (int)(LBM_FLUX_NOALLOC_MAX_NODES / lbm::FLUX_THREADS);
static_assert((long long)kMaxBlocks * lbm::FLUX_THREADS == LBM_FLUX_NOALLOC_MAX_NODES,
              "the list limit must be a whole number of blocks");

static __device__ __align__(256) double g_flux_partials[kMaxBlocks];

int fail(int code, const std::string& msg) {
    lbm::set_global_error("lbm_flux_noalloc: " + msg);
    return code;
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
    void* partials = nullptr;
    cudaError_t ce = cudaGetSymbolAddress(&partials, g_flux_partials);
    if (ce != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
    // the caller's layout [node][q]: stride q between nodes, 1 between directions
    ce = lbm::launch_flux(q, f, q, 1, n_nodes, reinterpret_cast<const long long*>(nodes), n_list, normal,
                          static_cast<double*>(partials), flux, static_cast<cudaStream_t>(stream));
    if (ce != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(ce));
    return LBM_OK;
}
