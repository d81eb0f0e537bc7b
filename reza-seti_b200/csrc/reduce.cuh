// FP64 boundary mass-flux reduction: Phi = sum over a node list of
// (sum_q c_q f_q) . normal, the momentum density through an inlet or outlet
// plane. Two stages: each block reduces its nodes with warp shuffles and
// writes one partial sum to scratch; one block then sums the partials.
// Populations are read through strides so both the engine's [q][ld] layout and
// a caller's [node][q] layout work. List entries outside [0, n_nodes)
// contribute nothing (lbm_flux_noalloc takes lists the host cannot inspect).
#pragma once

#include <cuda_runtime.h>

#include "lattice.cuh"

namespace lbm {

constexpr int FLUX_THREADS = 256;

static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <int Q>
__global__ void __launch_bounds__(FLUX_THREADS) flux_partial_kernel(const double* __restrict__ f,
                                                                    long long stride_node, long long stride_q,
                                                                    long long n_nodes,
                                                                    const long long* __restrict__ nodes,
                                                                    long long n_list, double nx, double ny,
                                                                    double nz, double* partials) {
    using L = Lat<Q>;
    __shared__ double warp_part[FLUX_THREADS / 32];
    const long long i = (long long)blockIdx.x * FLUX_THREADS + threadIdx.x;
    double v = 0.0;
    const long long node = i < n_list ? nodes[i] : -1;
    if (node >= 0 && node < n_nodes) {
        const double* p = f + node * stride_node;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double cn = L::cx(q) * nx + L::cy(q) * ny + L::cz(q) * nz;
            if (L::cx(q) || L::cy(q) || L::cz(q)) v += cn * p[q * stride_q];
        }
    }
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < FLUX_THREADS / 32 ? warp_part[threadIdx.x] : 0.0;
        w = warp_sum(w);
        if (threadIdx.x == 0) partials[blockIdx.x] = w;
    }
}

// static: the engine and the allocation-free entry point each instantiate it
static __global__ void __launch_bounds__(FLUX_THREADS) flux_final_kernel(const double* __restrict__ partials,
                                                                  int n_partials, double* out) {
    __shared__ double warp_part[FLUX_THREADS / 32];
    double v = 0.0;
    for (int i = threadIdx.x; i < n_partials; i += FLUX_THREADS) v += partials[i];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < FLUX_THREADS / 32 ? warp_part[threadIdx.x] : 0.0;
        w = warp_sum(w);
        if (threadIdx.x == 0) *out = w;
    }
}

// Launches both stages; partials needs one double per block of FLUX_THREADS
// list entries. An empty list writes 0.
inline cudaError_t launch_flux(int q, const double* f, long long stride_node, long long stride_q,
                               long long n_nodes, const long long* nodes, long long n_list,
                               const double normal[3], double* partials, double* out, cudaStream_t st) {
    const int blocks = (int)((n_list + FLUX_THREADS - 1) / FLUX_THREADS);
    if (blocks > 0) {
        if (q == 19)
            flux_partial_kernel<19><<<blocks, FLUX_THREADS, 0, st>>>(f, stride_node, stride_q, n_nodes, nodes,
                                                                     n_list, normal[0], normal[1], normal[2],
                                                                     partials);
        else
            flux_partial_kernel<27><<<blocks, FLUX_THREADS, 0, st>>>(f, stride_node, stride_q, n_nodes, nodes,
                                                                     n_list, normal[0], normal[1], normal[2],
                                                                     partials);
    }
    flux_final_kernel<<<1, FLUX_THREADS, 0, st>>>(partials, blocks, out);
    return cudaGetLastError();
}

}  // namespace lbm
