// Template bodies of the launchers in launch.h; included once per
// instantiation unit.
#pragma once

#include "launch.h"
#include "pair.cuh"

namespace lbm {

template <class S, int Q, int PHASE, int BC>
static cudaError_t step_obs(const StepArgs<S, Q>& a, int obs, dim3 g, cudaStream_t st) {
    const int smem = PHASE == 1 ? a.seg_smem_bytes : 0;
    switch (obs) {
        case 0: step_kernel<S, Q, PHASE, BC, 0><<<g, BLOCK_NODES, smem, st>>>(a); break;
        case 1: step_kernel<S, Q, PHASE, BC, 1><<<g, BLOCK_NODES, smem, st>>>(a); break;
        case 2: step_kernel<S, Q, PHASE, BC, 2><<<g, BLOCK_NODES, smem, st>>>(a); break;
        default: step_kernel<S, Q, PHASE, BC, 3><<<g, BLOCK_NODES, smem, st>>>(a); break;
    }
    return cudaGetLastError();
}

template <class S, int Q>
static cudaError_t pair_phase0(const StepArgs<S, Q>& a, int obs, dim3 g, cudaStream_t st) {
    const dim3 b(PAIR_THREADS);
    switch (obs) {
        case 0: return launch_pdl(pair_phase0_kernel<S, Q, 0>, g, b, 0, st, a);
        case 1: return launch_pdl(pair_phase0_kernel<S, Q, 1>, g, b, 0, st, a);
        case 2: return launch_pdl(pair_phase0_kernel<S, Q, 2>, g, b, 0, st, a);
        default: return launch_pdl(pair_phase0_kernel<S, Q, 3>, g, b, 0, st, a);
    }
}

// Persistent phase-1 pair kernel: one CTA per resident slot (SM count times
// the occupancy at its shared-memory size), cached per host thread.
template <class S, int Q, int OBS>
static cudaError_t pair_phase1_launch(const StepArgs<S, Q>& a, cudaStream_t st) {
    auto kern = pair_phase1_kernel<S, Q, OBS>;
    const int n_tiles = (a.n + BLOCK_NODES - 1) / BLOCK_NODES;
    const int smem = 2 * pair_buffer_bytes<Q>(a.seg_smem_bytes);
    static thread_local int cached_dev = -1, cached_smem = -1, cached_grid = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev != cached_dev || smem != cached_smem) {
        if (smem > 48 * 1024) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
        }
        int sms = 0, per_sm = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PAIR_THREADS, smem)) != cudaSuccess)
            return e;
        cached_grid = sms * (per_sm > 0 ? per_sm : 1);
        cached_dev = dev;
        cached_smem = smem;
    }
    const int grid = n_tiles < cached_grid ? n_tiles : cached_grid;
    return launch_pdl(kern, dim3(grid), dim3(PAIR_THREADS), smem, st, a, n_tiles);
}

template <class S, int Q>
static cudaError_t pair_phase1(const StepArgs<S, Q>& a, int obs, cudaStream_t st) {
    switch (obs) {
        case 0: return pair_phase1_launch<S, Q, 0>(a, st);
        case 1: return pair_phase1_launch<S, Q, 1>(a, st);
        case 2: return pair_phase1_launch<S, Q, 2>(a, st);
        default: return pair_phase1_launch<S, Q, 3>(a, st);
    }
}

template <class S, int Q>
cudaError_t launch_step(const StepArgs<S, Q>& a, int phase, int bc, int obs, cudaStream_t st) {
    const dim3 g((a.n + BLOCK_NODES - 1) / BLOCK_NODES);
    if constexpr (Store<S>::SHIFTED) {
        // physics mode, shifted storage: two nodes per thread, 32-bit slot
        // indices (lattices beyond 2^32 slots use step_kernel)
        if (bc == BC_PHYSICS && (long long)Q * a.ld < (1LL << 32))
            return phase ? pair_phase1<S, Q>(a, obs, st) : pair_phase0<S, Q>(a, obs, g, st);
    }
    if (bc == BC_REFERENCE) {
        if constexpr (Q == 19) {
            return phase ? step_obs<S, Q, 1, BC_REFERENCE>(a, obs, g, st)
                         : step_obs<S, Q, 0, BC_REFERENCE>(a, obs, g, st);
        } else {
            return cudaErrorInvalidValue;
        }
    }
    return phase ? step_obs<S, Q, 1, BC_PHYSICS>(a, obs, g, st) : step_obs<S, Q, 0, BC_PHYSICS>(a, obs, g, st);
}

template <class S, int Q>
cudaError_t launch_init(const StepArgs<S, Q>& a, int bc, cudaStream_t st) {
    const dim3 g((a.n + BLOCK_NODES - 1) / BLOCK_NODES);
    if (bc == BC_REFERENCE) init_kernel<S, Q, BC_REFERENCE><<<g, BLOCK_NODES, 0, st>>>(a);
    else init_kernel<S, Q, BC_PHYSICS><<<g, BLOCK_NODES, 0, st>>>(a);
    return cudaGetLastError();
}

template <class S, int Q>
cudaError_t launch_boundary(const BoundaryArgs<S, Q>& a, int phase, cudaStream_t st) {
    const long long items = (long long)a.n_wss + (long long)a.n_out * Q;
    if (items == 0) return cudaSuccess;
    const int tpb = 128;
    const dim3 g((unsigned)((items + tpb - 1) / tpb));
    if (phase) boundary_kernel<S, Q, 1><<<g, tpb, 0, st>>>(a);
    else boundary_kernel<S, Q, 0><<<g, tpb, 0, st>>>(a);
    return cudaGetLastError();
}

template <class S, int Q>
cudaError_t launch_open(const OpenArgs<S, Q>& a, cudaStream_t st) {
    const int items = a.n_in + a.n_out;
    if (items == 0) return cudaSuccess;
    open_boundary_kernel<S, Q><<<(items + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

template <class S, int Q>
cudaError_t launch_post(const BoundaryArgs<S, Q>& b, const OpenArgs<S, Q>& o, cudaStream_t st) {
    const long long items = (long long)b.n_wss + o.n_in + o.n_out;
    if (items == 0) return cudaSuccess;
    const int tpb = 128;
    return launch_pdl(post_kernel<S, Q>, dim3((unsigned)((items + tpb - 1) / tpb)), dim3(tpb), 0, st, b, o);
}

#define LBM_INSTANTIATE(S, Q)                                                                          \
    template cudaError_t launch_step<S, Q>(const StepArgs<S, Q>&, int, int, int, cudaStream_t);        \
    template cudaError_t launch_init<S, Q>(const StepArgs<S, Q>&, int, cudaStream_t);                  \
    template cudaError_t launch_boundary<S, Q>(const BoundaryArgs<S, Q>&, int, cudaStream_t);          \
    template cudaError_t launch_open<S, Q>(const OpenArgs<S, Q>&, cudaStream_t);                      \
    template cudaError_t launch_post<S, Q>(const BoundaryArgs<S, Q>&, const OpenArgs<S, Q>&, cudaStream_t);

}  // namespace lbm
