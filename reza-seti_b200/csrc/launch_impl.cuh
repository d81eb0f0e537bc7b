// Template bodies of the launchers in launch.h; included once per
// instantiation unit.
#pragma once

#include "launch.h"

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
cudaError_t launch_step(const StepArgs<S, Q>& a, int phase, int bc, int obs, cudaStream_t st) {
    const dim3 g((a.n + BLOCK_NODES - 1) / BLOCK_NODES);
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

#define LBM_INSTANTIATE(S, Q)                                                                          \
    template cudaError_t launch_step<S, Q>(const StepArgs<S, Q>&, int, int, int, cudaStream_t);        \
    template cudaError_t launch_init<S, Q>(const StepArgs<S, Q>&, int, cudaStream_t);                  \
    template cudaError_t launch_boundary<S, Q>(const BoundaryArgs<S, Q>&, int, cudaStream_t);          \
    template cudaError_t launch_open<S, Q>(const OpenArgs<S, Q>&, cudaStream_t);

}  // namespace lbm
