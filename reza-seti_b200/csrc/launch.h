// Launchers for the engine's kernels, instantiated in kernels_f64.cu and
// kernels_lowp.cu. The host engine (engine.cu) only sees these declarations.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace lbm {

template <class S, int Q>
cudaError_t launch_step(const StepArgs<S, Q>& a, int phase, int bc, int obs, cudaStream_t st);

template <class S, int Q>
cudaError_t launch_init(const StepArgs<S, Q>& a, int bc, cudaStream_t st);

template <class S, int Q>
cudaError_t launch_boundary(const BoundaryArgs<S, Q>& a, int phase, cudaStream_t st);

template <class S, int Q>
cudaError_t launch_open(const OpenArgs<S, Q>& a, cudaStream_t st);

// Physics mode: wall shear stress of the step just taken and the
// open-boundary corrections of its store, in one launch.
template <class S, int Q>
cudaError_t launch_post(const BoundaryArgs<S, Q>& b, const OpenArgs<S, Q>& o, cudaStream_t st);

// Fills natural-layout populations with the lattice weights (f = w).
cudaError_t launch_fill_weights(double* obs_pop, long long ld, int n, int q, cudaStream_t st);

// nw_mom holds float (narrow) or double values: the compute type of the
// storage (FP32 for shifted storage, FP64 for FP64 storage).
cudaError_t launch_nearwall_moments(int n_nw, const int* nw_node, const double* obs_mom, long long ld,
                                    bool shifted, void* nw_mom, bool narrow, cudaStream_t st);

// Reorders between the caller's [node][q] order and the engine's [q][ld] order;
// perm[i] is the caller index of internal node i.
cudaError_t launch_pop_from_caller(const double* caller, const int* perm, int n, int q, long long ld,
                                   double* obs_pop, cudaStream_t st);
cudaError_t launch_pop_to_caller(const double* obs_pop, const int* perm, int n, int q, long long ld,
                                 double* caller, cudaStream_t st);
cudaError_t launch_mom_to_caller(const double* obs_mom, const int* perm, int n, long long ld, double* rho,
                                 double* u, cudaStream_t st);

}  // namespace lbm
