// FP64 instantiations, compiled with -fmad=false: no multiply-add
// contraction, so every FP64 result is rounded exactly as the reference's
// (g++ without FMA) rounds it. Also the layout kernels, which move doubles.
#include "launch_impl.cuh"

namespace lbm {

LBM_INSTANTIATE(double, 19)
LBM_INSTANTIATE(double, 27)

__global__ void fill_weights_kernel(double* obs_pop, long long ld, int n, int q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < q; ++d) obs_pop[(long long)d * ld + i] = q == 19 ? Lat<19>::w(d) : Lat<27>::w(d);
}

cudaError_t launch_fill_weights(double* obs_pop, long long ld, int n, int q, cudaStream_t st) {
    fill_weights_kernel<<<(n + 255) / 256, 256, 0, st>>>(obs_pop, ld, n, q);
    return cudaGetLastError();
}

// Moments of the near-wall nodes from obs_mom, after initialisation, in the
// compute type T of the wall shear stress pass.
template <class T>
__global__ void nearwall_moments_kernel(int n_nw, const int* nw_node, const double* obs_mom, long long ld,
                                        bool shifted, T* nw_mom) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nw) return;
    const int n = nw_node[i];
    nw_mom[4 * (long long)i] = (T)(shifted ? obs_mom[n] - 1.0 : obs_mom[n]);
    nw_mom[4 * (long long)i + 1] = (T)obs_mom[ld + n];
    nw_mom[4 * (long long)i + 2] = (T)obs_mom[2 * ld + n];
    nw_mom[4 * (long long)i + 3] = (T)obs_mom[3 * ld + n];
}

cudaError_t launch_nearwall_moments(int n_nw, const int* nw_node, const double* obs_mom, long long ld,
                                    bool shifted, void* nw_mom, bool narrow, cudaStream_t st) {
    if (n_nw == 0) return cudaSuccess;
    if (narrow)
        nearwall_moments_kernel<float><<<(n_nw + 127) / 128, 128, 0, st>>>(n_nw, nw_node, obs_mom, ld, shifted,
                                                                            (float*)nw_mom);
    else
        nearwall_moments_kernel<double><<<(n_nw + 127) / 128, 128, 0, st>>>(n_nw, nw_node, obs_mom, ld, shifted,
                                                                             (double*)nw_mom);
    return cudaGetLastError();
}

__global__ void pop_from_caller_kernel(const double* caller, const int* perm, int n, int q, long long ld,
                                       double* obs_pop) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * q) return;
    const int i = (int)(t / q), d = (int)(t % q);
    obs_pop[(long long)d * ld + i] = caller[(long long)perm[i] * q + d];
}

__global__ void pop_to_caller_kernel(const double* obs_pop, const int* perm, int n, int q, long long ld,
                                     double* caller) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * q) return;
    const int i = (int)(t / q), d = (int)(t % q);
    caller[(long long)perm[i] * q + d] = obs_pop[(long long)d * ld + i];
}

__global__ void mom_to_caller_kernel(const double* obs_mom, const int* perm, int n, long long ld, double* rho,
                                     double* u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long c = perm[i];
    rho[c] = obs_mom[i];
    u[3 * c] = obs_mom[ld + i];
    u[3 * c + 1] = obs_mom[2 * ld + i];
    u[3 * c + 2] = obs_mom[3 * ld + i];
}

cudaError_t launch_pop_from_caller(const double* caller, const int* perm, int n, int q, long long ld,
                                   double* obs_pop, cudaStream_t st) {
    const long long tot = (long long)n * q;
    pop_from_caller_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(caller, perm, n, q, ld, obs_pop);
    return cudaGetLastError();
}

cudaError_t launch_pop_to_caller(const double* obs_pop, const int* perm, int n, int q, long long ld,
                                 double* caller, cudaStream_t st) {
    const long long tot = (long long)n * q;
    pop_to_caller_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(obs_pop, perm, n, q, ld, caller);
    return cudaGetLastError();
}

cudaError_t launch_mom_to_caller(const double* obs_mom, const int* perm, int n, long long ld, double* rho,
                                 double* u, cudaStream_t st) {
    mom_to_caller_kernel<<<(n + 255) / 256, 256, 0, st>>>(obs_mom, perm, n, ld, rho, u);
    return cudaGetLastError();
}

}  // namespace lbm
