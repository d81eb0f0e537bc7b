// Host interface of the adjoint module (adjoint.cu), used by the C ABI in
// engine.cu. Plain pointers and standard containers only.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace lbm {

// Geometry, boundary data and run settings of one adjoint run. Device
// pointers are the engine's own arrays (internal node order).
struct AdjointSetup {
    int Q = 19;
    bool fp64 = false;          // FP64 or FP32 arithmetic and storage
    bool gradient = true;       // false: objective only (forward sweep)
    int objective = 0;          // 0: time-averaged sum of |WSS|^2, 1: mean OSI over the targets
    int n = 0;
    long long ld = 0;
    const void* meta = nullptr;      // Meta<Q>::T [n]
    const int* seg_base = nullptr;
    const int* seg_delta = nullptr;
    int max_block_segs = 1;          // most segments of one BLOCK_NODES block (shared-memory rows)
    const int* aux = nullptr;        // inlet / outlet / near-wall table index per node
    double in_normal[3] = {0, 0, 0}; // outward inlet normal
    int n_in = 0;
    const float* out_nrm = nullptr;  // [n_out][3] outward normal per outlet node
    double out_rho = 1.0;
    int n_nw = 0;
    const int* nw_node = nullptr;    // [n_nw] internal node of each near-wall entry
    const double* nw_normal = nullptr;
    double wss_c = 1.0;
    double tau = 1.0;
    const double* f0 = nullptr;      // [Q][ld] initial populations f (not shifted)
    int64_t n_steps = 0;             // T
    int64_t checkpoint_every = 1;    // K
    std::vector<double> factors;     // [T] inlet waveform factor of each step
    std::vector<double> speed;       // [n_in] inlet speed along -in_normal
    std::vector<int> targets;        // near-wall entries in the objective
    double* final_pop = nullptr;     // optional [Q][ld] device output: f^T (not shifted)
    cudaStream_t stream = nullptr;
};

struct AdjointOut {
    double J = 0.0;
    double dJ_domega = 0.0;
    std::vector<double> dJ_dspeed;   // [n_in]
    float forward_ms = 0.f;          // forward sweep (objective, checkpoints)
    float reverse_ms = 0.f;          // recomputation and backward sweep
    int64_t steps_recomputed = 0;
    size_t bytes = 0;                // device memory the run allocated
    std::string err;
};

// Returns 0, or -1 for an invalid setup (err says why), -2 for a CUDA error.
int adjoint_run(const AdjointSetup& s, AdjointOut& out);

}  // namespace lbm
