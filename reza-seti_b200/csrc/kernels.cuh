// Device code of the LBM engine: AA-pattern stream+collide kernels, the
// boundary pre-pass (wall shear stress and outlet sources), initialisation and
// reductions. Instantiated for each storage type in kernels_f64.cu (built
// without FMA contraction, so FP64 results equal the reference's rounding)
// and kernels_lowp.cu (FP32 / FP16 / BF16 storage, FP32 arithmetic).
//
// State layout in HBM: one population buffer pop[q * ld + n] (structure of
// arrays, ld = node count padded to BLOCK_NODES), updated in place with the
// AA access pattern. A kernel either reads the "natural" layout (phase 0:
// slot (n, q) holds the population arriving at n in direction q) or the
// "swapped" layout (phase 1: that population sits in slot (n - c_q, opp q)),
// and leaves the other layout for the next step:
//   phase 0: read slot (n, q);             write slot (n, opp q)
//   phase 1: read slot (n - c_q, opp q);   write slot (n + c_q, q)
// Every node reads and writes the same set of slots, so the in-place update
// has no inter-thread hazard.
//
// Missing neighbours. In reference mode a population whose upstream node does
// not exist keeps the value the node held before the step (the reference only
// streams into existing neighbours, Simulation.cpp:247-251); the kernel keeps
// that value in the slot the missing upstream would have written, which no
// other thread touches. In physics mode the same slot receives the node's own
// post-collision population in the opposite direction (halfway bounce-back),
// with the velocity (inlet) or pressure (outlet) correction on open-boundary
// links.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lattice.cuh"

namespace lbm {

// ---------------------------------------------------------------- storage ---
// Populations are stored as f (FP64) or as the deviation f - w_q from the
// lattice weight (FP32 / FP16 / BF16), and computed in double or float.
template <class S>
struct Store;

template <>
struct Store<double> {
    using C = double;
    static constexpr bool SHIFTED = false;
    static constexpr int MIN_BLOCKS = 1;  // resident 256-thread blocks per SM the step kernel targets
    __device__ static C get(const double* p) { return *p; }
    __device__ static void put(double* p, C v) { *p = v; }
};
template <>
struct Store<float> {
    using C = float;
    static constexpr bool SHIFTED = true;
    static constexpr int MIN_BLOCKS = 4;
    __device__ static C get(const float* p) { return *p; }
    __device__ static void put(float* p, C v) { *p = v; }
};
template <>
struct Store<__half> {
    using C = float;
    static constexpr bool SHIFTED = true;
    static constexpr int MIN_BLOCKS = 4;
    __device__ static C get(const __half* p) { return __half2float(*p); }
    __device__ static void put(__half* p, C v) { *p = __float2half_rn(v); }
};
template <>
struct Store<__nv_bfloat16> {
    using C = float;
    static constexpr bool SHIFTED = true;
    static constexpr int MIN_BLOCKS = 4;
    __device__ static C get(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ static void put(__nv_bfloat16* p, C v) { *p = __float2bfloat16_rn(v); }
};

enum BcMode : int { BC_REFERENCE = 0, BC_PHYSICS = 1 };

enum Flag : unsigned {
    FLAG_ZERO_SKIP = 1u,  // a streamed population was exactly 0.0 (reference skips it)
    FLAG_NONFINITE = 2u,  // a density became NaN or infinite
};

// ------------------------------------------------------------- arguments ---
template <class S, int Q>
struct StepArgs {
    using C = typename Store<S>::C;
    using MT = typename Meta<Q>::T;
    S* pop;
    long long ld;
    int n;
    const MT* meta;
    const int* seg_base;   // [blocks] first segment of each block
    const int* seg_delta;  // [segments][Q] neighbour index offsets
    // shifted storage: [segments][Q] slot offsets d * ld + delta (mod 2^32),
    // the rows of the pair phase-1 kernel (one add per slot index)
    const int* seg_slot;
    int seg_smem_bytes;    // shared memory for the largest block's segment rows
    const int* aux;        // [n] index into the inlet / outlet / near-wall tables
    C omega;               // 1 / tau
    // reference-mode inlet: one normal and one velocity for all inlet nodes
    double inlet_normal[3];
    double inlet_vel;
    // reference-mode outlets: per outlet node, has-source flag and the
    // populations copied from its source (written by the pre-pass)
    const int* out_src;
    const C* out_buf;
    // physics mode: velocity of each outlet node's collision, [n_out][3],
    // for the open-boundary pass
    double* io_u;
    // near-wall nodes hand the wall-shear pass what it needs of the step,
    // [handoff_rows][n_nw] (aux[n] is the index): FP64 the Q arriving
    // populations, the shifted types their six second moments and the
    // collision's drho, u
    C* nw_s;
    int n_nw;
    // observation (written only by observing launches)
    double* obs_pop;       // [Q][ld] post-boundary populations f (natural layout)
    double* obs_mom;       // [4][ld] rho, ux, uy, uz
    unsigned* flags;
    // phase-1 pair kernel: 1 = every warp takes the per-node path, never the
    // twin path (LBM_B200_PHASE1_GENERAL=1; the two give identical results)
    int force_general;
    // persistent phase-1 kernel: [0] the tile counter CTAs take their next
    // tile from, [1] CTAs finished; the last CTA out zeroes both
    int* tile_sched;
};

template <class S, int Q>
struct BoundaryArgs {
    using C = typename Store<S>::C;
    using MT = typename Meta<Q>::T;
    const S* pop;
    long long ld;
    const MT* meta;
    const int* seg_base;
    const int* seg_delta;
    // wall shear stress of the previous step's near-wall nodes (n_wss = 0
    // when there is none pending)
    int n_wss;
    int n_nw;
    const C* nw_s;            // [handoff_rows][n_nw] hand-off of the previous step
    // normals and moments in the compute type: the FP32 traction reads both
    // as float, and the moments it stores are FP32 values, so FP32 storage
    // keeps them exactly in 28 instead of 56 bytes per node
    const C* nw_normal;       // [n_nw][3]
    C* nw_mom;                // [n_nw][4] moments that step's f_eq used (rho or rho-1, u)
    double* wss;              // [n_nw]
    double* acc;              // [n_nw][3]
    double* accmag;           // [n_nw]
    double wss_c;             // 1060 dt^2 / (spacing^2 1e-6)
    // outlet sources, one thread per (outlet node, direction)
    int n_out;
    const int* out_src;       // [n_out] source node or -1; ~src for a source that is an inlet node
    C* out_buf;               // [n_out][Q]
    double inlet_normal[3];
    double inlet_vel;
};

// ------------------------------------------------------------ neighbours ---
template <int Q>
__device__ __forceinline__ const int* seg_row(const int* seg_base, const int* seg_delta, int n,
                                              typename Meta<Q>::T m) {
    const int s = __ldg(seg_base + n / BLOCK_NODES) + (int)(m >> Meta<Q>::SEG_SHIFT);
    return seg_delta + (long long)s * Q;
}

// Populations arriving at node n (post-streaming values) in compute type.
template <class S, int Q, int PHASE>
__device__ __forceinline__ void gather(const S* __restrict__ pop, long long ld, int n,
                                       typename Meta<Q>::T m, const int* sd,
                                       typename Store<S>::C s[Q]) {
    using L = Lat<Q>;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        long long idx;
        if (PHASE == 0 || q == L::REST) {
            idx = (long long)q * ld + n;
        } else {
            const int oq = L::opp(q);
            idx = ((m >> oq) & 1) ? (long long)oq * ld + (n + sd[oq]) : (long long)q * ld + n;
        }
        s[q] = Store<S>::get(pop + idx);
    }
}

// ------------------------------------------ programmatic dependent launch ---
// Physics-mode step and post kernels go out with programmatic stream
// serialisation: a kernel's CTAs may be scheduled while the previous kernel
// on the stream finishes. Each waits here (griddepcontrol.wait: until the
// previous grid has completed and its writes are visible) before it reads
// anything that kernel or an earlier one wrote; a kernel launched without
// such a predecessor passes straight through. allow_next_grid lets the next
// kernel's CTAs be scheduled once every CTA of this one has called it.
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// A launch with programmatic stream serialisation (the kernel must call
// wait_prior_grid before it reads earlier kernels' results).
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

// --------------------------------------------------------------- moments ---
// FP64, reference operand order (Simulation.cpp:85-139 for D3Q19).
template <int Q>
__device__ __forceinline__ void moments_ref(const double f[Q], bool wall, double& rho, double u[3]) {
    using L = Lat<Q>;
    rho = 0.0;
#pragma unroll
    for (int q = 0; q < Q; ++q) rho += f[q];
    if (wall) {
        u[0] = 0.0;
        u[1] = 0.0;
        u[2] = 0.0;
        return;
    }
    if constexpr (Q == 19) {
        u[0] = ((f[0] + f[6] + f[7] + f[8] + f[9]) - (f[1] + f[10] + f[11] + f[12] + f[13])) / rho;
        u[1] = ((f[2] + f[6] + f[10] + f[14] + f[15]) - (f[3] + f[7] + f[11] + f[16] + f[17])) / rho;
        u[2] = ((f[4] + f[8] + f[12] + f[14] + f[16]) - (f[5] + f[9] + f[13] + f[15] + f[17])) / rho;
    } else {
        double j[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (L::cx(q)) j[0] += L::cx(q) > 0 ? f[q] : -f[q];
            if (L::cy(q)) j[1] += L::cy(q) > 0 ? f[q] : -f[q];
            if (L::cz(q)) j[2] += L::cz(q) > 0 ? f[q] : -f[q];
        }
        u[0] = j[0] / rho;
        u[1] = j[1] / rho;
        u[2] = j[2] / rho;
    }
}

// f_eq of direction q, reference operand order (Simulation.cpp:214-223).
template <int Q>
__device__ __forceinline__ double feq_ref(int q, double rho, const double u[3]) {
    using L = Lat<Q>;
    const double du = u[0] * (double)L::cx(q) + u[1] * (double)L::cy(q) + u[2] * (double)L::cz(q);
    const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    return L::w(q) * rho * (1.0 + 3.0 * du + 4.5 * du * du - 1.5 * usq);
}

// FP32 arithmetic on deviations d_q = f_q - w_q: drho = rho - 1 = sum d,
// momentum = sum c d (the weights carry no momentum).
template <int Q>
__device__ __forceinline__ void moments_shifted(const float d[Q], bool wall, float& drho, float u[3]) {
    using L = Lat<Q>;
    float a = 0.f, b = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) (q & 1 ? b : a) += d[q];
    drho = a + b;
    if (wall) {
        u[0] = u[1] = u[2] = 0.f;
        return;
    }
    float j[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (L::cx(q)) j[0] += L::cx(q) > 0 ? d[q] : -d[q];
        if (L::cy(q)) j[1] += L::cy(q) > 0 ? d[q] : -d[q];
        if (L::cz(q)) j[2] += L::cz(q) > 0 ? d[q] : -d[q];
    }
    const float inv = 1.f / (1.f + drho);
    u[0] = j[0] * inv;
    u[1] = j[1] * inv;
    u[2] = j[2] * inv;
}

// deviation of f_eq from w_q
template <int Q>
__device__ __forceinline__ float deq_shifted(int q, float drho, const float u[3]) {
    using L = Lat<Q>;
    const float cu = u[0] * (float)L::cx(q) + u[1] * (float)L::cy(q) + u[2] * (float)L::cz(q);
    const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    return (float)L::w(q) * (drho + (1.f + drho) * (3.f * cu + 4.5f * cu * cu - 1.5f * usq));
}

// BGK collision: c = s + omega (s_eq - s). Returns the moments it used:
// m0 = rho (FP64) or rho - 1 (shifted), u.
template <class C, int Q>
__device__ __forceinline__ void collide(const C s[Q], bool wall, C omega, C c[Q], C& m0, C u[3]) {
    if constexpr (sizeof(C) == 8) {
        double rho;
        moments_ref<Q>(s, wall, rho, u);
        m0 = rho;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double fe = feq_ref<Q>(q, rho, u);
            c[q] = s[q] + omega * (fe - s[q]);
        }
    } else {
        float drho;
        moments_shifted<Q>(s, wall, drho, u);
        m0 = drho;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float de = deq_shifted<Q>(q, drho, u);
            c[q] = s[q] + omega * (de - s[q]);
        }
    }
}

// ------------------------------------------------------------ Zou-He inlet ---
// Velocity inlet of the reference, Boundary::ApplyBc (Boundary.cpp:111-289).
// The six face branches are independent `if`s in the reference, applied in
// this order. The rows keep its quirks: the y branches prescribe u_y = 1
// (:178, :206) and the +z branch sums the -y population set (:239-241).
struct ZouHeRow {
    int comp, positive, vel_comp, unit_velocity;
    int tang[9];
    int out[5];
    int denom_sign;
    int nplus[2][3], nminus[2][3], nvcomp[2];
    int dst[5], src[5], third[5], ca[5], sa[5], cb[5], sb[5], nidx[5], nsign[5];
};

__constant__ ZouHeRow kZouHe[6] = {
    // +x (:115-140)
    {0, 1, 0, 0, {2, 3, 4, 5, 14, 15, 16, 17, 18}, {0, 6, 7, 8, 9}, +1,
     {{2, 14, 15}, {4, 16, 14}}, {{3, 16, 17}, {5, 15, 17}}, {1, 2},
     {1, 10, 11, 13, 12}, {0, 7, 6, 8, 9}, {1, 0, 0, 0, 0}, {0, 0, 0, 0, 0},
     {-1, -1, -1, -1, -1}, {0, 1, 1, 2, 2}, {0, +1, -1, -1, +1}, {0, 0, 0, 1, 1},
     {0, -1, +1, +1, -1}},
    // -x (:143-168)
    {0, 0, 0, 0, {2, 3, 4, 5, 14, 15, 16, 17, 18}, {1, 10, 11, 12, 13}, -1,
     {{2, 14, 15}, {4, 16, 14}}, {{3, 16, 17}, {5, 15, 17}}, {1, 2},
     {0, 7, 6, 8, 9}, {1, 10, 11, 13, 12}, {1, 0, 0, 0, 0}, {0, 0, 0, 0, 0},
     {+1, +1, +1, +1, +1}, {0, 1, 1, 2, 2}, {0, -1, +1, +1, -1}, {0, 0, 0, 1, 1},
     {0, +1, -1, -1, +1}},
    // +y (:171-195)
    {1, 1, 1, 1, {0, 1, 4, 5, 8, 9, 12, 13, 18}, {2, 6, 10, 14, 15}, +1,
     {{0, 8, 9}, {4, 8, 12}}, {{1, 12, 13}, {5, 9, 13}}, {0, 2},
     {3, 11, 7, 17, 16}, {2, 6, 10, 14, 15}, {1, 0, 0, 0, 0}, {1, 0, 1, 1, 1},
     {-1, -1, -1, -1, -1}, {0, 1, 0, 2, 2}, {0, -1, +1, -1, +1}, {0, 0, 0, 1, 1},
     {0, +1, -1, +1, -1}},
    // -y (:197-221)
    {1, 0, 1, 1, {0, 1, 4, 5, 8, 9, 12, 13, 18}, {3, 7, 11, 16, 17}, -1,
     {{0, 8, 9}, {4, 8, 12}}, {{1, 12, 13}, {5, 9, 13}}, {0, 2},
     {2, 6, 10, 14, 15}, {3, 11, 7, 17, 16}, {1, 0, 0, 0, 0}, {1, 0, 1, 1, 1},
     {+1, +1, +1, +1, +1}, {0, 1, 0, 2, 2}, {0, +1, -1, +1, -1}, {0, 0, 0, 1, 1},
     {0, -1, +1, -1, +1}},
    // +z (:225-249)
    {2, 1, 2, 0, {0, 1, 4, 5, 8, 9, 12, 13, 18}, {3, 7, 11, 16, 17}, +1,
     {{0, 6, 7}, {2, 6, 10}}, {{1, 10, 11}, {3, 7, 11}}, {0, 1},
     {5, 9, 13, 15, 17}, {4, 12, 8, 16, 14}, {1, 0, 0, 0, 0}, {2, 0, 0, 1, 1},
     {-1, +1, -1, +1, -1}, {0, 2, 2, 2, 2}, {0, -1, -1, -1, -1}, {0, 0, 0, 1, 1},
     {0, -1, +1, -1, +1}},
    // -z (:262-288)
    {2, 0, 2, 0, {0, 1, 2, 3, 6, 7, 10, 11, 18}, {5, 9, 13, 15, 17}, -1,
     {{0, 6, 7}, {2, 6, 10}}, {{1, 10, 11}, {3, 7, 11}}, {0, 1},
     {4, 8, 12, 14, 16}, {5, 13, 9, 17, 15}, {1, 0, 0, 0, 0}, {2, 0, 0, 1, 1},
     {+1, +1, -1, +1, -1}, {0, 2, 2, 2, 2}, {0, +1, +1, +1, +1}, {0, 0, 0, 1, 1},
     {0, -1, +1, -1, +1}},
};

// Applies the reference Zou-He inlet to one node's D3Q19 populations s (f in
// FP64, deviations f - w in the shifted types; the weights of every summed
// set add up to 1 and cancel in every difference, so the same rows serve both).
template <class C>
__device__ __forceinline__ void zou_he(C s_in[19], const double normal[3], double vel) {
    C f[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = s_in[q];
    for (int b = 0; b < 6; ++b) {
        const ZouHeRow& z = kZouHe[b];
        const double nc = normal[z.comp];
        if (!(z.positive ? nc > 0 : nc < 0)) continue;
        C u[3] = {C(0), C(0), C(0)};
        u[z.vel_comp] = z.unit_velocity ? C(1) : C(vel);
        C tsum = f[z.tang[0]];
        for (int k = 1; k < 9; ++k) tsum += f[z.tang[k]];
        C osum = f[z.out[0]];
        for (int k = 1; k < 5; ++k) osum += f[z.out[k]];
        const C denom = z.denom_sign > 0 ? C(1) + u[z.vel_comp] : C(1) - u[z.vel_comp];
        C rhoN;
        if constexpr (sizeof(C) == 8) rhoN = (tsum + 2 * osum) / denom;
        else rhoN = (C(1) + (tsum + 2 * osum)) / denom;
        C N[2];
        for (int c = 0; c < 2; ++c) {
            const C d = f[z.nplus[c][0]] + f[z.nplus[c][1]] + f[z.nplus[c][2]] - f[z.nminus[c][0]] -
                        f[z.nminus[c][1]] - f[z.nminus[c][2]];
            N[c] = (C(1.0) / 2) * d - (C(1.0) / 3) * (rhoN * u[z.nvcomp[c]]);
        }
        for (int k = 0; k < 5; ++k) {
            if (z.third[k]) {
                const C t = (1 / C(3.0)) * rhoN * u[z.ca[k]];
                f[z.dst[k]] = z.sa[k] > 0 ? f[z.src[k]] + t : f[z.src[k]] - t;
            } else {
                const C va = z.sa[k] > 0 ? u[z.ca[k]] : -u[z.ca[k]];
                const C vb = z.sb[k] > 0 ? u[z.cb[k]] : -u[z.cb[k]];
                const C t = f[z.src[k]] + (1 / C(6.0)) * rhoN * (va + vb);
                f[z.dst[k]] = z.nsign[k] > 0 ? t + N[z.nidx[k]] : t - N[z.nidx[k]];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) s_in[q] = f[q];
}

// Wall fix-up of the reference (Simulation.cpp:746-763): in direction order,
// a missing neighbour in direction q copies the population of q into opp(q).
template <class C, int Q>
__device__ __forceinline__ void wall_fixup(C s[Q], typename Meta<Q>::T m) {
    using L = Lat<Q>;
#pragma unroll
    for (int q = 0; q < Q; ++q)
        if (!((m >> q) & 1)) s[L::opp(q)] = s[q];
}

// ------------------------------------------------------ wall shear stress ---
// Rows of the near-wall hand-off per node. FP64 hands over the Q arriving
// populations: the reference's triple loop runs on f - f_eq per direction.
// The shifted types hand over what their traction needs, 10 values instead
// of Q: the second moments Pi_ab = sum_q d_q c_qa c_qb of the arriving
// deviations (rows 0-5: xx yy zz xy xz yz) and the moments of the node's
// collision, drho and u (rows 6-9), which become the f_eq of the next step's
// wall shear stress.
template <class C, int Q>
__host__ __device__ constexpr int handoff_rows() {
    return sizeof(C) == 8 ? Q : 10;
}
constexpr int HANDOFF_MOM_ROW = 6;

// Pi_ab = sum_q v_q c_qa c_qb over the moving directions, entry J of
// xx yy zz xy xz yz, for a scalar or a packed pair (add / sub give the
// arithmetic). One entry at a time: a caller that stores each entry as it
// comes holds one accumulator, not six.
template <int Q, int J, class T, class Add, class Sub>
__device__ __forceinline__ T second_moment(const T v[Q], T zero, Add add, Sub sub) {
    using L = Lat<Q>;
    constexpr int A = J < 3 ? J : (J == 5 ? 1 : 0);  // the entry's two axes
    constexpr int B = J < 3 ? J : (J == 3 ? 1 : 2);
    T p = zero;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int c[3] = {L::cx(q), L::cy(q), L::cz(q)};
        const int cc = c[A] * c[B];
        if (cc > 0) p = add(p, v[q]);
        else if (cc < 0) p = sub(p, v[q]);
    }
    return p;
}

template <int Q, class T, class Add, class Sub>
__device__ __forceinline__ void second_moments(const T v[Q], T P[6], T zero, Add add, Sub sub) {
    P[0] = second_moment<Q, 0>(v, zero, add, sub);
    P[1] = second_moment<Q, 1>(v, zero, add, sub);
    P[2] = second_moment<Q, 2>(v, zero, add, sub);
    P[3] = second_moment<Q, 3>(v, zero, add, sub);
    P[4] = second_moment<Q, 4>(v, zero, add, sub);
    P[5] = second_moment<Q, 5>(v, zero, add, sub);
}

// Simulation::ComputeWallShearStress (Simulation.cpp:767-799), operand order
// kept. fne[q] = f - f_eq of the near-wall node.
template <class C, int Q>
__device__ __forceinline__ void shear_traction(const C fne[Q], const double nrm_d[3], double wss_c,
                                               double tau[3]) {
    using L = Lat<Q>;
    const C nrm[3] = {C(nrm_d[0]), C(nrm_d[1]), C(nrm_d[2])};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        C sum_alpha = C(0);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const C c[3] = {C(L::cx(q)), C(L::cy(q)), C(L::cz(q))};
            C sum_k = C(0);
#pragma unroll
            for (int b = 0; b < 3; ++b) sum_k += c[b] * nrm[b] * nrm[a];
            C sum_j = C(0);
#pragma unroll
            for (int b = 0; b < 3; ++b) sum_j += c[b] * nrm[b] * (c[a] - sum_k);
            sum_alpha += fne[q] * sum_j;
        }
        tau[a] = wss_c * (double)sum_alpha;
    }
}

// Wall shear stress of near-wall node k from what its step handed over and
// the moments its previous collision used (the f_eq the reference keeps in
// m_eqdistributions), accumulated in FP64 (Simulation.cpp:767-799).
template <class S, int Q>
__device__ __forceinline__ void wall_shear(const BoundaryArgs<S, Q>& a, int k) {
    using C = typename Store<S>::C;
    using L = Lat<Q>;
    constexpr int R = handoff_rows<C, Q>();
    C h[R];
#pragma unroll
    for (int r = 0; r < R; ++r) h[r] = a.nw_s[(long long)r * a.n_nw + k];
    C* mom = a.nw_mom + 4 * (long long)k;
    const C* nd = a.nw_normal + 3 * (long long)k;
    // the accumulators are read with the rest, not after the stores below:
    // one memory round trip per node instead of two
    double* acc = a.acc + 3 * (long long)k;
    const double acc0 = acc[0], acc1 = acc[1], acc2 = acc[2], accm = a.accmag[k];
    double tau[3];
    C m0, u[3];
    if constexpr (sizeof(C) == 8) {
        // FP64: the reference's own triple loop, operand order kept
        C fne[Q];
        const double up[3] = {mom[1], mom[2], mom[3]};
#pragma unroll
        for (int q = 0; q < Q; ++q) fne[q] = h[q] - feq_ref<Q>(q, mom[0], up);
        shear_traction<C, Q>(fne, nd, a.wss_c, tau);
        // moments of these populations: the f_eq of the next step's WSS (the
        // same arithmetic as that step's collision of this node)
        double rho;
        moments_ref<Q>(h, false, rho, u);
        m0 = rho;
    } else {
        // the traction through the non-equilibrium stress tensor,
        // Pi_ab = sum_q fne_q c_qa c_qb:  sum_q fne_q (c.n)(c_a - (c.n) n_a)
        // = (Pi n)_a - (n.Pi.n) n_a, with Pi(fne) = Pi(d) - Pi(deq)
        const float up[3] = {(float)mom[1], (float)mom[2], (float)mom[3]};
        const float drho = (float)mom[0];
        float de[Q], Pe[6];
#pragma unroll
        for (int q = 0; q < Q; ++q) de[q] = q == L::REST ? 0.f : deq_shifted<Q>(q, drho, up);
        second_moments<Q>(de, Pe, 0.f, [](float x, float y) { return x + y; },
                          [](float x, float y) { return x - y; });
        float P[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) P[j] = h[j] - Pe[j];
        const float n0 = (float)nd[0], n1 = (float)nd[1], n2 = (float)nd[2];
        const float pn0 = P[0] * n0 + P[3] * n1 + P[4] * n2;
        const float pn1 = P[3] * n0 + P[1] * n1 + P[5] * n2;
        const float pn2 = P[4] * n0 + P[5] * n1 + P[2] * n2;
        const float t = pn0 * n0 + pn1 * n1 + pn2 * n2;
        tau[0] = a.wss_c * (double)(pn0 - t * n0);
        tau[1] = a.wss_c * (double)(pn1 - t * n1);
        tau[2] = a.wss_c * (double)(pn2 - t * n2);
        // the moments this step's collision used, handed over by the step
        m0 = h[HANDOFF_MOM_ROW];
        u[0] = h[HANDOFF_MOM_ROW + 1];
        u[1] = h[HANDOFF_MOM_ROW + 2];
        u[2] = h[HANDOFF_MOM_ROW + 3];
    }
    const double w = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
    a.wss[k] = w;
    acc[0] = acc0 + tau[0];
    acc[1] = acc1 + tau[1];
    acc[2] = acc2 + tau[2];
    a.accmag[k] = accm + w;
    mom[0] = m0;
    mom[1] = u[0];
    mom[2] = u[1];
    mom[3] = u[2];
}

// ---------------------------------------------------------------- kernels ---
// One AA step over all nodes. BC selects reference or physics boundaries;
// OBS writes the post-boundary populations and/or moments for the host.
template <class S, int Q, int PHASE, int BC, int OBS>
__global__ void __launch_bounds__(BLOCK_NODES, Store<S>::MIN_BLOCKS) step_kernel(StepArgs<S, Q> a) {
    using L = Lat<Q>;
    using C = typename Store<S>::C;
    using MT = typename Meta<Q>::T;
    extern __shared__ int seg_smem[];
    const int n = blockIdx.x * BLOCK_NODES + threadIdx.x;
    const bool live = n < a.n;
    const MT m = live ? a.meta[n] : MT(0);
    const int* sd = nullptr;
    if (PHASE == 1) {
        // the block's segment offsets, staged once in shared memory: the
        // neighbour addresses then depend on one global load (meta) only
        const int s0 = __ldg(a.seg_base + blockIdx.x);
        const int cnt = (__ldg(a.seg_base + blockIdx.x + 1) - s0) * Q;
        const int* src = a.seg_delta + (long long)s0 * Q;
        for (int i = threadIdx.x; i < cnt; i += BLOCK_NODES) seg_smem[i] = __ldg(src + i);
        __syncthreads();
        sd = seg_smem + Q * (int)(m >> Meta<Q>::SEG_SHIFT);
    }
    if (!live) return;
    const int kind = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);

    C s[Q];
    gather<S, Q, PHASE>(a.pop, a.ld, n, m, sd, s);

    if constexpr (BC == BC_REFERENCE) {
        if constexpr (!Store<S>::SHIFTED) {
            // the reference does not stream a population that is exactly 0.0
            // (Simulation.cpp:249); flag it, the AA layout cannot keep both values
            bool zero = false;
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (q == L::REST || ((m >> L::opp(q)) & 1)) zero |= (s[q] == 0.0);
            if (zero) atomicOr(a.flags, FLAG_ZERO_SKIP);
        }
        if (kind == KIND_INLET) {
            if constexpr (Q == 19) zou_he<C>(s, a.inlet_normal, a.inlet_vel);
        } else if (kind == KIND_OUTLET) {
            const int k = a.aux[n];
            if (a.out_src[k] != -1) {
#pragma unroll
                for (int q = 0; q < Q; ++q) s[q] = a.out_buf[(long long)k * Q + q];
            }
        } else if (kind == KIND_WALL) {
            wall_fixup<C, Q>(s, m);
        }
    }

    if (OBS & 1) {
#pragma unroll
        for (int q = 0; q < Q; ++q)
            a.obs_pop[(long long)q * a.ld + n] = Store<S>::SHIFTED ? (double)s[q] + L::w(q) : (double)s[q];
    }

    // near-wall nodes hand the boundary pass that computes this step's wall
    // shear stress their arriving populations (FP64) or their second moments
    // and, after the collision, its moments (the shifted types)
    const bool nw = (m >> Meta<Q>::NW_SHIFT) & 1;
    if (nw) {
        const int k = a.aux[n];
        if constexpr (sizeof(C) == 8) {
#pragma unroll
            for (int q = 0; q < Q; ++q) a.nw_s[(long long)q * a.n_nw + k] = s[q];
        } else {
            float P[6];
            second_moments<Q>(s, P, 0.f, [](float x, float y) { return x + y; },
                              [](float x, float y) { return x - y; });
#pragma unroll
            for (int j = 0; j < 6; ++j) a.nw_s[(long long)j * a.n_nw + k] = P[j];
        }
    }

    C c[Q], m0, u[3];
    collide<C, Q>(s, BC == BC_REFERENCE && kind == KIND_WALL, a.omega, c, m0, u);
    if (!isfinite((double)m0)) atomicOr(a.flags, FLAG_NONFINITE);
    if constexpr (sizeof(C) != 8) {
        // a near-wall node is never a wall node: u is its velocity
        if (nw) {
            C* h = a.nw_s + (long long)HANDOFF_MOM_ROW * a.n_nw + a.aux[n];
            h[0] = m0;
            h[a.n_nw] = u[0];
            h[2 * (long long)a.n_nw] = u[1];
            h[3 * (long long)a.n_nw] = u[2];
        }
    }

    if (OBS & 2) {
        a.obs_mom[n] = Store<S>::SHIFTED ? 1.0 + (double)m0 : (double)m0;
        a.obs_mom[a.ld + n] = (double)u[0];
        a.obs_mom[2 * a.ld + n] = (double)u[1];
        a.obs_mom[3 * a.ld + n] = (double)u[2];
    }

    // Values for links whose far end is missing: reference mode keeps the
    // node's own pre-collision value of the opposite direction; physics mode
    // bounces the post-collision population back (the open-boundary pass then
    // corrects inlet and outlet links, and needs the outlet node's velocity).
    C back[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) back[q] = BC == BC_REFERENCE ? s[L::opp(q)] : c[q];
    if constexpr (BC == BC_PHYSICS) {
        if (kind == KIND_OUTLET) {
            double* o = a.io_u + 3 * (long long)a.aux[n];
            o[0] = (double)u[0];
            o[1] = (double)u[1];
            o[2] = (double)u[2];
        }
    }

    if (PHASE == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int oq = L::opp(q);
            const C v = (q == L::REST || ((m >> q) & 1)) ? c[q] : back[q];
            Store<S>::put(a.pop + (long long)oq * a.ld + n, v);
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (q == L::REST) {
                Store<S>::put(a.pop + (long long)q * a.ld + n, c[q]);
            } else {
                if ((m >> q) & 1) Store<S>::put(a.pop + (long long)q * a.ld + (n + sd[q]), c[q]);
                const int oq = L::opp(q);
                // slot (n, oq) is free when the node n - c_oq = n + c_q is missing
                if (!((m >> q) & 1)) Store<S>::put(a.pop + (long long)oq * a.ld + n, back[q]);
            }
        }
    }
}

// Initialisation from natural-layout populations f (double) in obs_pop: one
// collision and a phase-0 store, so the next step reads phase 1. Writes the
// moments of the given state to obs_mom.
template <class S, int Q, int BC>
__global__ void __launch_bounds__(BLOCK_NODES) init_kernel(StepArgs<S, Q> a) {
    using L = Lat<Q>;
    using C = typename Store<S>::C;
    using MT = typename Meta<Q>::T;
    const int n = blockIdx.x * BLOCK_NODES + threadIdx.x;
    if (n >= a.n) return;
    const MT m = a.meta[n];
    const int kind = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);
    C s[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double f = a.obs_pop[(long long)q * a.ld + n];
        s[q] = Store<S>::SHIFTED ? (C)(f - L::w(q)) : (C)f;
        // round through the storage type so every later step sees stored values
        S tmp;
        Store<S>::put(&tmp, s[q]);
        s[q] = Store<S>::get(&tmp);
    }
    C c[Q], m0, u[3];
    collide<C, Q>(s, BC == BC_REFERENCE && kind == KIND_WALL, a.omega, c, m0, u);
    a.obs_mom[n] = Store<S>::SHIFTED ? 1.0 + (double)m0 : (double)m0;
    a.obs_mom[a.ld + n] = (double)u[0];
    a.obs_mom[2 * a.ld + n] = (double)u[1];
    a.obs_mom[3 * a.ld + n] = (double)u[2];
    if (BC == BC_PHYSICS && kind == KIND_OUTLET) {
        double* o = a.io_u + 3 * (long long)a.aux[n];
        o[0] = (double)u[0];
        o[1] = (double)u[1];
        o[2] = (double)u[2];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int oq = L::opp(q);
        C v = c[q];
        if (q != L::REST && !((m >> q) & 1)) v = BC == BC_REFERENCE ? s[oq] : c[q];
        Store<S>::put(a.pop + (long long)oq * a.ld + n, v);
    }
}

// Open-boundary pass of physics mode, after every store (step or
// initialisation). The store bounced back every population whose far node is
// missing into slot (n, opp q); on inlet and outlet nodes the links that point
// out through the open plane (c_q . n > 0) are corrected here:
//   inlet  (velocity bounce-back): f <- f - 6 w_q (c_q . u_in)
//   outlet (anti-bounce-back at rho_out): f <- -f + 2 w_q rho_out
//          (1 + 4.5 (c_q . u)^2 - 1.5 u^2), u the node's collision velocity.
// Items: inlet nodes, then outlet nodes.
template <class S, int Q>
struct OpenArgs {
    S* pop;
    long long ld;
    const typename Meta<Q>::T* meta;
    int n_in;
    const int* in_node;     // [n_in]
    const double* in_vel;   // [n_in][3] inlet velocity profile
    double in_scale;        // waveform factor of the step the store streams into
    double in_normal[3];    // outward inlet normal
    int n_out;
    const int* out_node;    // [n_out]
    const float* out_nrm;   // [n_out][3] outward normal of each node's outlet
    const double* io_u;     // [n_out][3] velocity of each outlet node
    double out_rho;
};

template <class S, int Q>
__device__ __forceinline__ void open_item(const OpenArgs<S, Q>& a, int i) {
    using L = Lat<Q>;
    using C = typename Store<S>::C;
    const bool inlet = i < a.n_in;
    const int k = inlet ? i : i - a.n_in;
    const int n = inlet ? a.in_node[k] : a.out_node[k];
    const typename Meta<Q>::T m = a.meta[n];
    double nrm[3], uv[3];
    if (inlet) {
        for (int c = 0; c < 3; ++c) {
            nrm[c] = a.in_normal[c];
            uv[c] = a.in_vel[3 * (long long)k + c] * a.in_scale;
        }
    } else {
        for (int c = 0; c < 3; ++c) {
            nrm[c] = a.out_nrm[3 * (long long)k + c];
            uv[c] = a.io_u[3 * (long long)k + c];
        }
    }
    // every corrected slot is read before any is written: the loads go out
    // together instead of one memory round trip per link
    C f_all[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        f_all[q] = C(0);
        if (q == L::REST || ((m >> q) & 1)) continue;
        const double cn = L::cx(q) * nrm[0] + L::cy(q) * nrm[1] + L::cz(q) * nrm[2];
        if (cn > 0.0) f_all[q] = Store<S>::get(a.pop + (long long)L::opp(q) * a.ld + n);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST || ((m >> q) & 1)) continue;
        const double cn = L::cx(q) * nrm[0] + L::cy(q) * nrm[1] + L::cz(q) * nrm[2];
        if (!(cn > 0.0)) continue;
        S* slot = a.pop + (long long)L::opp(q) * a.ld + n;
        const double f = (double)f_all[q];
        const double cu = L::cx(q) * uv[0] + L::cy(q) * uv[1] + L::cz(q) * uv[2];
        double v;
        if (inlet) {
            v = f - 6.0 * L::w(q) * cu;
        } else {
            const double eq = 1.0 + 4.5 * cu * cu - 1.5 * (uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
            // stored deviations: -(w + d) + 2 w rho eq - w = -d + 2 w (rho eq - 1)
            v = Store<S>::SHIFTED ? -f + 2.0 * L::w(q) * (a.out_rho * eq - 1.0) : -f + 2.0 * L::w(q) * a.out_rho * eq;
        }
        Store<S>::put(slot, (C)v);
    }
}

template <class S, int Q>
__global__ void open_boundary_kernel(OpenArgs<S, Q> a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n_in + a.n_out) open_item<S, Q>(a, i);
}


// Boundary pass, launched before the step kernel of each step:
//  * items [0, n_wss): wall shear stress of the previous step's near-wall
//    nodes, from the populations that step's kernel handed over;
//  * then one item per (outlet node, direction): the source population of
//    the outlet copy (post-streaming, post-inlet value of the node the
//    reference's in-order copy sweep ends up reading), gathered before the
//    step kernel overwrites it. A source that is itself an inlet node needs
//    its Zou-He update first, so one thread does that whole node.
template <class S, int Q, int PHASE>
__global__ void boundary_kernel(BoundaryArgs<S, Q> a) {
    using C = typename Store<S>::C;
    using MT = typename Meta<Q>::T;
    using L = Lat<Q>;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n_wss) {
        wall_shear<S, Q>(a, (int)i);
        return;
    }
    const long long j = i - a.n_wss;
    if (j >= (long long)a.n_out * Q) return;
    const int k = (int)(j / Q), q = (int)(j % Q);
    const int src = a.out_src[k];
    if (src == -1) return;
    if (src <= -2) {
        if (q != 0) return;
        const int n = -(src + 2);
        const MT m = a.meta[n];
        const int* sd = PHASE == 1 ? seg_row<Q>(a.seg_base, a.seg_delta, n, m) : nullptr;
        C s[Q];
        gather<S, Q, PHASE>(a.pop, a.ld, n, m, sd, s);
        if constexpr (Q == 19) zou_he<C>(s, a.inlet_normal, a.inlet_vel);
#pragma unroll
        for (int d = 0; d < Q; ++d) a.out_buf[(long long)k * Q + d] = s[d];
        return;
    }
    const MT m = a.meta[src];
    long long idx = (long long)q * a.ld + src;
    if (PHASE == 1 && q != L::REST) {
        const int oq = L::opp(q);
        if ((m >> oq) & 1) idx = (long long)oq * a.ld + (src + seg_row<Q>(a.seg_base, a.seg_delta, src, m)[oq]);
    }
    a.out_buf[(long long)k * Q + q] = Store<S>::get(a.pop + idx);
}

// Physics-mode pass after each step kernel: the open-boundary corrections of
// its store (items [0, n_in + n_out): one per inlet / outlet node) and the
// wall shear stress of the step just taken (then one item per near-wall
// node). The two touch disjoint data (the inlet and outlet nodes' bounce-back
// slots; the near-wall hand-off buffers and accumulators), so one launch does
// both; the open-boundary items, the longer ones, go first so that they do not
// trail the launch.
template <class S, int Q>
__global__ void post_kernel(BoundaryArgs<S, Q> b, OpenArgs<S, Q> o) {
    allow_next_grid();
    wait_prior_grid();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n_open = (long long)o.n_in + o.n_out;
    if (i < n_open) {
        open_item<S, Q>(o, (int)i);
        return;
    }
    if (i - n_open < b.n_wss) wall_shear<S, Q>(b, (int)(i - n_open));
}

}  // namespace lbm
