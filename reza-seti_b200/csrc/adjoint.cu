// Hand-written discrete adjoint of the physics-mode time step (halfway
// bounce-back walls, velocity bounce-back inlet, anti-bounce-back pressure
// outlet), D3Q19 and D3Q27, FP32 or FP64.
//
// Forward model. State f^t (stored as deviations d = f - w, two lattices in
// natural layout [q][ld] so that past states can be kept); for t = 0..T-1 each
// node collides and pushes its populations:
//   c_q      = d_q + omega (deq_q(d) - d_q)                         (BGK)
//   f^{t+1}[n + c_q][q]  = c_q                  where that node exists,
//   f^{t+1}[n][opp q]    = c_q                  (halfway bounce-back) otherwise,
//     + 6 w_q (c_q . n_in) v(n) s_t             on inlet links (c_q . n_in > 0),
//     or -c_q + 2 w_q (rho_out eq_q(u) - 1)     on outlet links (c_q . n_out > 0),
//   with eq_q(u) = 1 + 4.5 (c_q.u)^2 - 1.5 u^2, u the velocity of f^t at n,
//   v(n) the inlet speed (along -n_in) and s_t the waveform factor of step t.
// This is the engine's physics step (same links, same corrections) written as
// a push. Objective, over the target near-wall nodes k:
//   J = (1/T) sum_{t=1..T} sum_k |tau_k^t|^2,
//   tau^t = C_w sum_q (f^t_q - feq_q(f^{t-1})) M_q,  M_q = (c_q.n)(c_q - (c_q.n) n)
// which is the engine's wall shear stress of step t (its f_eq comes from the
// previous state's moments).
//
// Reverse sweep: lambda^t = dJ/df^t, from lambda^{t+1} (pull form of the push):
//   mu_q     = lambda^{t+1}[n + c_q][q], or the bounce-back link's
//              lambda^{t+1}[n][opp q] (negated on outlet links);
//   lambda_q = (1 - omega) mu_q + omega (A + B . c_q) + G . (c_q - u) / rho
//              + dJ_t/df^t_q + dJ_{t+1}/df^t_q (target nodes),
//   A = sum_r mu_r w_r (1 - 4.5 (c_r.u)^2 + 1.5 u^2),
//   B = sum_r mu_r w_r (3 c_r + 9 (c_r.u) c_r - 3 u)   (Jacobian of feq through rho, j),
//   G = sum over outlet links of lambda 2 w_r rho_out (9 (c_r.u) c_r - 3 u);
//   dJ/domega += sum_q mu_q (deq_q - d_q);  dJ/dv(n) += lambda 6 w_q (c_q.n_in) s_t.
// Memory: f^t is checkpointed every K steps; the reverse sweep recomputes each
// segment's K states from its checkpoint (the last segment is kept from the
// forward sweep) and walks it backwards. Gradient sums are FP64.
#include <algorithm>
#include <cmath>

#include "adjoint.h"
#include "lattice.cuh"

namespace lbm {
namespace {

constexpr int AT = 256;  // threads per block of the node kernels

template <class R, int Q>
struct AGeom {
    using MT = typename Meta<Q>::T;
    long long ld;
    int n;
    const MT* meta;
    const int* seg_base;
    const int* seg_delta;
    const int* aux;
    double in_normal[3];
    const double* speed;    // [n_in]
    const float* out_nrm;   // [n_out][3]
    double out_rho;
    R omega;
};

template <int Q>
__device__ __forceinline__ const int* nbr_row(const int* seg_base, const int* seg_delta, int n,
                                              typename Meta<Q>::T m) {
    const int s = __ldg(seg_base + n / BLOCK_NODES) + (int)(m >> Meta<Q>::SEG_SHIFT);
    return seg_delta + (long long)s * Q;
}

template <class R, int Q>
__device__ __forceinline__ void dmoments(const R d[Q], R& drho, R u[3]) {
    using L = Lat<Q>;
    drho = R(0);
    R j[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        drho += d[q];
        if (L::cx(q)) j[0] += L::cx(q) > 0 ? d[q] : -d[q];
        if (L::cy(q)) j[1] += L::cy(q) > 0 ? d[q] : -d[q];
        if (L::cz(q)) j[2] += L::cz(q) > 0 ? d[q] : -d[q];
    }
    const R inv = R(1) / (R(1) + drho);
    u[0] = j[0] * inv;
    u[1] = j[1] * inv;
    u[2] = j[2] * inv;
}

// feq_q - w_q
template <class R, int Q>
__device__ __forceinline__ R deq(int q, R drho, const R u[3]) {
    using L = Lat<Q>;
    const R cu = R(L::cx(q)) * u[0] + R(L::cy(q)) * u[1] + R(L::cz(q)) * u[2];
    const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    return R(L::w(q)) * (drho + (R(1) + drho) * (R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq));
}

// sum_r g_r d feq_r / d f_q = A + B . c_q
template <class R, int Q>
__device__ __forceinline__ void feq_adjoint(const R g[Q], const R u[3], R& A, R B[3]) {
    using L = Lat<Q>;
    const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    A = R(0);
    B[0] = B[1] = B[2] = R(0);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const R c0 = R(L::cx(q)), c1 = R(L::cy(q)), c2 = R(L::cz(q));
        const R cu = c0 * u[0] + c1 * u[1] + c2 * u[2];
        const R gw = g[q] * R(L::w(q));
        A += gw * (R(1) - R(4.5) * cu * cu + R(1.5) * usq);
        const R k = R(3) + R(9) * cu;
        B[0] += gw * (k * c0 - R(3) * u[0]);
        B[1] += gw * (k * c1 - R(3) * u[1]);
        B[2] += gw * (k * c2 - R(3) * u[2]);
    }
}

// tau = C_w sum_q fne_q (c_q.n)(c_q - (c_q.n) n), in FP64
template <int Q, class R>
__device__ __forceinline__ void traction(const R fne[Q], const double nrm[3], double cw, double tau[3]) {
    using L = Lat<Q>;
    double t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
        const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
        const double f = (double)fne[q] * cn;
        t0 += f * (c0 - cn * nrm[0]);
        t1 += f * (c1 - cn * nrm[1]);
        t2 += f * (c2 - cn * nrm[2]);
    }
    tau[0] = cw * t0;
    tau[1] = cw * t1;
    tau[2] = cw * t2;
}

// dJ/dfne_q = scale tau . M_q
template <int Q, class R>
__device__ __forceinline__ void traction_adjoint(const double tau[3], const double nrm[3], double scale, R g[Q]) {
    using L = Lat<Q>;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
        const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
        const double d = tau[0] * (c0 - cn * nrm[0]) + tau[1] * (c1 - cn * nrm[1]) + tau[2] * (c2 - cn * nrm[2]);
        g[q] = (R)(scale * cn * d);
    }
}

// Sum over the block (blockDim.x a multiple of 32, at most 32 warps); the
// result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;
}

// d = f - w, rounded to R
template <class R, int Q>
__global__ void adj_load_kernel(const double* __restrict__ f, long long ld, int n, R* __restrict__ D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int q = 0; q < Q; ++q) D[(long long)q * ld + i] = (R)(f[(long long)q * ld + i] - Lat<Q>::w(q));
}

template <class R, int Q>
__global__ void adj_store_kernel(const R* __restrict__ D, long long ld, int n, double* __restrict__ f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int q = 0; q < Q; ++q) f[(long long)q * ld + i] = (double)D[(long long)q * ld + i] + Lat<Q>::w(q);
}

// One forward step: collide f^t at each node and push it into f^{t+1}.
template <class R, int Q>
__global__ void __launch_bounds__(AT) adj_push_kernel(AGeom<R, Q> g, const R* __restrict__ D, R* __restrict__ Dn,
                                                       double s_t) {
    using L = Lat<Q>;
    const int n = blockIdx.x * AT + threadIdx.x;
    if (n >= g.n) return;
    const auto m = g.meta[n];
    const int kind = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);
    R d[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) d[q] = D[(long long)q * g.ld + n];
    R drho, u[3];
    dmoments<R, Q>(d, drho, u);
    const int* sd = nbr_row<Q>(g.seg_base, g.seg_delta, n, m);
    double nrm[3] = {0, 0, 0};
    double vin = 0.0;
    if (kind == KIND_INLET) {
        for (int c = 0; c < 3; ++c) nrm[c] = g.in_normal[c];
        vin = g.speed[g.aux[n]] * s_t;
    } else if (kind == KIND_OUTLET) {
        for (int c = 0; c < 3; ++c) nrm[c] = g.out_nrm[3 * (long long)g.aux[n] + c];
    }
    const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const R c = d[q] + g.omega * (deq<R, Q>(q, drho, u) - d[q]);
        if (q == L::REST) {
            Dn[(long long)q * g.ld + n] = c;
        } else if ((m >> q) & 1) {
            Dn[(long long)q * g.ld + (n + sd[q])] = c;
        } else {
            R v = c;
            const double cn = L::cx(q) * nrm[0] + L::cy(q) * nrm[1] + L::cz(q) * nrm[2];
            if (cn > 0.0) {
                if (kind == KIND_INLET) {
                    v = c + (R)(6.0 * L::w(q) * cn * vin);
                } else {
                    const R cu = R(L::cx(q)) * u[0] + R(L::cy(q)) * u[1] + R(L::cz(q)) * u[2];
                    const R eq = R(1) + R(4.5) * cu * cu - R(1.5) * usq;
                    v = -c + R(2.0 * L::w(q)) * (R(g.out_rho) * eq - R(1));
                }
            }
            Dn[(long long)L::opp(q) * g.ld + n] = v;
        }
    }
}

template <class R, int Q>
struct ObjArgs {
    long long ld;
    int n_target;
    const int* node;         // [n_target] internal node
    const int* nw;           // [n_target] near-wall entry
    const double* nw_normal; // [n_nw][3]
    double* mom;             // [T + 1][n_target][4]: drho, u of f^t
    double cw, inv_T;
    double* J;
};

// Objective term of step t at the target nodes (forward sweep): records the
// moments of f^t and adds |tau^t|^2 / T for t >= 1.
template <class R, int Q>
__global__ void adj_objective_kernel(ObjArgs<R, Q> a, const R* __restrict__ D, int t) {
    __shared__ double red[4];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double jl = 0.0;
    if (k < a.n_target) {
        const int n = a.node[k];
        R d[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q] = D[(long long)q * a.ld + n];
        R drho, u[3];
        dmoments<R, Q>(d, drho, u);
        double* mt = a.mom + ((long long)t * a.n_target + k) * 4;
        if (t >= 1) {
            const double* mp = mt - 4 * (long long)a.n_target;
            const R up[3] = {(R)mp[1], (R)mp[2], (R)mp[3]};
            R fne[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) fne[q] = d[q] - deq<R, Q>(q, (R)mp[0], up);
            double tau[3];
            traction<Q>(fne, a.nw_normal + 3 * (long long)a.nw[k], a.cw, tau);
            jl = a.inv_T * (tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
        }
        mt[0] = (double)drho;
        mt[1] = (double)u[0];
        mt[2] = (double)u[1];
        mt[3] = (double)u[2];
    }
    const double s = block_sum(jl, red);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(a.J, s);
}

// lambda^t from lambda^{t+1} at every node (the transpose of the push). One
// pass gathers mu (bounce-back links take the node's own lambda^{t+1}, negated
// on outlet links) while it accumulates the moments of f^t and sum mu d; the
// outlet velocity terms and the collision Jacobian follow from mu alone, so
// the node's populations are never held as an array.
template <class R, int Q>
__global__ void __launch_bounds__(AT) adj_pull_kernel(AGeom<R, Q> g, const R* __restrict__ D,
                                                       const R* __restrict__ Ln, R* __restrict__ Lc, double s_t,
                                                       double* __restrict__ dspeed, double* __restrict__ domega) {
    using L = Lat<Q>;
    __shared__ double red[AT / 32];
    const int n = blockIdx.x * AT + threadIdx.x;
    double wl = 0.0;
    if (n < g.n) {
        const auto m = g.meta[n];
        const int kind = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);
        const int* sd = nbr_row<Q>(g.seg_base, g.seg_delta, n, m);
        R nrm[3] = {R(0), R(0), R(0)};
        if (kind == KIND_INLET) {
            for (int c = 0; c < 3; ++c) nrm[c] = (R)g.in_normal[c];
        } else if (kind == KIND_OUTLET) {
            for (int c = 0; c < 3; ++c) nrm[c] = (R)g.out_nrm[3 * (long long)g.aux[n] + c];
        }
        R mu[Q];
        R drho = R(0), j0 = R(0), j1 = R(0), j2 = R(0), mud = R(0), gin = R(0);
        unsigned out_links = 0;  // bit q: q is an outlet link (mu_q = -lambda)
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const R dq = D[(long long)q * g.ld + n];
            drho += dq;
            if (L::cx(q)) j0 += L::cx(q) > 0 ? dq : -dq;
            if (L::cy(q)) j1 += L::cy(q) > 0 ? dq : -dq;
            if (L::cz(q)) j2 += L::cz(q) > 0 ? dq : -dq;
            R v;
            if (q == L::REST) {
                v = Ln[(long long)q * g.ld + n];
            } else if ((m >> q) & 1) {
                v = Ln[(long long)q * g.ld + (n + sd[q])];
            } else {
                v = Ln[(long long)L::opp(q) * g.ld + n];
                const R cn = R(L::cx(q)) * nrm[0] + R(L::cy(q)) * nrm[1] + R(L::cz(q)) * nrm[2];
                if (cn > R(0)) {
                    if (kind == KIND_INLET) {
                        gin += v * R(6.0 * L::w(q)) * cn;
                    } else {
                        v = -v;
                        out_links |= 1u << q;
                    }
                }
            }
            mu[q] = v;
            mud += v * dq;
        }
        const R irho = R(1) / (R(1) + drho);
        const R u[3] = {j0 * irho, j1 * irho, j2 * irho};
        // outlet links: d/du of 2 w rho_out eq(u), times lambda = -mu
        R G[3] = {R(0), R(0), R(0)};
        if (out_links) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                if (!((out_links >> q) & 1)) continue;
                const R c0 = R(L::cx(q)), c1 = R(L::cy(q)), c2 = R(L::cz(q));
                const R cu = c0 * u[0] + c1 * u[1] + c2 * u[2];
                const R k = -mu[q] * R(2.0 * L::w(q) * g.out_rho);
                G[0] += k * (R(9) * cu * c0 - R(3) * u[0]);
                G[1] += k * (R(9) * cu * c1 - R(3) * u[1]);
                G[2] += k * (R(9) * cu * c2 - R(3) * u[2]);
            }
        }
        R A, B[3];
        feq_adjoint<R, Q>(mu, u, A, B);
        const R om = g.omega;
        const R gu = G[0] * u[0] + G[1] * u[1] + G[2] * u[2];
        R mueq = R(0);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            mueq += mu[q] * deq<R, Q>(q, drho, u);
            const R cb = R(L::cx(q)) * B[0] + R(L::cy(q)) * B[1] + R(L::cz(q)) * B[2];
            const R cg = R(L::cx(q)) * G[0] + R(L::cy(q)) * G[1] + R(L::cz(q)) * G[2];
            Lc[(long long)q * g.ld + n] = (R(1) - om) * mu[q] + om * (A + cb) + (cg - gu) * irho;
        }
        wl = (double)(mueq - mud);
        if (kind == KIND_INLET) dspeed[g.aux[n]] += (double)gin * s_t;
    }
    const double s = block_sum(wl, red);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(domega, s);
}

// Objective terms of lambda^t at the target nodes: dJ_t/df^t (t >= 1) and
// dJ_{t+1}/df^t through the f_eq of tau^{t+1} (t < T).
template <class R, int Q>
__global__ void adj_objective_adjoint_kernel(ObjArgs<R, Q> a, const R* __restrict__ D, const R* __restrict__ Dn,
                                             R* __restrict__ Lc, int t, int T) {
    using L = Lat<Q>;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n_target) return;
    const int n = a.node[k];
    const double* nrm = a.nw_normal + 3 * (long long)a.nw[k];
    const double scale = 2.0 * a.inv_T * a.cw;
    R acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) acc[q] = R(0);
    if (t >= 1) {
        const double* mp = a.mom + ((long long)(t - 1) * a.n_target + k) * 4;
        const R up[3] = {(R)mp[1], (R)mp[2], (R)mp[3]};
        R fne[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) fne[q] = D[(long long)q * a.ld + n] - deq<R, Q>(q, (R)mp[0], up);
        double tau[3];
        traction<Q>(fne, nrm, a.cw, tau);
        traction_adjoint<Q>(tau, nrm, scale, acc);
    }
    if (t < T) {
        const double* mt = a.mom + ((long long)t * a.n_target + k) * 4;
        const R ut[3] = {(R)mt[1], (R)mt[2], (R)mt[3]};
        R fne[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) fne[q] = Dn[(long long)q * a.ld + n] - deq<R, Q>(q, (R)mt[0], ut);
        double tau[3];
        traction<Q>(fne, nrm, a.cw, tau);
        R gq[Q];
        traction_adjoint<Q>(tau, nrm, scale, gq);
        R A, B[3];
        feq_adjoint<R, Q>(gq, ut, A, B);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            acc[q] -= A + R(L::cx(q)) * B[0] + R(L::cy(q)) * B[1] + R(L::cz(q)) * B[2];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) Lc[(long long)q * a.ld + n] += acc[q];
}

struct Arena {
    std::vector<void*> ptrs;
    size_t bytes = 0;
    cudaError_t err = cudaSuccess;
    template <class T>
    T* get(size_t count) {
        if (err != cudaSuccess) return nullptr;
        void* p = nullptr;
        const size_t b = std::max<size_t>(count, 1) * sizeof(T);
        err = cudaMalloc(&p, b);
        if (err != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        bytes += b;
        return (T*)p;
    }
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

struct Events {
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    Events() {
        for (auto& x : e) cudaEventCreate(&x);
    }
    ~Events() {
        for (auto& x : e)
            if (x) cudaEventDestroy(x);
    }
};

template <class R, int Q>
int run(const AdjointSetup& s, AdjointOut& o) {
    using MT = typename Meta<Q>::T;
    const int64_t T = s.n_steps;
    const int64_t K = s.gradient ? std::max<int64_t>(1, std::min<int64_t>(s.checkpoint_every, T)) : T;
    const int64_t nseg = s.gradient ? (T + K - 1) / K : 1;
    const int nt = (int)s.targets.size();
    const size_t field = (size_t)Q * s.ld;
    cudaStream_t st = s.stream;
    Arena ar;
    // seg[j] holds f^{t0 + j} of the current segment; with gradients seg[0]
    // points at the segment's checkpoint
    std::vector<R*> seg((size_t)(s.gradient ? K + 1 : 2), nullptr);
    for (size_t j = s.gradient ? 1 : 0; j < seg.size(); ++j) seg[j] = ar.get<R>(field);
    std::vector<R*> ck((size_t)(s.gradient ? nseg : 0));
    for (auto& p : ck) p = ar.get<R>(field);
    R* lam[2] = {nullptr, nullptr};
    if (s.gradient) {
        lam[0] = ar.get<R>(field);
        lam[1] = ar.get<R>(field);
    }
    double* mom = ar.get<double>((size_t)(T + 1) * std::max(nt, 1) * 4);
    double* speed = ar.get<double>(std::max(s.n_in, 1));
    double* dspeed = ar.get<double>(std::max(s.n_in, 1));
    double* scal = ar.get<double>(2);
    int* tnode = ar.get<int>(std::max(nt, 1));
    int* tnw = ar.get<int>(std::max(nt, 1));
    if (ar.err != cudaSuccess) {
        o.err = std::string("adjoint buffers (") + std::to_string(ar.bytes >> 20) + " MiB allocated before): " +
                cudaGetErrorString(ar.err);
        return -2;
    }
    o.bytes = ar.bytes;
    {
        std::vector<int> tn(std::max(nt, 1)), tw(std::max(nt, 1));
        std::vector<int> nw_node(s.n_nw);
        if (s.n_nw) cudaMemcpy(nw_node.data(), s.nw_node, sizeof(int) * s.n_nw, cudaMemcpyDeviceToHost);
        for (int k = 0; k < nt; ++k) {
            tw[k] = s.targets[k];
            tn[k] = nw_node[s.targets[k]];
        }
        cudaMemcpyAsync(tnode, tn.data(), sizeof(int) * tn.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(tnw, tw.data(), sizeof(int) * tw.size(), cudaMemcpyHostToDevice, st);
        if (s.n_in) cudaMemcpyAsync(speed, s.speed.data(), sizeof(double) * s.n_in, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(dspeed, 0, sizeof(double) * std::max(s.n_in, 1), st);
        cudaMemsetAsync(scal, 0, 2 * sizeof(double), st);
        // the host vectors above die at the end of this block
        cudaError_t ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) {
            o.err = std::string("adjoint setup: ") + cudaGetErrorString(ce);
            return -2;
        }
    }
    AGeom<R, Q> g{};
    g.ld = s.ld;
    g.n = s.n;
    g.meta = (const MT*)s.meta;
    g.seg_base = s.seg_base;
    g.seg_delta = s.seg_delta;
    g.aux = s.aux;
    for (int c = 0; c < 3; ++c) g.in_normal[c] = s.in_normal[c];
    g.speed = speed;
    g.out_nrm = s.out_nrm;
    g.out_rho = s.out_rho;
    g.omega = (R)(1.0 / s.tau);
    ObjArgs<R, Q> oa{};
    oa.ld = s.ld;
    oa.n_target = nt;
    oa.node = tnode;
    oa.nw = tnw;
    oa.nw_normal = s.nw_normal;
    oa.mom = mom;
    oa.cw = s.wss_c;
    oa.inv_T = 1.0 / (double)T;
    oa.J = scal;

    const dim3 grid((unsigned)((s.n + AT - 1) / AT));
    const unsigned tgrid = (unsigned)((nt + 127) / 128);
    auto push = [&](const R* D, R* Dn, int64_t t) {
        adj_push_kernel<R, Q><<<grid, AT, 0, st>>>(g, D, Dn, s.factors[t]);
    };
    auto objective = [&](const R* D, int64_t t) {
        if (nt) adj_objective_kernel<R, Q><<<tgrid, 128, 0, st>>>(oa, D, (int)t);
    };
    Events ev;
    cudaEventRecord(ev.e[0], st);
    const R* fT = nullptr;
    if (!s.gradient) {
        adj_load_kernel<R, Q><<<grid, AT, 0, st>>>(s.f0, s.ld, s.n, seg[0]);
        for (int64_t t = 0; t < T; ++t) {
            objective(seg[0], t);
            push(seg[0], seg[1], t);
            std::swap(seg[0], seg[1]);
        }
        objective(seg[0], T);
        fT = seg[0];
    } else {
        // forward sweep: f^{sK} into ck[s]; the last segment's states stay in seg
        adj_load_kernel<R, Q><<<grid, AT, 0, st>>>(s.f0, s.ld, s.n, ck[0]);
        for (int64_t sg = 0; sg < nseg; ++sg) {
            const int64_t t0 = sg * K, t1 = std::min(T, t0 + K);
            seg[0] = ck[sg];
            for (int64_t t = t0; t < t1; ++t) {
                objective(seg[t - t0], t);
                push(seg[t - t0], seg[t - t0 + 1], t);
            }
            if (sg + 1 < nseg)
                cudaMemcpyAsync(ck[sg + 1], seg[t1 - t0], field * sizeof(R), cudaMemcpyDeviceToDevice, st);
        }
        const int64_t tl = (nseg - 1) * K;
        objective(seg[T - tl], T);
        fT = seg[T - tl];
    }
    if (s.final_pop) adj_store_kernel<R, Q><<<grid, AT, 0, st>>>(fT, s.ld, s.n, s.final_pop);
    cudaEventRecord(ev.e[1], st);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        o.err = std::string("adjoint forward sweep: ") + cudaGetErrorString(ce);
        cudaStreamSynchronize(st);
        return -2;
    }
    if (s.gradient) {
        // reverse sweep, segment by segment
        R* Lnext = lam[0];
        R* Lcur = lam[1];
        for (int64_t sg = nseg - 1; sg >= 0; --sg) {
            const int64_t t0 = sg * K, t1 = std::min(T, t0 + K);
            seg[0] = ck[sg];
            if (sg + 1 < nseg) {
                for (int64_t t = t0; t < t1; ++t) push(seg[t - t0], seg[t - t0 + 1], t);
                o.steps_recomputed += t1 - t0;
            }
            // lambda^{t1} of an earlier segment was finished by the later one
            for (int64_t t = (t1 == T ? T : t1 - 1); t >= t0; --t) {
                if (t == T) {
                    cudaMemsetAsync(Lcur, 0, field * sizeof(R), st);
                } else {
                    adj_pull_kernel<R, Q><<<grid, AT, 0, st>>>(g, seg[t - t0], Lnext, Lcur, s.factors[t], dspeed,
                                                                scal + 1);
                }
                if (nt)
                    adj_objective_adjoint_kernel<R, Q><<<tgrid, 128, 0, st>>>(
                        oa, seg[t - t0], t < T ? seg[t - t0 + 1] : nullptr, Lcur, (int)t, (int)T);
                std::swap(Lnext, Lcur);
            }
        }
        ce = cudaGetLastError();
        if (ce != cudaSuccess) {
            o.err = std::string("adjoint reverse sweep: ") + cudaGetErrorString(ce);
            cudaStreamSynchronize(st);
            return -2;
        }
    }
    cudaEventRecord(ev.e[2], st);
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
        o.err = std::string("adjoint run: ") + cudaGetErrorString(ce);
        return -2;
    }
    cudaEventElapsedTime(&o.forward_ms, ev.e[0], ev.e[1]);
    if (s.gradient) cudaEventElapsedTime(&o.reverse_ms, ev.e[1], ev.e[2]);
    double hs[2] = {0, 0};
    cudaMemcpy(hs, scal, sizeof(hs), cudaMemcpyDeviceToHost);
    o.J = hs[0];
    o.dJ_domega = hs[1];
    o.dJ_dspeed.assign(s.n_in, 0.0);
    if (s.gradient && s.n_in)
        cudaMemcpy(o.dJ_dspeed.data(), dspeed, sizeof(double) * s.n_in, cudaMemcpyDeviceToHost);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        o.err = std::string("adjoint results: ") + cudaGetErrorString(ce);
        return -2;
    }
    return 0;
}

}  // namespace

int adjoint_run(const AdjointSetup& s, AdjointOut& o) {
    if (s.Q != 19 && s.Q != 27) {
        o.err = "adjoint: lattice must be D3Q19 or D3Q27";
        return -1;
    }
    if (s.n_steps < 1 || (int64_t)s.factors.size() != s.n_steps) {
        o.err = "adjoint: need at least one step and one waveform factor per step";
        return -1;
    }
    if (s.n_steps > (int64_t)1 << 30) {
        o.err = "adjoint: too many steps";
        return -1;
    }
    if ((int)s.speed.size() != s.n_in) {
        o.err = "adjoint: one inlet speed per inlet node";
        return -1;
    }
    std::vector<char> seen(s.n_nw, 0);
    for (int k : s.targets) {
        if (k < 0 || k >= s.n_nw) {
            o.err = "adjoint: target outside the near-wall list";
            return -1;
        }
        if (seen[k]) {
            o.err = "adjoint: target listed twice";
            return -1;
        }
        seen[k] = 1;
    }
    if (s.Q == 19) return s.fp64 ? run<double, 19>(s, o) : run<float, 19>(s, o);
    return s.fp64 ? run<double, 27>(s, o) : run<float, 27>(s, o);
}

}  // namespace lbm
