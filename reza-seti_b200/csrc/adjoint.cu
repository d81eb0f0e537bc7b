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
// a push. Objective, over the target near-wall nodes k, either the
// time-averaged squared wall shear
//   J = (1/T) sum_{t=1..T} sum_k |tau_k^t|^2,
// or the mean oscillatory shear index
//   J = (1/n) sum_k (1 - |A_k| / M_k) / 2,  A_k = sum_t tau_k^t, M_k = sum_t |tau_k^t|
// (dJ/dtau_k^t = dJ/dA_k + dJ/dM_k tau_k^t / |tau_k^t|, with the sums taken
// from the forward sweep), where
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

#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "adjoint.h"
#include "lattice.cuh"
#include "pair.cuh"

namespace lbm {
namespace {

constexpr int AT = 256;  // threads per block of the node kernels

// Resident CTAs per SM the FP32 pair kernels are compiled for (caps their
// registers): push 6 (80 registers), pull 5 (96 registers, a few spilled:
// faster than 4 at 128 registers, while 6 spills heavily).
#ifndef LBM_ADJ_PUSH_MIN_BLOCKS
#define LBM_ADJ_PUSH_MIN_BLOCKS 6
#endif
#ifndef LBM_ADJ_PULL_MIN_BLOCKS
#define LBM_ADJ_PULL_MIN_BLOCKS 5
#endif

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
    // target index of each near-wall entry (-1: not a target), for the pull
    // kernel that adds the objective's term to lambda at the targets
    const int* nw_target;
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

// FP64 sums without block barriers: each warp adds its total to one of
// N_PARTIALS slots (spread to avoid contention on one address); the host adds
// the slots at the end of the run.
constexpr int N_PARTIALS = 1024;

// Sum over the warp, valid in every lane (all 32 lanes active).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void warp_accumulate(double v, double* partials) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v != 0.0) {
        const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        atomicAdd(partials + (w & (N_PARTIALS - 1)), v);
    }
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
    int osi;                 // objective: 0 time-averaged WSS^2, 1 mean OSI
    double* acc;             // OSI: [n_target][4] sum of tau (3) and of |tau|
    const double* coef;      // OSI: [n_target][4] dJ/dtau^t = coef[0..2] + coef[3] tau^t / |tau^t|
};

// dJ/dtau^t of one target for the objective
__device__ __forceinline__ void objective_dtau(int osi, const double* coef, double inv_T, const double tau[3],
                                               double out[3]) {
    if (!osi) {
        for (int c = 0; c < 3; ++c) out[c] = 2.0 * inv_T * tau[c];
        return;
    }
    const double m = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
    const double k = m > 0.0 ? coef[3] / m : 0.0;
    for (int c = 0; c < 3; ++c) out[c] = coef[c] + k * tau[c];
}

// Objective term of step t at the target nodes (forward sweep), one warp per
// target and one lane per direction: records the moments of f^t and adds
// |tau^t|^2 / T for t >= 1.
template <class R, int Q>
__device__ __forceinline__ void objective_warp_body(const ObjArgs<R, Q>& a, const R* __restrict__ D, int t,
                                                    int bid) {
    using L = Lat<Q>;
    const int lane = threadIdx.x & 31;
    const int k = bid * (blockDim.x >> 5) + (threadIdx.x >> 5);
    double jl = 0.0;
    if (k < a.n_target) {  // uniform over the warp
        const int n = a.node[k];
        const bool on = lane < Q;
        const int q = on ? lane : 0;
        const R dq = on ? D[(long long)q * a.ld + n] : R(0);
        const double c0 = on ? L::cx(q) : 0, c1 = on ? L::cy(q) : 0, c2 = on ? L::cz(q) : 0;
        const double drho = warp_sum((double)dq);
        const double rho = 1.0 + drho;
        const double u0 = warp_sum(c0 * (double)dq) / rho, u1 = warp_sum(c1 * (double)dq) / rho,
                     u2 = warp_sum(c2 * (double)dq) / rho;
        double* mt = a.mom + ((long long)t * a.n_target + k) * 4;
        if (t >= 1) {
            const double* mp = mt - 4 * (long long)a.n_target;
            const R up[3] = {(R)mp[1], (R)mp[2], (R)mp[3]};
            const double fne = on ? (double)(dq - deq<R, Q>(q, (R)mp[0], up)) : 0.0;
            const double* nrm = a.nw_normal + 3 * (long long)a.nw[k];
            const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
            const double f = fne * cn;
            const double t0 = a.cw * warp_sum(f * (c0 - cn * nrm[0]));
            const double t1 = a.cw * warp_sum(f * (c1 - cn * nrm[1]));
            const double t2 = a.cw * warp_sum(f * (c2 - cn * nrm[2]));
            if (lane == 0) {
                if (a.osi) {
                    double* ac = a.acc + 4 * (long long)k;
                    ac[0] += t0;
                    ac[1] += t1;
                    ac[2] += t2;
                    ac[3] += sqrt(t0 * t0 + t1 * t1 + t2 * t2);
                } else {
                    jl = a.inv_T * (t0 * t0 + t1 * t1 + t2 * t2);
                }
            }
        }
        if (lane == 0) {
            mt[0] = drho;
            mt[1] = u0;
            mt[2] = u1;
            mt[3] = u2;
        }
    }
    warp_accumulate(jl, a.J);
}

template <class R, int Q>
__global__ void adj_objective_kernel(ObjArgs<R, Q> a, const R* __restrict__ D, int t) {
    objective_warp_body<R, Q>(a, D, t, blockIdx.x);
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
    warp_accumulate(wl, domega);
}

// Objective terms of lambda^t at the target nodes, one warp per target and
// one lane per direction: dJ_t/df^t (t >= 1) and dJ_{t+1}/df^t through the
// f_eq of tau^{t+1} (t < T).
template <class R, int Q>
__device__ __forceinline__ void objective_adjoint_warp_body(const ObjArgs<R, Q>& a, const R* __restrict__ D,
                                                            const R* __restrict__ Dn, R* __restrict__ Lc, int t,
                                                            int T, int bid) {
    using L = Lat<Q>;
    const int lane = threadIdx.x & 31;
    const int k = bid * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (k >= a.n_target) return;  // uniform over the warp
    const int n = a.node[k];
    const bool on = lane < Q;
    const int q = on ? lane : 0;
    const double c0 = on ? L::cx(q) : 0, c1 = on ? L::cy(q) : 0, c2 = on ? L::cz(q) : 0;
    const double* nrm = a.nw_normal + 3 * (long long)a.nw[k];
    const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
    const double m0 = c0 - cn * nrm[0], m1 = c1 - cn * nrm[1], m2 = c2 - cn * nrm[2];
    const double* coef = a.osi ? a.coef + 4 * (long long)k : nullptr;
    double g = 0.0;
    if (t >= 1) {
        const double* mp = a.mom + ((long long)(t - 1) * a.n_target + k) * 4;
        const R up[3] = {(R)mp[1], (R)mp[2], (R)mp[3]};
        const double fne = on ? (double)(D[(long long)q * a.ld + n] - deq<R, Q>(q, (R)mp[0], up)) : 0.0;
        const double f = fne * cn;
        const double tau[3] = {a.cw * warp_sum(f * m0), a.cw * warp_sum(f * m1), a.cw * warp_sum(f * m2)};
        double dt[3];
        objective_dtau(a.osi, coef, a.inv_T, tau, dt);
        g = a.cw * cn * (dt[0] * m0 + dt[1] * m1 + dt[2] * m2);
    }
    if (t < T) {
        const double* mt = a.mom + ((long long)t * a.n_target + k) * 4;
        const R ut[3] = {(R)mt[1], (R)mt[2], (R)mt[3]};
        const double fne = on ? (double)(Dn[(long long)q * a.ld + n] - deq<R, Q>(q, (R)mt[0], ut)) : 0.0;
        const double f = fne * cn;
        const double tau[3] = {a.cw * warp_sum(f * m0), a.cw * warp_sum(f * m1), a.cw * warp_sum(f * m2)};
        double dt[3];
        objective_dtau(a.osi, coef, a.inv_T, tau, dt);
        const double gq = on ? a.cw * cn * (dt[0] * m0 + dt[1] * m1 + dt[2] * m2) : 0.0;
        // sum_r gq_r d feq_r / d f_q = A + B . c_q at the moments of f^t
        const double u[3] = {mt[1], mt[2], mt[3]};
        const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const double cu = c0 * u[0] + c1 * u[1] + c2 * u[2];
        const double gw = gq * (on ? L::w(q) : 0.0);
        const double A = warp_sum(gw * (1.0 - 4.5 * cu * cu + 1.5 * usq));
        const double kk = 3.0 + 9.0 * cu;
        const double B0 = warp_sum(gw * (kk * c0 - 3.0 * u[0]));
        const double B1 = warp_sum(gw * (kk * c1 - 3.0 * u[1]));
        const double B2 = warp_sum(gw * (kk * c2 - 3.0 * u[2]));
        g -= A + B0 * c0 + B1 * c1 + B2 * c2;
    }
    if (on) Lc[(long long)q * a.ld + n] += (R)g;
}

// Adds the objective's term to lambda^t at the targets.
template <class R, int Q>
__global__ void adj_objective_adjoint_kernel(ObjArgs<R, Q> a, const R* __restrict__ D, const R* __restrict__ Dn,
                                             R* __restrict__ Lc, int t, int T) {
    objective_adjoint_warp_body<R, Q>(a, D, Dn, Lc, t, T, blockIdx.x);
}

// The same two objective kernels with one thread per target, for large
// target sets: a thread keeps the target's Q values in registers and sums
// them in direction order, where the warp forms spend most of their
// instructions on FP64 shuffle reductions (sums here run in another order,
// so results agree to rounding). Used when there are enough targets to fill
// the GPU with threads.
constexpr int OBJ_THREAD_MIN_TARGETS = 8192;

template <class R, int Q>
__device__ __forceinline__ void objective_thread_body(const ObjArgs<R, Q>& a, const R* __restrict__ D, int t,
                                                      int bid) {
    using L = Lat<Q>;
    const int k = bid * blockDim.x + threadIdx.x;
    double jl = 0.0;
    if (k < a.n_target) {
        const int n = a.node[k];
        R d[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q] = D[(long long)q * a.ld + n];
        double drho = 0.0, j0 = 0.0, j1 = 0.0, j2 = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double v = (double)d[q];
            drho += v;
            j0 += L::cx(q) * v;
            j1 += L::cy(q) * v;
            j2 += L::cz(q) * v;
        }
        const double rho = 1.0 + drho;
        double* mt = a.mom + ((long long)t * a.n_target + k) * 4;
        if (t >= 1) {
            const double* mp = mt - 4 * (long long)a.n_target;
            const R up[3] = {(R)mp[1], (R)mp[2], (R)mp[3]};
            const double* nrm = a.nw_normal + 3 * (long long)a.nw[k];
            double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const double c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
                const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
                const double f = (double)(d[q] - deq<R, Q>(q, (R)mp[0], up)) * cn;
                t0 += f * (c0 - cn * nrm[0]);
                t1 += f * (c1 - cn * nrm[1]);
                t2 += f * (c2 - cn * nrm[2]);
            }
            t0 *= a.cw;
            t1 *= a.cw;
            t2 *= a.cw;
            if (a.osi) {
                double* ac = a.acc + 4 * (long long)k;
                ac[0] += t0;
                ac[1] += t1;
                ac[2] += t2;
                ac[3] += sqrt(t0 * t0 + t1 * t1 + t2 * t2);
            } else {
                jl = a.inv_T * (t0 * t0 + t1 * t1 + t2 * t2);
            }
        }
        mt[0] = drho;
        mt[1] = j0 / rho;
        mt[2] = j1 / rho;
        mt[3] = j2 / rho;
    }
    warp_accumulate(jl, a.J);
}

template <class R, int Q>
__global__ void __launch_bounds__(128) adj_objective_thread_kernel(ObjArgs<R, Q> a, const R* __restrict__ D, int t) {
    objective_thread_body<R, Q>(a, D, t, blockIdx.x);
}

// The objective's term of lambda^t at target k, one thread: added to Lc, or
// stored in Gout[k][q] when Gout is given.
template <class R, int Q>
__device__ __forceinline__ void objective_adjoint_thread_body(const ObjArgs<R, Q>& a, const R* __restrict__ D,
                                                              const R* __restrict__ Dn, R* __restrict__ Lc,
                                                              R* __restrict__ Gout, int k, int t, int T) {
    using L = Lat<Q>;
    const int n = a.node[k];
    const double* nrm = a.nw_normal + 3 * (long long)a.nw[k];
    const double* coef = a.osi ? a.coef + 4 * (long long)k : nullptr;
    // traction of populations src with the f_eq of moments m (drho, u)
    auto traction = [&](const R* src, const double* m, double tau[3]) {
        const R um[3] = {(R)m[1], (R)m[2], (R)m[3]};
        tau[0] = tau[1] = tau[2] = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
            const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
            const double f = (double)(src[(long long)q * a.ld + n] - deq<R, Q>(q, (R)m[0], um)) * cn;
            tau[0] += f * (c0 - cn * nrm[0]);
            tau[1] += f * (c1 - cn * nrm[1]);
            tau[2] += f * (c2 - cn * nrm[2]);
        }
        for (int c = 0; c < 3; ++c) tau[c] *= a.cw;
    };
    // g_q = cw cn_q (dtp . m_q) - (A + B . c_q): dtp = dJ_t/dtau^t (t >= 1), and
    // A, B the f_eq adjoint of dJ_{t+1}/dtau^{t+1} at the moments of f^t (t < T)
    double dtp[3] = {0.0, 0.0, 0.0}, A = 0.0, B0 = 0.0, B1 = 0.0, B2 = 0.0;
    if (t >= 1) {
        const double* mp = a.mom + ((long long)(t - 1) * a.n_target + k) * 4;
        double tau[3];
        traction(D, mp, tau);
        objective_dtau(a.osi, coef, a.inv_T, tau, dtp);
    }
    if (t < T) {
        const double* mt = a.mom + ((long long)t * a.n_target + k) * 4;
        double tau[3], dt[3];
        traction(Dn, mt, tau);
        objective_dtau(a.osi, coef, a.inv_T, tau, dt);
        const double u[3] = {mt[1], mt[2], mt[3]};
        const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
            const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
            const double gq =
                a.cw * cn * (dt[0] * (c0 - cn * nrm[0]) + dt[1] * (c1 - cn * nrm[1]) + dt[2] * (c2 - cn * nrm[2]));
            const double cu = c0 * u[0] + c1 * u[1] + c2 * u[2];
            const double gw = gq * L::w(q);
            const double kk = 3.0 + 9.0 * cu;
            A += gw * (1.0 - 4.5 * cu * cu + 1.5 * usq);
            B0 += gw * (kk * c0 - 3.0 * u[0]);
            B1 += gw * (kk * c1 - 3.0 * u[1]);
            B2 += gw * (kk * c2 - 3.0 * u[2]);
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const double c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
        const double cn = c0 * nrm[0] + c1 * nrm[1] + c2 * nrm[2];
        const double g = a.cw * cn * (dtp[0] * (c0 - cn * nrm[0]) + dtp[1] * (c1 - cn * nrm[1]) +
                                      dtp[2] * (c2 - cn * nrm[2])) -
                         (A + B0 * c0 + B1 * c1 + B2 * c2);
        if (Gout) Gout[(long long)k * Q + q] = (R)g;
        else Lc[(long long)q * a.ld + n] += (R)g;
    }
}

template <class R, int Q>
__global__ void __launch_bounds__(128)
    adj_objective_adjoint_thread_kernel(ObjArgs<R, Q> a, const R* __restrict__ D, const R* __restrict__ Dn,
                                        R* __restrict__ Lc, int t, int T) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < a.n_target) objective_adjoint_thread_body<R, Q>(a, D, Dn, Lc, nullptr, k, t, T);
}

// The objective's terms of a whole checkpoint segment, steps t0 .. t0 +
// n_steps - 1 (all below T), one thread per (step, target): a term needs
// f^t, f^{t+1} and the forward sweep's moments, not lambda, so the segment's
// terms are computed as soon as its states are, in one launch wide enough to
// fill the GPU. State j of the segment is `first` for j = 0, else states[j];
// the term of step t0 + j goes to Gout[j][k][q], which the pull of that step
// adds at the targets.
template <class R, int Q>
__global__ void __launch_bounds__(128)
    adj_objective_adjoint_segment_kernel(ObjArgs<R, Q> a, const R* const* __restrict__ states,
                                         const R* __restrict__ first, int t0, int n_steps, int T,
                                         R* __restrict__ Gout) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)n_steps * a.n_target) return;
    const int j = (int)(i / a.n_target);
    const int k = (int)(i - (long long)j * a.n_target);
    const R* D = j == 0 ? first : states[j];
    objective_adjoint_thread_body<R, Q>(a, D, states[j + 1], nullptr, Gout + (long long)j * a.n_target * Q, k,
                                        t0 + j, T);
}

// ------------------------------------------------ FP32 kernels, node pairs ---
// FP32 forms of the push and pull kernels over two adjacent nodes per thread
// (the engine's pair layout, n even): 2-wide coalesced access to the nodes'
// own slots, packed FP32 arithmetic (the engine's collide_pair for the
// forward collision), and one address per direction for both nodes of a
// "twin" pair (same segment row and neighbour mask, neither node on an open
// boundary). Other pairs take each node through the scalar rules. Slot
// indices are 32-bit (the launcher requires Q * ld < 2^32).

template <int Q>
__device__ __forceinline__ bool adj_open(typename Meta<Q>::T m) {
    const int k = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);
    return k == KIND_INLET || k == KIND_OUTLET;
}

template <int Q>
__device__ __forceinline__ bool adj_twin(typename Meta<Q>::T m0, typename Meta<Q>::T m1) {
    return ((m0 ^ m1) & Meta<Q>::mask_all()) == 0 && (m0 >> Meta<Q>::SEG_SHIFT) == (m1 >> Meta<Q>::SEG_SHIFT) &&
           !adj_open<Q>(m0) && !adj_open<Q>(m1);
}

// c_q . v for two nodes, from adds and subtractions
template <int Q>
__device__ __forceinline__ float2 cdot2(int q, const float2 v[3]) {
    using L = Lat<Q>;
    float2 r = f2s(0.f);
    bool first = true;
    const int c[3] = {L::cx(q), L::cy(q), L::cz(q)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!c[k]) continue;
        if (first) {
            r = c[k] > 0 ? v[k] : f2mul(f2s(-1.f), v[k]);
            first = false;
        } else {
            r = c[k] > 0 ? f2add(r, v[k]) : f2sub(r, v[k]);
        }
    }
    return r;
}

// One node's push scatter with the open-boundary corrections (scalar rules).
template <int Q>
__device__ __forceinline__ void push_scatter_node(const AGeom<float, Q>& g, float* __restrict__ Dn, int n,
                                                  typename Meta<Q>::T m, const int* sd, const float c[Q],
                                                  const float u[3], double s_t) {
    using L = Lat<Q>;
    const unsigned ld = (unsigned)g.ld, un = (unsigned)n;
    const int kind = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);
    if (kind != KIND_INLET && kind != KIND_OUTLET) {
        // no open link: each value to its neighbour's slot or bounced back
        // into the node's own opposite slot, no branch between the stores
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const unsigned i = q == L::REST ? q * ld + un
                                            : (((m >> q) & 1) ? q * ld + (unsigned)(n + sd[q]) : L::opp(q) * ld + un);
            Dn[i] = c[q];
        }
        return;
    }
    float nrm[3] = {0.f, 0.f, 0.f};
    float vin = 0.f;
    if (kind == KIND_INLET) {
        for (int k = 0; k < 3; ++k) nrm[k] = (float)g.in_normal[k];
        vin = (float)(g.speed[g.aux[n]] * s_t);
    } else if (kind == KIND_OUTLET) {
        for (int k = 0; k < 3; ++k) nrm[k] = g.out_nrm[3 * (long long)g.aux[n] + k];
    }
    const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST) {
            Dn[q * ld + un] = c[q];
        } else if ((m >> q) & 1) {
            Dn[q * ld + (unsigned)(n + sd[q])] = c[q];
        } else {
            float v = c[q];
            const float cn = L::cx(q) * nrm[0] + L::cy(q) * nrm[1] + L::cz(q) * nrm[2];
            if (cn > 0.f) {
                if (kind == KIND_INLET) {
                    v = c[q] + (float)(6.0 * L::w(q)) * cn * vin;
                } else {
                    const float cu = L::cx(q) * u[0] + L::cy(q) * u[1] + L::cz(q) * u[2];
                    const float eq = 1.f + 4.5f * cu * cu - 1.5f * usq;
                    v = -c[q] + (float)(2.0 * L::w(q)) * ((float)g.out_rho * eq - 1.f);
                }
            }
            Dn[L::opp(q) * ld + un] = v;
        }
    }
}

template <int Q>
__device__ __forceinline__ void push_pair_body(const AGeom<float, Q>& g, const float* __restrict__ D,
                                               float* __restrict__ Dn, double s_t, int bid) {
    using L = Lat<Q>;
    using MT = typename Meta<Q>::T;
    const int n0 = bid * BLOCK_NODES + 2 * threadIdx.x;
    const bool live0 = n0 < g.n, live1 = n0 + 1 < g.n;
    const MT m0 = live0 ? g.meta[n0] : MT(0);
    const MT m1 = live1 ? g.meta[n0 + 1] : MT(0);
    // node words never change; the state comes from the previous launch
    wait_prior_grid();
    // a warp whose every pair is a twin takes the twin path; mixed warps take
    // the general one, which serves twins too, instead of running both
    const bool twin = __all_sync(0xffffffffu, !live0 || adj_twin<Q>(m0, m1));
    if (!live0) return;
    const unsigned ld = (unsigned)g.ld, u0 = (unsigned)n0;
    float2 s[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) s[q] = *reinterpret_cast<const float2*>(D + (q * ld + u0));
    float2 drho, u[3];
    collide_pair<Q>(s, g.omega, drho, u);
    const int* sd0 = nbr_row<Q>(g.seg_base, g.seg_delta, n0, m0);
    if (twin) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (q == L::REST) {
                *reinterpret_cast<float2*>(Dn + (q * ld + u0)) = s[q];
                continue;
            }
            const unsigned i = ((m0 >> q) & 1) ? q * ld + (unsigned)(n0 + sd0[q]) : L::opp(q) * ld + u0;
            Dn[i] = s[q].x;
            Dn[i + 1] = s[q].y;
        }
    } else {
        float c[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) c[q] = s[q].x;
        const float ux[3] = {u[0].x, u[1].x, u[2].x};
        push_scatter_node<Q>(g, Dn, n0, m0, sd0, c, ux, s_t);
        if (live1) {
#pragma unroll
            for (int q = 0; q < Q; ++q) c[q] = s[q].y;
            const float uy[3] = {u[0].y, u[1].y, u[2].y};
            push_scatter_node<Q>(g, Dn, n0 + 1, m1, nbr_row<Q>(g.seg_base, g.seg_delta, n0 + 1, m1), c, uy, s_t);
        }
    }
}

template <int Q>
__global__ void __launch_bounds__(PAIR_THREADS, LBM_ADJ_PUSH_MIN_BLOCKS)
    adj_push_pair_kernel(AGeom<float, Q> g, const float* __restrict__ D, float* __restrict__ Dn, double s_t,
                         int rev) {
    allow_next_grid();
    push_pair_body<Q>(g, D, Dn, s_t, rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x);
}

// The forward sweep's objective term and push of one step in one launch: the
// first obj_blocks blocks evaluate the objective at the targets, the others
// push. Both read f^t; the objective writes only its per-target moments and
// sums and the push only f^{t+1}, so the two run side by side instead of the
// short objective launch idling the GPU before each push.
template <int Q, bool THREADS>
__global__ void __launch_bounds__(PAIR_THREADS, LBM_ADJ_PUSH_MIN_BLOCKS)
    adj_push_objective_kernel(AGeom<float, Q> g, const float* __restrict__ D, float* __restrict__ Dn, double s_t,
                              ObjArgs<float, Q> a, int t, int obj_blocks, int rev) {
    allow_next_grid();
    if ((int)blockIdx.x < obj_blocks) {
        wait_prior_grid();
        if (THREADS) objective_thread_body<float, Q>(a, D, t, blockIdx.x);
        else objective_warp_body<float, Q>(a, D, t, blockIdx.x);
    } else {
        const int b = (int)blockIdx.x - obj_blocks, nb = (int)gridDim.x - obj_blocks;
        push_pair_body<Q>(g, D, Dn, s_t, rev ? nb - 1 - b : b);
    }
}

// The boundary rules of one node's pulled values (scalar rules): mu holds
// the raw values (lambda^{t+1} of the neighbour along each link, or of the
// node's own opposite slot where the link is missing) and becomes mu_q; gin
// gathers the inlet-speed sensitivity factor and out_links the outlet links.
template <int Q>
__device__ __forceinline__ void pull_fix_node(const AGeom<float, Q>& g, int n, typename Meta<Q>::T m, float mu[Q],
                                              float& gin, unsigned& out_links) {
    using L = Lat<Q>;
    const int kind = (int)((m >> Meta<Q>::KIND_SHIFT) & 3);
    if (kind != KIND_INLET && kind != KIND_OUTLET) return;
    float nrm[3] = {0.f, 0.f, 0.f};
    if (kind == KIND_INLET) {
        for (int k = 0; k < 3; ++k) nrm[k] = (float)g.in_normal[k];
    } else {
        for (int k = 0; k < 3; ++k) nrm[k] = g.out_nrm[3 * (long long)g.aux[n] + k];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST || ((m >> q) & 1)) continue;
        const float cn = L::cx(q) * nrm[0] + L::cy(q) * nrm[1] + L::cz(q) * nrm[2];
        if (cn > 0.f) {
            if (kind == KIND_INLET) {
                gin += mu[q] * (float)(6.0 * L::w(q)) * cn;
            } else {
                mu[q] = -mu[q];
                out_links |= 1u << q;
            }
        }
    }
}

// Slot of lambda^{t+1} that node n pulls in direction q: the neighbour's
// along the link, or the node's own opposite slot where the link is missing.
template <int Q>
__device__ __forceinline__ unsigned pull_slot(unsigned ld, int n, typename Meta<Q>::T m, const int* sd, int q) {
    using L = Lat<Q>;
    if (q == L::REST) return q * ld + (unsigned)n;
    return ((m >> q) & 1) ? q * ld + (unsigned)(n + sd[q]) : L::opp(q) * ld + (unsigned)n;
}

// One node's pull gather: mu_q, the inlet-speed factor and the outlet links.
template <int Q>
__device__ __forceinline__ void pull_gather_node(const AGeom<float, Q>& g, const float* __restrict__ Ln, int n,
                                                 typename Meta<Q>::T m, const int* sd, float mu[Q], float& gin,
                                                 unsigned& out_links) {
#pragma unroll
    for (int q = 0; q < Q; ++q) mu[q] = Ln[pull_slot<Q>((unsigned)g.ld, n, m, sd, q)];
    pull_fix_node<Q>(g, n, m, mu, gin, out_links);
}

// A second read of two adjacent floats the thread has just read (an L1 hit).
__device__ __forceinline__ float2 reload2(const float* p) {
    float2 v;
    asm volatile("ld.global.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}

// The reverse step of a pair once its pulled values mu (boundary rules
// applied) and the moment sums of f^t (ra + rb = drho, j) and sum mu d are
// known: lambda^t = (1 - omega) mu + omega (A + B.c) + G terms, stored, plus
// the objective's term at targets and the inlet-speed sensitivity. Returns
// the pair's share of dJ/domega.
template <int Q>
__device__ __forceinline__ double pull_pair_math(const AGeom<float, Q>& g, float* __restrict__ Lc, double s_t,
                                                 double* __restrict__ dspeed, const float* __restrict__ Gadd,
                                                 int n0, bool live1, typename Meta<Q>::T m0,
                                                 typename Meta<Q>::T m1, const float2 mu[Q], float2 ra, float2 rb,
                                                 float2 j0, float2 j1, float2 j2, float2 mud, float gin0,
                                                 float gin1, unsigned ol0, unsigned ol1) {
    using L = Lat<Q>;
    const unsigned ld = (unsigned)g.ld, u0 = (unsigned)n0;
    const float2 drho = f2add(ra, rb);
    const float2 rho = f2add(f2s(1.f), drho);
    const float2 irho = make_float2(1.f / rho.x, 1.f / rho.y);
    const float2 u[3] = {f2mul(j0, irho), f2mul(j1, irho), f2mul(j2, irho)};
    const float2 usq = f2fma(u[0], u[0], f2fma(u[1], u[1], f2mul(u[2], u[2])));
    // outlet links: d/du of 2 w rho_out eq(u), times lambda = -mu (scalar, rare)
    float2 G[3] = {f2s(0.f), f2s(0.f), f2s(0.f)};
    if (ol0 | ol1) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float c0 = (float)L::cx(q), c1 = (float)L::cy(q), c2 = (float)L::cz(q);
            const float k2 = (float)(2.0 * L::w(q) * g.out_rho);
            if ((ol0 >> q) & 1) {
                const float cu = c0 * u[0].x + c1 * u[1].x + c2 * u[2].x;
                const float k = -mu[q].x * k2;
                G[0].x += k * (9.f * cu * c0 - 3.f * u[0].x);
                G[1].x += k * (9.f * cu * c1 - 3.f * u[1].x);
                G[2].x += k * (9.f * cu * c2 - 3.f * u[2].x);
            }
            if ((ol1 >> q) & 1) {
                const float cu = c0 * u[0].y + c1 * u[1].y + c2 * u[2].y;
                const float k = -mu[q].y * k2;
                G[0].y += k * (9.f * cu * c0 - 3.f * u[0].y);
                G[1].y += k * (9.f * cu * c1 - 3.f * u[1].y);
                G[2].y += k * (9.f * cu * c2 - 3.f * u[2].y);
            }
        }
    }
    // A = sum mu w (1 - 4.5 cu^2 + 1.5 u^2), B = sum mu w (3 + 9 cu) c - 3 u sum mu w,
    // sum mu deq, over direction pairs (q, opp q): cu flips sign
    const float2 base = f2fma(rho, f2mul(f2s(-1.5f), usq), drho);
    const float2 rho3 = f2mul(f2s(3.f), rho);
    const float2 a0 = f2fma(f2s(1.5f), usq, f2s(1.f));
    float2 A = f2s(0.f), Wm = f2s(0.f), mueq = f2s(0.f);
    float2 Bc[3] = {f2s(0.f), f2s(0.f), f2s(0.f)};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int o = L::opp(q);
        const float2 w = f2s((float)L::w(q));
        if (q == L::REST) {
            const float2 wm = f2mul(w, mu[q]);
            A = f2fma(wm, a0, A);
            Wm = f2add(Wm, wm);
            mueq = f2fma(wm, base, mueq);
            continue;
        }
        if (o < q) continue;
        const float2 cu = cdot2<Q>(q, u);
        const float2 mp = f2mul(w, f2add(mu[q], mu[o]));
        const float2 mm = f2mul(w, f2sub(mu[q], mu[o]));
        const float2 cu2 = f2mul(cu, cu);
        A = f2fma(mp, f2fma(f2s(-4.5f), cu2, a0), A);
        Wm = f2add(Wm, mp);
        const float2 sym = f2fma(rho, f2mul(f2s(4.5f), cu2), base);
        const float2 anti = f2mul(rho3, cu);
        mueq = f2fma(sym, mp, f2fma(anti, mm, mueq));
        // (3 mm + 9 cu mp) c
        const float2 bk = f2fma(f2s(9.f), f2mul(cu, mp), f2mul(f2s(3.f), mm));
        if (L::cx(q)) Bc[0] = L::cx(q) > 0 ? f2add(Bc[0], bk) : f2sub(Bc[0], bk);
        if (L::cy(q)) Bc[1] = L::cy(q) > 0 ? f2add(Bc[1], bk) : f2sub(Bc[1], bk);
        if (L::cz(q)) Bc[2] = L::cz(q) > 0 ? f2add(Bc[2], bk) : f2sub(Bc[2], bk);
    }
    const float2 B[3] = {f2fma(f2s(-3.f), f2mul(u[0], Wm), Bc[0]), f2fma(f2s(-3.f), f2mul(u[1], Wm), Bc[1]),
                         f2fma(f2s(-3.f), f2mul(u[2], Wm), Bc[2])};
    const float2 gu = f2fma(G[0], u[0], f2fma(G[1], u[1], f2mul(G[2], u[2])));
    const float2 keep = f2s(1.f - g.omega), om = f2s(g.omega);
    // lambda_q = (1 - omega) mu_q + omega (A + B.c_q) + (G.c_q - G.u) / rho
    const float2 Ao = f2mul(om, A);
    const float2 ngu = f2mul(f2s(-1.f), f2mul(gu, irho));
    // targets among the two nodes (near-wall nodes are plain fluid nodes,
    // aux = their near-wall entry)
    int tk0 = -1, tk1 = -1;
    if (Gadd) {
        if ((m0 >> Meta<Q>::NW_SHIFT) & 1) tk0 = g.nw_target[g.aux[n0]];
        if (live1 && ((m1 >> Meta<Q>::NW_SHIFT) & 1)) tk1 = g.nw_target[g.aux[n0 + 1]];
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float2 bc = cdot2<Q>(q, B);
        const float2 gc = cdot2<Q>(q, G);
        float2 lam = f2fma(keep, mu[q], f2fma(om, bc, Ao));
        lam = f2add(lam, f2fma(gc, irho, ngu));
        if (tk0 >= 0) lam.x += Gadd[(long long)tk0 * Q + q];
        if (tk1 >= 0) lam.y += Gadd[(long long)tk1 * Q + q];
        *reinterpret_cast<float2*>(Lc + (q * ld + u0)) = lam;
    }
    const float2 wq = f2sub(mueq, mud);
    const double wl = (double)wq.x + (live1 ? (double)wq.y : 0.0);
    if ((int)((m0 >> Meta<Q>::KIND_SHIFT) & 3) == KIND_INLET) dspeed[g.aux[n0]] += (double)gin0 * s_t;
    if (live1 && (int)((m1 >> Meta<Q>::KIND_SHIFT) & 3) == KIND_INLET)
        dspeed[g.aux[n0 + 1]] += (double)gin1 * s_t;
    return wl;
}

// Gadd (optional): the objective's term of this step per target, [target][Q],
// added to lambda^t at the target nodes before it is stored.
template <int Q>
__device__ __forceinline__ void pull_pair_body(const AGeom<float, Q>& g, const float* __restrict__ D,
                                               const float* __restrict__ Ln, float* __restrict__ Lc, double s_t,
                                               double* __restrict__ dspeed, double* __restrict__ domega,
                                               const float* __restrict__ Gadd, int bid) {
    using L = Lat<Q>;
    using MT = typename Meta<Q>::T;
    extern __shared__ int pull_rows[];
    const int n0 = bid * BLOCK_NODES + 2 * threadIdx.x;
    const unsigned ld = (unsigned)g.ld, u0 = (unsigned)n0;
    const bool live0 = n0 < g.n;
    // the node's own f^t and word do not depend on the neighbour rows: the
    // moments of f^t are taken first, so that their loads overlap the staging
    // of the block's segment rows in shared memory (one barrier, as the
    // engine's kernels do), and f^t is not held in registers through the
    // gather of lambda^{t+1}
    const MT m0 = live0 ? g.meta[n0] : MT(0);
    const MT m1 = n0 + 1 < g.n ? g.meta[n0 + 1] : MT(0);
    // node words never change; f^t and lambda^{t+1} come from earlier launches
    wait_prior_grid();
    float2 ra = f2s(0.f), rb = f2s(0.f), j0 = f2s(0.f), j1 = f2s(0.f), j2 = f2s(0.f);
    if (live0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float2 dq = *reinterpret_cast<const float2*>(D + (q * ld + u0));
            if (q & 1) rb = f2add(rb, dq);
            else ra = f2add(ra, dq);
            if (L::cx(q)) j0 = L::cx(q) > 0 ? f2add(j0, dq) : f2sub(j0, dq);
            if (L::cy(q)) j1 = L::cy(q) > 0 ? f2add(j1, dq) : f2sub(j1, dq);
            if (L::cz(q)) j2 = L::cz(q) > 0 ? f2add(j2, dq) : f2sub(j2, dq);
        }
    }
    {
        const int s0 = __ldg(g.seg_base + bid);
        const int cnt = (__ldg(g.seg_base + bid + 1) - s0) * Q;
        const int* src = g.seg_delta + (long long)s0 * Q;
        for (int i = threadIdx.x; i < cnt; i += PAIR_THREADS) pull_rows[i] = __ldg(src + i);
        __syncthreads();
    }
    double wl = 0.0;
    const bool live1 = n0 + 1 < g.n;
    // warp-uniform twin path, as in the push
    const bool twin = __all_sync(0xffffffffu, !live0 || adj_twin<Q>(m0, m1));
    if (live0) {
        const int* sd0 = pull_rows + Q * (int)(m0 >> Meta<Q>::SEG_SHIFT);
        float2 mu[Q];
        float gin0 = 0.f, gin1 = 0.f;
        unsigned ol0 = 0, ol1 = 0;
        if (twin) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                if (q == L::REST) {
                    mu[q] = *reinterpret_cast<const float2*>(Ln + (q * ld + u0));
                } else {
                    const unsigned i = ((m0 >> q) & 1) ? q * ld + (unsigned)(n0 + sd0[q]) : L::opp(q) * ld + u0;
                    mu[q] = make_float2(Ln[i], Ln[i + 1]);
                }
            }
        } else {
            float t[Q];
            pull_gather_node<Q>(g, Ln, n0, m0, sd0, t, gin0, ol0);
#pragma unroll
            for (int q = 0; q < Q; ++q) mu[q].x = t[q];
            if (live1) {
                pull_gather_node<Q>(g, Ln, n0 + 1, m1, pull_rows + Q * (int)(m1 >> Meta<Q>::SEG_SHIFT), t, gin1,
                                    ol1);
#pragma unroll
                for (int q = 0; q < Q; ++q) mu[q].y = t[q];
            } else {
#pragma unroll
                for (int q = 0; q < Q; ++q) mu[q].y = 0.f;
            }
        }
        // sum mu d: f^t read again, from L1 (the load is volatile so that the
        // first read's values are not kept in registers instead)
        float2 mud = f2s(0.f);
#pragma unroll
        for (int q = 0; q < Q; ++q) mud = f2fma(mu[q], reload2(D + (q * ld + u0)), mud);
        wl = pull_pair_math<Q>(g, Lc, s_t, dspeed, Gadd, n0, live1, m0, m1, mu, ra, rb, j0, j1, j2, mud, gin0, gin1,
                               ol0, ol1);
    }
    warp_accumulate(wl, domega);
}

template <int Q>
__global__ void __launch_bounds__(PAIR_THREADS, LBM_ADJ_PULL_MIN_BLOCKS)
    adj_pull_pair_kernel(AGeom<float, Q> g, const float* __restrict__ D, const float* __restrict__ Ln,
                         float* __restrict__ Lc, double s_t, double* __restrict__ dspeed,
                         double* __restrict__ domega, const float* __restrict__ Gadd, int rev) {
    allow_next_grid();
    pull_pair_body<Q>(g, D, Ln, Lc, s_t, dspeed, domega, Gadd,
                      rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x);
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

// The reverse sweep's recomputation stream and the events that order it
// against the main stream.
struct AuxStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t forward_done = nullptr, reversed = nullptr, recomputed[2] = {nullptr, nullptr};
    cudaError_t err = cudaSuccess;
    cudaError_t init() {
        err = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        cudaEvent_t* evs[4] = {&forward_done, &reversed, &recomputed[0], &recomputed[1]};
        for (cudaEvent_t* e : evs)
            if (err == cudaSuccess) err = cudaEventCreateWithFlags(e, cudaEventDisableTiming);
        return err;
    }
    ~AuxStream() {
        if (stream) cudaStreamSynchronize(stream);
        cudaEvent_t evs[4] = {forward_done, reversed, recomputed[0], recomputed[1]};
        for (cudaEvent_t e : evs)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
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
    // a second set for the reverse sweep: the states of segment sg - 1 are
    // recomputed into one set while segment sg's reverse steps read the other
    std::vector<R*> seg2((size_t)(s.gradient && nseg > 1 ? K + 1 : 0), nullptr);
    for (size_t j = 1; j < seg2.size(); ++j) seg2[j] = ar.get<R>(field);
    std::vector<R*> ck((size_t)(s.gradient ? nseg : 0));
    for (auto& p : ck) p = ar.get<R>(field);
    R* lam[2] = {nullptr, nullptr};
    if (s.gradient) {
        lam[0] = ar.get<R>(field);
        lam[1] = ar.get<R>(field);
    }
    double* mom = ar.get<double>((size_t)(T + 1) * std::max(nt, 1) * 4);
    double* osi_acc = ar.get<double>((size_t)std::max(nt, 1) * 4);
    double* osi_coef = ar.get<double>((size_t)std::max(nt, 1) * 4);
    double* speed = ar.get<double>(std::max(s.n_in, 1));
    double* dspeed = ar.get<double>(std::max(s.n_in, 1));
    double* scal = ar.get<double>(2 * N_PARTIALS);  // J, then dJ/domega partial sums
    int* tnode = ar.get<int>(std::max(nt, 1));
    int* tnw = ar.get<int>(std::max(nt, 1));
    // FP32 pair kernels: the pull adds the objective's term of its step at
    // the targets (distinct, checked by adjoint_run), a checkpoint segment's
    // terms computed in one launch once its states are ready ("segment"
    // staging). The FP64 kernels keep a kernel per step that adds the term to
    // lambda ("step" staging); LBM_B200_OBJECTIVE_STAGING=step forces it for
    // FP32 too (tests compare the two).
    const bool pairs = std::is_same<R, float>::value && (long long)Q * s.ld < (1LL << 32);
    bool seg_terms = pairs && s.gradient && nt > 0;
    if (const char* f = getenv("LBM_B200_OBJECTIVE_STAGING"); f && !strcmp(f, "step")) seg_terms = false;
    // objective term per target of every step of a segment, one buffer per
    // segment set: [step in segment][target][Q]
    const size_t gsize = seg_terms ? (size_t)nt * Q * (size_t)K : 1;
    R* gterm[2] = {ar.get<R>(gsize), ar.get<R>(gsize)};
    // device copies of the two segment sets' state pointers (entry 0, the
    // checkpoint, is passed on its own)
    R** states_dev[2] = {ar.get<R*>((size_t)K + 1), ar.get<R*>((size_t)K + 1)};
    // target index of each near-wall entry
    int* nw_target = ar.get<int>(std::max(s.n_nw, 1));
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
        std::vector<int> ntg((size_t)std::max(s.n_nw, 1), -1);
        for (int k = 0; k < nt; ++k) ntg[s.targets[k]] = k;
        std::vector<R*> tab[2] = {seg, seg2.empty() ? seg : seg2};
        for (auto& v : tab) v.resize((size_t)K + 1, nullptr);
        for (int j = 0; j < 2; ++j)
            cudaMemcpyAsync(states_dev[j], tab[j].data(), sizeof(R*) * ((size_t)K + 1), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(nw_target, ntg.data(), sizeof(int) * ntg.size(), cudaMemcpyHostToDevice, st);
        if (s.n_in) cudaMemcpyAsync(speed, s.speed.data(), sizeof(double) * s.n_in, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(dspeed, 0, sizeof(double) * std::max(s.n_in, 1), st);
        cudaMemsetAsync(scal, 0, 2 * N_PARTIALS * sizeof(double), st);
        cudaMemsetAsync(osi_acc, 0, sizeof(double) * 4 * std::max(nt, 1), st);
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
    g.nw_target = nw_target;
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
    oa.osi = s.objective == 1;
    oa.acc = osi_acc;
    oa.coef = osi_coef;

    const dim3 grid((unsigned)((s.n + AT - 1) / AT));
    const unsigned tgrid = (unsigned)((nt + 3) / 4);  // one warp per target, 4 per block
    // one thread per target once there are enough targets to fill the GPU;
    // LBM_B200_OBJECTIVE_FORM=thread|warp picks a form (tests compare them)
    bool obj_threads = nt >= OBJ_THREAD_MIN_TARGETS;
    if (const char* form = getenv("LBM_B200_OBJECTIVE_FORM")) {
        if (!strcmp(form, "thread")) obj_threads = true;
        else if (!strcmp(form, "warp")) obj_threads = false;
    }
    const unsigned tgrid_t = (unsigned)((nt + 127) / 128);
    const dim3 pgrid((unsigned)((s.n + BLOCK_NODES - 1) / BLOCK_NODES));
    // the pull kernel stages its block's segment rows in shared memory
    const int pull_smem = s.max_block_segs * Q * (int)sizeof(int);
    if (pairs && pull_smem > 48 * 1024) {
        const cudaError_t ca = cudaFuncSetAttribute(adj_pull_pair_kernel<Q>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, pull_smem);
        if (ca != cudaSuccess) {
            o.err = std::string("adjoint pull kernel shared memory: ") + cudaGetErrorString(ca);
            return -2;
        }
    }
    auto push_on = [&](cudaStream_t stream, const R* D, R* Dn, int64_t t) {
        if constexpr (std::is_same<R, float>::value) {
            if (pairs) {
                const cudaError_t e = launch_pdl(adj_push_pair_kernel<Q>, pgrid, dim3(PAIR_THREADS), 0, stream, g, D,
                                                 Dn, s.factors[t], (int)(t & 1));
                (void)e;  // launch errors surface through cudaGetLastError after the sweep
                return;
            }
        }
        adj_push_kernel<R, Q><<<grid, AT, 0, stream>>>(g, D, Dn, s.factors[t]);
    };
    auto push = [&](const R* D, R* Dn, int64_t t) { push_on(st, D, Dn, t); };
    auto pull = [&](const R* D, const R* Ln, R* Lc, int64_t t, const R* Gadd) {
        if constexpr (std::is_same<R, float>::value) {
            if (pairs) {
                const cudaError_t e = launch_pdl(adj_pull_pair_kernel<Q>, pgrid, dim3(PAIR_THREADS), (size_t)pull_smem, st,
                                                 g, D, Ln, Lc, s.factors[t], dspeed, scal + N_PARTIALS, Gadd,
                                                 (int)(t & 1));
                (void)e;  // launch errors surface through cudaGetLastError after the sweep
                return;
            }
        }
        adj_pull_kernel<R, Q><<<grid, AT, 0, st>>>(g, D, Ln, Lc, s.factors[t], dspeed, scal + N_PARTIALS);
    };
    auto objective = [&](const R* D, int64_t t) {
        if (nt && obj_threads) adj_objective_thread_kernel<R, Q><<<tgrid_t, 128, 0, st>>>(oa, D, (int)t);
        else if (nt) adj_objective_kernel<R, Q><<<tgrid, 128, 0, st>>>(oa, D, (int)t);
    };
    // a forward step: objective term at f^t and the push to f^{t+1}, fused in
    // one launch for the FP32 pair kernels
    auto objective_push = [&](const R* D, R* Dn, int64_t t) {
        if constexpr (std::is_same<R, float>::value) {
            if (pairs && nt) {
                const int ob = (int)(obj_threads ? tgrid_t : tgrid);
                const dim3 fgrid(pgrid.x + (unsigned)ob);
                cudaError_t e;
                if (obj_threads)
                    e = launch_pdl(adj_push_objective_kernel<Q, true>, fgrid, dim3(PAIR_THREADS), 0, st, g, D, Dn,
                                   s.factors[t], oa, (int)t, ob, (int)(t & 1));
                else
                    e = launch_pdl(adj_push_objective_kernel<Q, false>, fgrid, dim3(PAIR_THREADS), 0, st, g, D, Dn,
                                   s.factors[t], oa, (int)t, ob, (int)(t & 1));
                (void)e;  // launch errors surface through cudaGetLastError after the sweep
                return;
            }
        }
        objective(D, t);
        push(D, Dn, t);
    };
    Events ev;
    cudaEventRecord(ev.e[0], st);
    const R* fT = nullptr;
    if (!s.gradient) {
        adj_load_kernel<R, Q><<<grid, AT, 0, st>>>(s.f0, s.ld, s.n, seg[0]);
        for (int64_t t = 0; t < T; ++t) {
            objective_push(seg[0], seg[1], t);
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
            if (sg + 1 < nseg) {
                // of this segment only the next checkpoint is kept: the steps
                // alternate between two buffers (a state the size of L2 stays
                // there) and the last one writes the checkpoint itself
                const R* src = ck[sg];
                for (int64_t t = t0; t < t1; ++t) {
                    R* dst = t + 1 == t1 ? ck[sg + 1] : seg[1 + ((t - t0) & 1)];
                    objective_push(src, dst, t);
                    src = dst;
                }
            } else {
                for (int64_t t = t0; t < t1; ++t) objective_push(seg[t - t0], seg[t - t0 + 1], t);
            }
        }
        const int64_t tl = (nseg - 1) * K;
        objective(seg[T - tl], T);
        fT = seg[T - tl];
    }
    if (s.final_pop) adj_store_kernel<R, Q><<<grid, AT, 0, st>>>(fT, s.ld, s.n, s.final_pop);
    // mean OSI: J and its derivative w.r.t. each target's sums A = sum tau,
    // M = sum |tau| (OSI = (1 - |A| / M) / 2), once the forward sweep is done
    double J_osi = 0.0;
    if (oa.osi && nt) {
        std::vector<double> acc(4 * (size_t)nt), coef(4 * (size_t)nt, 0.0);
        cudaMemcpyAsync(acc.data(), osi_acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost, st);
        cudaError_t e1 = cudaStreamSynchronize(st);
        if (e1 != cudaSuccess) {
            o.err = std::string("adjoint OSI sums: ") + cudaGetErrorString(e1);
            return -2;
        }
        for (int k = 0; k < nt; ++k) {
            const double* a4 = &acc[4 * (size_t)k];
            const double A = std::sqrt(a4[0] * a4[0] + a4[1] * a4[1] + a4[2] * a4[2]), M = a4[3];
            if (!(M > 0.0)) continue;
            J_osi += 0.5 * (1.0 - A / M) / nt;
            if (A > 0.0)
                for (int c = 0; c < 3; ++c) coef[4 * (size_t)k + c] = -0.5 * a4[c] / (A * M * nt);
            coef[4 * (size_t)k + 3] = 0.5 * A / (M * M * nt);
        }
        cudaMemcpyAsync(osi_coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice, st);
        // coef must stay alive until the copy has run
        e1 = cudaStreamSynchronize(st);
        if (e1 != cudaSuccess) {
            o.err = std::string("adjoint OSI coefficients: ") + cudaGetErrorString(e1);
            return -2;
        }
    }
    cudaEventRecord(ev.e[1], st);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        o.err = std::string("adjoint forward sweep: ") + cudaGetErrorString(ce);
        cudaStreamSynchronize(st);
        return -2;
    }
    if (s.gradient) {
        // reverse sweep, segment by segment. The last segment's states are
        // still in seg from the forward sweep; the states of segment sg - 1
        // are recomputed on a second stream into the other set while the
        // reverse steps of segment sg run, so the two overlap. The set a
        // recomputation overwrites was last read by segment sg + 1's reverse
        // steps, which it waits for.
        R* Lnext = lam[0];
        R* Lcur = lam[1];
        std::vector<R*>* sets[2] = {&seg, &seg2};
        AuxStream aux;
        if (nseg > 1 && aux.init() != cudaSuccess) {
            o.err = "adjoint recomputation stream: " + std::string(cudaGetErrorString(aux.err));
            cudaStreamSynchronize(st);
            return -2;
        }
        // the objective's terms of segment sg, once its states are in its
        // set, into that set's term buffer
        auto segment_terms = [&](cudaStream_t stream, int64_t sg) {
            if (!seg_terms) return;
            const int64_t t0 = sg * K, n_steps = std::min(T, t0 + K) - t0;
            const int set = (int)((nseg - 1 - sg) & 1);
            const unsigned blocks = (unsigned)((n_steps * nt + 127) / 128);
            adj_objective_adjoint_segment_kernel<R, Q><<<blocks, 128, 0, stream>>>(
                oa, states_dev[set], ck[sg], (int)t0, (int)n_steps, (int)T, gterm[set]);
        };
        auto recompute = [&](int64_t sg) {
            const int64_t t0 = sg * K, t1 = std::min(T, t0 + K);
            std::vector<R*>& S = *sets[(nseg - 1 - sg) & 1];
            S[0] = ck[sg];
            for (int64_t t = t0; t < t1; ++t) push_on(aux.stream, S[t - t0], S[t - t0 + 1], t);
            segment_terms(aux.stream, sg);
            cudaEventRecord(aux.recomputed[sg & 1], aux.stream);
            o.steps_recomputed += t1 - t0;
        };
        segment_terms(st, nseg - 1);
        if (nseg > 1) {
            // the checkpoints come from the forward sweep on st
            cudaEventRecord(aux.forward_done, st);
            cudaStreamWaitEvent(aux.stream, aux.forward_done, 0);
            recompute(nseg - 2);
        }
        for (int64_t sg = nseg - 1; sg >= 0; --sg) {
            const int64_t t0 = sg * K, t1 = std::min(T, t0 + K);
            std::vector<R*>& S = *sets[(nseg - 1 - sg) & 1];
            S[0] = ck[sg];
            if (sg + 1 < nseg) cudaStreamWaitEvent(st, aux.recomputed[sg & 1], 0);
            // lambda^{t1} of an earlier segment was finished by the later one
            const R* gseg = gterm[(nseg - 1 - sg) & 1];
            const int64_t top = t1 == T ? T : t1 - 1;
            for (int64_t t = top; t >= t0; --t) {
                if (t < T && seg_terms) {
                    pull(S[t - t0], Lnext, Lcur, t, gseg + (size_t)(t - t0) * nt * Q);
                } else {
                    if (t == T) cudaMemsetAsync(Lcur, 0, field * sizeof(R), st);
                    else pull(S[t - t0], Lnext, Lcur, t, nullptr);
                    if (nt && obj_threads)
                        adj_objective_adjoint_thread_kernel<R, Q><<<tgrid_t, 128, 0, st>>>(
                            oa, S[t - t0], t < T ? S[t - t0 + 1] : nullptr, Lcur, (int)t, (int)T);
                    else if (nt)
                        adj_objective_adjoint_kernel<R, Q><<<tgrid, 128, 0, st>>>(
                            oa, S[t - t0], t < T ? S[t - t0 + 1] : nullptr, Lcur, (int)t, (int)T);
                }
                std::swap(Lnext, Lcur);
            }
            if (sg >= 2) {
                // segment sg - 2 goes into this segment's set once its reverse steps are done
                cudaEventRecord(aux.reversed, st);
                cudaStreamWaitEvent(aux.stream, aux.reversed, 0);
                recompute(sg - 2);
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
    std::vector<double> hs(2 * N_PARTIALS);
    cudaMemcpy(hs.data(), scal, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost);
    o.J = 0.0;
    o.dJ_domega = 0.0;
    for (int i = 0; i < N_PARTIALS; ++i) {
        o.J += hs[i];
        o.dJ_domega += hs[N_PARTIALS + i];
    }
    if (oa.osi) o.J = J_osi;
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
