// Physics-mode step kernels for shifted storage (FP32 / FP16 / BF16), two
// nodes per thread.
//
// The nodes n and n + 1 of a thread are adjacent in memory (n even; ld is a
// multiple of BLOCK_NODES), so:
//  * phase 0 reads and writes both nodes' slots with one 2-wide access
//    (float2, __half2, __nv_bfloat162): its slots (n, q) and (n, opp q) do not
//    depend on the neighbours, and physics mode stores c_q into (n, opp q)
//    whether or not the neighbour exists;
//  * the collision of the two nodes runs in packed FP32 (fma.rn.f32x2 and
//    friends), one instruction for both nodes. Opposite directions share
//    c.u, so each direction pair costs one symmetric and one antisymmetric
//    term.
// Phase 1 gathers and scatters each node on its own (the neighbours' slots
// are not pairwise aligned), with a select between the neighbour's slot and
// the node's own opposite slot for missing neighbours, as in step_kernel.
// Results equal step_kernel's up to FP32 rounding (the arithmetic is
// rearranged).
#pragma once

#include "kernels.cuh"

namespace lbm {

__device__ __forceinline__ float2 f2s(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __ffma2_rn(b, f2s(-1.f), a); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// 2-wide and scalar access to the stored deviations, in FP32.
template <class S>
struct PairIO;
template <>
struct PairIO<float> {
    __device__ static float2 get2(const float* p) { return *reinterpret_cast<const float2*>(p); }
    __device__ static void put2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
    __device__ static float get(const float* p) { return *p; }
    __device__ static void put(float* p, float v) { *p = v; }
};
template <>
struct PairIO<__half> {
    __device__ static float2 get2(const __half* p) { return __half22float2(*reinterpret_cast<const __half2*>(p)); }
    __device__ static void put2(__half* p, float2 v) { *reinterpret_cast<__half2*>(p) = __float22half2_rn(v); }
    __device__ static float get(const __half* p) { return __half2float(*p); }
    __device__ static void put(__half* p, float v) { *p = __float2half_rn(v); }
};
template <>
struct PairIO<__nv_bfloat16> {
    __device__ static float2 get2(const __nv_bfloat16* p) {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    }
    __device__ static void put2(__nv_bfloat16* p, float2 v) {
        *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v);
    }
    __device__ static float get(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ static void put(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

constexpr int PAIR_THREADS = BLOCK_NODES / 2;

// Resident CTAs per SM the phase-0 kernel is compiled for (caps registers).
// Its loads carry no dependency, so occupancy is what keeps bytes in flight:
// 6 CTAs (80 registers) for FP32, 8 (64 registers) for the 16-bit types,
// whose 2-wide loads move half the bytes per instruction. D3Q27 holds 27
// pairs of values and gets its own caps: 5 CTAs (96 registers, no spills)
// for every storage type (FP32 at 4 was 2 % slower on the bifurcation).
template <class S, int Q>
constexpr int pair0_min_blocks() {
#ifdef LBM_PAIR0_MIN_BLOCKS
    return LBM_PAIR0_MIN_BLOCKS;
#else
    if (Q == 27) {
#ifdef LBM_PAIR0_MIN_BLOCKS_Q27
        return LBM_PAIR0_MIN_BLOCKS_Q27;
#else
        return 5;
#endif
    }
    return sizeof(S) == 4 ? 6 : 8;
#endif
}

// BGK collision of two nodes' deviations d (in place): c = (1 - omega) d +
// omega deq, deq_q = w_q (drho + (1 + drho)(3 c.u + 4.5 (c.u)^2 - 1.5 u^2)).
// Returns drho and u of the input.
//
// omega w_q deq_q = B_w + t (4.5 c.u + 3) with B_w = omega w (drho - 1.5 rho
// u^2) and t = omega w rho c.u; the opposite direction has c.u negated, which
// is B_w + t (4.5 c.u - 3). A direction pair costs c.u, t, two fmas for the
// brackets, two for the equilibria and two for the relaxations.
template <int Q>
__device__ __forceinline__ void collide_pair(float2 d[Q], float omega, float2& drho, float2 u[3]) {
    using L = Lat<Q>;
    float2 ra = f2s(0.f), rb = f2s(0.f);
    float2 j0 = f2s(0.f), j1 = f2s(0.f), j2 = f2s(0.f);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q & 1) rb = f2add(rb, d[q]);
        else ra = f2add(ra, d[q]);
        if (L::cx(q)) j0 = L::cx(q) > 0 ? f2add(j0, d[q]) : f2sub(j0, d[q]);
        if (L::cy(q)) j1 = L::cy(q) > 0 ? f2add(j1, d[q]) : f2sub(j1, d[q]);
        if (L::cz(q)) j2 = L::cz(q) > 0 ? f2add(j2, d[q]) : f2sub(j2, d[q]);
    }
    drho = f2add(ra, rb);
    const float2 rho = f2add(f2s(1.f), drho);
    const float2 inv = make_float2(__frcp_rn(rho.x), __frcp_rn(rho.y));
    u[0] = f2mul(j0, inv);
    u[1] = f2mul(j1, inv);
    u[2] = f2mul(j2, inv);
    const float2 usq = f2fma(u[0], u[0], f2fma(u[1], u[1], f2mul(u[2], u[2])));
    const float2 base = f2fma(rho, f2mul(f2s(-1.5f), usq), drho);  // drho - 1.5 rho u^2
    const float2 keep = f2s(1.f - omega);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int o = L::opp(q);
        const float ow = omega * (float)L::w(q);
        if (q == L::REST) {
            d[q] = f2fma(keep, d[q], f2mul(f2s(ow), base));
            continue;
        }
        if (o < q) continue;  // handled with its opposite
        float2 cu = f2s(0.f);
        bool first = true;
        auto acc = [&](int c, float2 v) {
            if (!c) return;
            if (first) {
                cu = c > 0 ? v : f2mul(f2s(-1.f), v);
                first = false;
            } else {
                cu = c > 0 ? f2add(cu, v) : f2sub(cu, v);
            }
        };
        acc(L::cx(q), u[0]);
        acc(L::cy(q), u[1]);
        acc(L::cz(q), u[2]);
        // per weight class (the compiler keeps one copy of each)
        const float2 Bw = f2mul(f2s(ow), base);
        const float2 t = f2mul(f2mul(f2s(ow), rho), cu);
        const float2 plus = f2fma(t, f2fma(f2s(4.5f), cu, f2s(3.f)), Bw);
        const float2 minus = f2fma(t, f2fma(f2s(4.5f), cu, f2s(-3.f)), Bw);
        d[q] = f2fma(keep, d[q], plus);
        d[o] = f2fma(keep, d[o], minus);
    }
}

// Everything between the gather and the scatter of a pair: observation,
// near-wall hand-off, collision, non-finite flag, outlet velocities.
template <class S, int Q, int OBS>
__device__ __forceinline__ void pair_middle(const StepArgs<S, Q>& a, float2 s[Q], typename Meta<Q>::T m0,
                                            typename Meta<Q>::T m1, int n0, bool live1) {
    using L = Lat<Q>;
    const int n1 = n0 + 1;
    if (OBS & 1) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            a.obs_pop[(long long)q * a.ld + n0] = (double)s[q].x + L::w(q);
            if (live1) a.obs_pop[(long long)q * a.ld + n1] = (double)s[q].y + L::w(q);
        }
    }
    // near-wall nodes hand the wall-shear pass the second moments of their
    // arriving deviations and, after the collision, its moments
    const bool nw0 = (m0 >> Meta<Q>::NW_SHIFT) & 1, nw1 = (m1 >> Meta<Q>::NW_SHIFT) & 1;
    if (nw0 || nw1) {
        float* h0 = a.nw_s + (nw0 ? a.aux[n0] : 0);
        float* h1 = a.nw_s + (nw1 ? a.aux[n1] : 0);
        auto add = [](float2 x, float2 y) { return f2add(x, y); };
        auto sub = [](float2 x, float2 y) { return f2sub(x, y); };
        auto put = [&](int j, float2 p) {
            if (nw0) h0[(long long)j * a.n_nw] = p.x;
            if (nw1) h1[(long long)j * a.n_nw] = p.y;
        };
        put(0, second_moment<Q, 0>(s, f2s(0.f), add, sub));
        put(1, second_moment<Q, 1>(s, f2s(0.f), add, sub));
        put(2, second_moment<Q, 2>(s, f2s(0.f), add, sub));
        put(3, second_moment<Q, 3>(s, f2s(0.f), add, sub));
        put(4, second_moment<Q, 4>(s, f2s(0.f), add, sub));
        put(5, second_moment<Q, 5>(s, f2s(0.f), add, sub));
    }
    float2 drho, u[3];
    collide_pair<Q>(s, (float)a.omega, drho, u);
    if (!isfinite(drho.x) || (live1 && !isfinite(drho.y))) atomicOr(a.flags, FLAG_NONFINITE);
    if (nw0) {
        float* h = a.nw_s + (long long)HANDOFF_MOM_ROW * a.n_nw + a.aux[n0];
        h[0] = drho.x;
        h[a.n_nw] = u[0].x;
        h[2 * (long long)a.n_nw] = u[1].x;
        h[3 * (long long)a.n_nw] = u[2].x;
    }
    if (nw1) {
        float* h = a.nw_s + (long long)HANDOFF_MOM_ROW * a.n_nw + a.aux[n1];
        h[0] = drho.y;
        h[a.n_nw] = u[0].y;
        h[2 * (long long)a.n_nw] = u[1].y;
        h[3 * (long long)a.n_nw] = u[2].y;
    }
    if (OBS & 2) {
        a.obs_mom[n0] = 1.0 + (double)drho.x;
        a.obs_mom[a.ld + n0] = (double)u[0].x;
        a.obs_mom[2 * a.ld + n0] = (double)u[1].x;
        a.obs_mom[3 * a.ld + n0] = (double)u[2].x;
        if (live1) {
            a.obs_mom[n1] = 1.0 + (double)drho.y;
            a.obs_mom[a.ld + n1] = (double)u[0].y;
            a.obs_mom[2 * a.ld + n1] = (double)u[1].y;
            a.obs_mom[3 * a.ld + n1] = (double)u[2].y;
        }
    }
    // the open-boundary pass needs the outlet nodes' collision velocity
    if ((int)((m0 >> Meta<Q>::KIND_SHIFT) & 3) == KIND_OUTLET) {
        double* o = a.io_u + 3 * (long long)a.aux[n0];
        o[0] = (double)u[0].x;
        o[1] = (double)u[1].x;
        o[2] = (double)u[2].x;
    }
    if ((int)((m1 >> Meta<Q>::KIND_SHIFT) & 3) == KIND_OUTLET) {
        double* o = a.io_u + 3 * (long long)a.aux[n1];
        o[0] = (double)u[0].y;
        o[1] = (double)u[1].y;
        o[2] = (double)u[2].y;
    }
}

// Phase-1 gather of a pair: each node from its upstream neighbours' slots,
// or its own opposite slot where the upstream node is missing (a padding
// node has m = 0 and reads its own padding slots).
template <class S, int Q>
__device__ __forceinline__ void pair_gather1(const StepArgs<S, Q>& a, float2 s[Q], typename Meta<Q>::T m0,
                                             typename Meta<Q>::T m1, const int* sd0, const int* sd1, int n0) {
    using L = Lat<Q>;
    using IO = PairIO<S>;
    // element indices fit 32 bits (the launcher requires Q * ld < 2^32)
    const unsigned ld = (unsigned)a.ld, u0 = (unsigned)n0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST) {
            s[q] = IO::get2(a.pop + (q * ld + u0));
        } else {
            const int oq = L::opp(q);
            const unsigned own0 = q * ld + u0;
            const unsigned i0 = ((m0 >> oq) & 1) ? u0 + (unsigned)sd0[oq] : own0;
            const unsigned i1 = ((m1 >> oq) & 1) ? u0 + 1u + (unsigned)sd1[oq] : own0 + 1;
            s[q] = make_float2(IO::get(a.pop + i0), IO::get(a.pop + i1));
        }
    }
}

// Phase-1 scatter: to the downstream neighbours' slots, or bounced back into
// the node's own opposite slot where the neighbour is missing.
template <class S, int Q>
__device__ __forceinline__ void pair_scatter1(const StepArgs<S, Q>& a, const float2 s[Q], typename Meta<Q>::T m0,
                                              typename Meta<Q>::T m1, const int* sd0, const int* sd1, int n0) {
    using L = Lat<Q>;
    using IO = PairIO<S>;
    const unsigned ld = (unsigned)a.ld, u0 = (unsigned)n0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST) {
            IO::put2(a.pop + (q * ld + u0), s[q]);
            continue;
        }
        const int oq = L::opp(q);
        const unsigned own0 = oq * ld + u0;
        const unsigned i0 = ((m0 >> q) & 1) ? u0 + (unsigned)sd0[q] : own0;
        const unsigned i1 = ((m1 >> q) & 1) ? u0 + 1u + (unsigned)sd1[q] : own0 + 1;
        IO::put(a.pop + i0, s[q].x);
        IO::put(a.pop + i1, s[q].y);
    }
}

// The same gather and scatter for a pair whose two nodes share a segment row
// and a neighbour mask: node n + 1's slot is node n's plus one.
template <class S, int Q>
__device__ __forceinline__ void pair_gather1_twin(const StepArgs<S, Q>& a, float2 s[Q], typename Meta<Q>::T m,
                                                  const int* sd, int n0) {
    using L = Lat<Q>;
    using IO = PairIO<S>;
    const unsigned ld = (unsigned)a.ld, u0 = (unsigned)n0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST) {
            s[q] = IO::get2(a.pop + (q * ld + u0));
        } else {
            const int oq = L::opp(q);
            const unsigned i = ((m >> oq) & 1) ? u0 + (unsigned)sd[oq] : q * ld + u0;
            const S* p = a.pop + i;
            // an even slot index is 2-wide aligned: one access for both nodes
            if (i & 1) s[q] = make_float2(IO::get(p), IO::get(p + 1));
            else s[q] = IO::get2(p);
        }
    }
}

template <class S, int Q>
__device__ __forceinline__ void pair_scatter1_twin(const StepArgs<S, Q>& a, const float2 s[Q],
                                                   typename Meta<Q>::T m, const int* sd, int n0) {
    using L = Lat<Q>;
    using IO = PairIO<S>;
    const unsigned ld = (unsigned)a.ld, u0 = (unsigned)n0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (q == L::REST) {
            IO::put2(a.pop + (q * ld + u0), s[q]);
            continue;
        }
        const int oq = L::opp(q);
        const unsigned i = ((m >> q) & 1) ? u0 + (unsigned)sd[q] : oq * ld + u0;
        S* p = a.pop + i;
        if (i & 1) {
            IO::put(p, s[q].x);
            IO::put(p + 1, s[q].y);
        } else {
            IO::put2(p, s[q]);
        }
    }
}

// Phase 0 (local slots only), one pair per thread.
template <class S, int Q, int OBS>
__global__ void __launch_bounds__(PAIR_THREADS, pair0_min_blocks<S, Q>()) pair_phase0_kernel(StepArgs<S, Q> a) {
    using L = Lat<Q>;
    using MT = typename Meta<Q>::T;
    using IO = PairIO<S>;
    allow_next_grid();
    const int n0 = blockIdx.x * BLOCK_NODES + 2 * threadIdx.x;
    if (n0 >= a.n) {
        wait_prior_grid();
        return;
    }
    const bool live1 = n0 + 1 < a.n;
    // node words never change: read before the wait
    const MT m0 = a.meta[n0];
    const MT m1 = live1 ? a.meta[n0 + 1] : MT(0);
    wait_prior_grid();
    float2 s[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) s[q] = IO::get2(a.pop + (q * (unsigned)a.ld + (unsigned)n0));
    pair_middle<S, Q, OBS>(a, s, m0, m1, n0, live1);
    // a dead second node writes only its own padding slot
#pragma unroll
    for (int q = 0; q < Q; ++q) IO::put2(a.pop + (L::opp(q) * (unsigned)a.ld + (unsigned)n0), s[q]);
}

// ----------------------------------------------- phase 1, persistent form ---
// The phase-1 gather depends on two metadata loads (the node's word, then its
// segment's offsets) before the population loads can start. This form hides
// them: each CTA walks tiles of BLOCK_NODES nodes (tile, tile + gridDim.x,
// ...) and, while it gathers, collides and scatters one tile, copies the next
// tile's node words and segment offsets into the other half of a
// double-buffered shared-memory area with cp.async (global -> shared, no
// registers held). One __syncthreads per tile hands the buffers over.
// Tiles are taken in descending order: the phase-0 kernel before it sweeps
// the lattice upwards, so phase 1 starts on the tiles still in L2 from the
// end of that sweep and ends on tile 0, where the next phase 0 starts.

__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Resident CTAs per SM the phase-1 kernel is compiled for (caps its
// registers): 5 (96 registers, no spills for D3Q19) for FP32, 7 (72) for the
// 16-bit types, measured best on the 21.4M-node vessel.
template <class S, int Q>
constexpr int pair1_min_blocks() {
#ifdef LBM_PAIR1_MIN_BLOCKS
    return LBM_PAIR1_MIN_BLOCKS;
#else
    if (Q == 27) {
#ifdef LBM_PAIR1_MIN_BLOCKS_Q27
        return LBM_PAIR1_MIN_BLOCKS_Q27;
#else
        return sizeof(S) == 4 ? 4 : 5;
#endif
    }
    return sizeof(S) == 4 ? 5 : 7;
#endif
}

// Bytes of one metadata buffer: the tile's node words, then its segment rows
// (seg_smem_bytes), rounded up to 16.
template <int Q>
__host__ __device__ __forceinline__ int pair_buffer_bytes(int seg_smem_bytes) {
    const int b = BLOCK_NODES * (int)sizeof(typename Meta<Q>::T) + seg_smem_bytes;
    return (b + 15) & ~15;
}

template <class S, int Q, int OBS>
__global__ void __launch_bounds__(PAIR_THREADS, pair1_min_blocks<S, Q>()) pair_phase1_kernel(StepArgs<S, Q> a, int n_tiles) {
    using MT = typename Meta<Q>::T;
    extern __shared__ __align__(16) unsigned char pair_smem[];
    const int tid = threadIdx.x;
    const int buf_bytes = pair_buffer_bytes<Q>(a.seg_smem_bytes);
    auto meta_buf = [&](int b) { return reinterpret_cast<MT*>(pair_smem + b * buf_bytes); };
    auto rows_buf = [&](int b) {
        return reinterpret_cast<int*>(pair_smem + b * buf_bytes + BLOCK_NODES * (int)sizeof(MT));
    };
    auto prefetch = [&](int tile, int b) {
        // node words: the thread's two nodes (8 or 16 bytes, aligned: n even)
        const MT* src = a.meta + (long long)tile * BLOCK_NODES + 2 * tid;
        if (sizeof(MT) == 4) cp_async_8(meta_buf(b) + 2 * tid, src);
        else cp_async_16(meta_buf(b) + 2 * tid, src);
        const int s0 = __ldg(a.seg_base + tile);
        const int cnt = (__ldg(a.seg_base + tile + 1) - s0) * Q;
        const int* rows = a.seg_slot + (long long)s0 * Q;
        int* dst = rows_buf(b);
        for (int i = tid; i < cnt; i += PAIR_THREADS) cp_async_4(dst + i, rows + i);
        cp_async_commit();
    };

    // a CTA's first tile is its index; the later ones come from a counter
    // (one atomic per tile, taken a tile ahead), so that CTAs that finish
    // early take more tiles instead of every CTA walking the same stride
    __shared__ int sched[2];
    allow_next_grid();
    int tile = blockIdx.x;
    if (tile >= n_tiles) {
        wait_prior_grid();
        return;
    }
    // the k-th tile taken is tile n_tiles - 1 - k of the lattice
    auto lattice_tile = [&](int k) { return n_tiles - 1 - k; };
    int b = 0, sb = 1;
    // node words and segment rows never change: copied before the wait
    prefetch(lattice_tile(tile), 0);
    wait_prior_grid();
    if (tid == 0) sched[0] = gridDim.x + atomicAdd(a.tile_sched, 1);
    cp_async_wait_all();
    __syncthreads();
    int next = sched[0];
    for (;;) {
        const int n0 = lattice_tile(tile) * BLOCK_NODES + 2 * tid;
        const bool live0 = n0 < a.n, live1 = n0 + 1 < a.n;
        const MT m0 = meta_buf(b)[2 * tid];
        const MT m1 = meta_buf(b)[2 * tid + 1];
        const int* sd0 = rows_buf(b) + Q * (int)(m0 >> Meta<Q>::SEG_SHIFT);
        const int* sd1 = rows_buf(b) + Q * (int)(m1 >> Meta<Q>::SEG_SHIFT);
        // warps whose every pair shares one segment row and one neighbour
        // mask address each direction once for both nodes
        const bool twin = ((m0 ^ m1) & Meta<Q>::mask_all()) == 0 &&
                          (m0 >> Meta<Q>::SEG_SHIFT) == (m1 >> Meta<Q>::SEG_SHIFT);
        const bool uniform = !a.force_general && __all_sync(0xffffffffu, twin);
        float2 s[Q];
        if (uniform) pair_gather1_twin<S, Q>(a, s, m0, sd0, n0);
        else pair_gather1<S, Q>(a, s, m0, m1, sd0, sd1, n0);
        if (next < n_tiles) {
            prefetch(lattice_tile(next), b ^ 1);
            if (tid == 0) sched[sb] = gridDim.x + atomicAdd(a.tile_sched, 1);
        }
        if (live0) {
            pair_middle<S, Q, OBS>(a, s, m0, m1, n0, live1);
            if (uniform) pair_scatter1_twin<S, Q>(a, s, m0, sd0, n0);
            else pair_scatter1<S, Q>(a, s, m0, m1, sd0, sd1, n0);
        }
        if (next >= n_tiles) break;
        cp_async_wait_all();
        __syncthreads();
        tile = next;
        next = sched[sb];
        sb ^= 1;
        b ^= 1;
    }
    // the last CTA out leaves the counter at zero for the next launch (the
    // launches of one engine are ordered on its stream); the fence orders
    // this CTA's counter updates before its count of finished CTAs
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(a.tile_sched + 1, 1) == (int)gridDim.x - 1) {
            a.tile_sched[0] = 0;
            a.tile_sched[1] = 0;
        }
    }
}

}  // namespace lbm
