// Host side of the engine behind the C ABI (include/lbm_b200.h): flattens the
// caller's node set into the device layout, owns the device buffers, and
// sequences the kernels of each time step.
//
// Flattening (replaces the node graph SubDomain builds, Subdomain.cpp:364-611):
//   * nodes are sorted x-major, z-fastest — the order of the reference's own
//     Involved_Lat_ — so neighbours along z are adjacent and neighbours in
//     other directions lie in neighbouring z-runs, which keeps every
//     direction's accesses coalesced;
//   * neighbours are found as SubDomain::Connectivity finds them (the node at
//     x + c_q if it exists, Subdomain.cpp:447-471) through a column index of
//     z-runs, and encoded as a per-node existence mask plus per-segment index
//     offsets (lattice.cuh, Meta);
//   * outlet copies are resolved to source nodes by replaying the reference's
//     in-order sweep (Simulation.cpp:650-741): a node whose inward neighbour
//     was already overwritten by the sweep reads that neighbour's source.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "adjoint.h"
#include "engine_view.h"
#include "errors.h"
#include "lbm_b200.h"
#include "pulse.h"
#include "launch.h"
#include "reduce.cuh"

using namespace lbm;

namespace {

std::string g_create_error = "no error";

struct Topo {
    int n = 0;
    long long ld = 0;
    int nblocks = 0;
    int nseg = 0;
    int max_block_segs = 1;
    std::vector<int> perm;   // internal -> caller
    std::vector<int> iperm;  // caller -> internal
    std::vector<uint64_t> meta;
    std::vector<int> seg_base;
    std::vector<int> seg_delta;
    std::vector<int> aux;
    std::vector<int> in_node;   // internal index per caller inlet entry
    std::vector<int> out_node;  // internal index per outlet-table entry
    std::vector<int> out_src;   // source node (internal) or -1
    std::vector<long long> out_off;   // [n_outlets + 1] outlet k's entries of out_node
    std::vector<double> out_normal;   // [n_outlets][3]
    std::vector<float> out_nrm; // [n_out][3]
    std::vector<int> nw_node;
    std::vector<double> nw_normal;
};

struct ColumnIndex {
    int x0 = 0, y0 = 0, nx = 0, ny = 0;
    struct Run {
        int z0, z1, start;
    };
    std::vector<int> col_first;
    std::vector<Run> runs;
    int lookup(int x, int y, int z) const {
        if (x < x0 || y < y0 || x >= x0 + nx || y >= y0 + ny) return -1;
        const long long c = (long long)(x - x0) * ny + (y - y0);
        for (int r = col_first[c]; r < col_first[c + 1]; ++r)
            if (z >= runs[r].z0 && z <= runs[r].z1) return runs[r].start + (z - runs[r].z0);
        return -1;
    }
};

template <int Q>
std::string build_topology(const lbm_desc& d, Topo& t) {
    using L = Lat<Q>;
    using M = Meta<Q>;
    if (d.n_nodes <= 0 || d.n_nodes > (long long)INT_MAX - BLOCK_NODES) return "n_nodes out of range";
    if (!d.coords || !d.kind) return "coords and kind are required";
    const int n = (int)d.n_nodes;
    t.n = n;
    t.nblocks = (n + BLOCK_NODES - 1) / BLOCK_NODES;
    t.ld = (long long)t.nblocks * BLOCK_NODES;

    // order: x-major, z-fastest
    const int32_t* X = d.coords;
    auto less = [X](int a, int b) {
        if (X[3 * a] != X[3 * b]) return X[3 * a] < X[3 * b];
        if (X[3 * a + 1] != X[3 * b + 1]) return X[3 * a + 1] < X[3 * b + 1];
        return X[3 * a + 2] < X[3 * b + 2];
    };
    t.perm.resize(n);
    std::iota(t.perm.begin(), t.perm.end(), 0);
    if (!std::is_sorted(t.perm.begin(), t.perm.end(), less)) std::sort(t.perm.begin(), t.perm.end(), less);
    t.iperm.assign(n, -1);
    for (int i = 0; i < n; ++i) t.iperm[t.perm[i]] = i;
    std::vector<int> cx(n), cy(n), cz(n), kind(n);
    for (int i = 0; i < n; ++i) {
        const int c = t.perm[i];
        cx[i] = X[3 * c];
        cy[i] = X[3 * c + 1];
        cz[i] = X[3 * c + 2];
        kind[i] = d.kind[c];
        if (kind[i] > 3) return "node kind must be 0..3";
        if (i && cx[i] == cx[i - 1] && cy[i] == cy[i - 1] && cz[i] == cz[i - 1]) return "duplicate node coordinates";
    }

    // column index of z-runs
    ColumnIndex ci;
    const int xmin = *std::min_element(cx.begin(), cx.end()), xmax = *std::max_element(cx.begin(), cx.end());
    const int ymin = *std::min_element(cy.begin(), cy.end()), ymax = *std::max_element(cy.begin(), cy.end());
    ci.x0 = xmin;
    ci.y0 = ymin;
    ci.nx = xmax - xmin + 1;
    ci.ny = ymax - ymin + 1;
    if ((long long)ci.nx * ci.ny > (1LL << 30)) return "node set spans too many (x, y) columns";
    ci.col_first.assign((size_t)ci.nx * ci.ny + 1, 0);
    std::vector<int> col_of_run;
    for (int i = 0; i < n; ++i) {
        const bool cont = i && cx[i] == cx[i - 1] && cy[i] == cy[i - 1] && cz[i] == cz[i - 1] + 1;
        if (cont) {
            ci.runs.back().z1 = cz[i];
        } else {
            ci.runs.push_back({cz[i], cz[i], i});
            col_of_run.push_back((cx[i] - xmin) * ci.ny + (cy[i] - ymin));
        }
    }
    for (int c : col_of_run) ci.col_first[c + 1]++;
    for (size_t c = 0; c + 1 < ci.col_first.size(); ++c) ci.col_first[c + 1] += ci.col_first[c];

    // metadata and segments
    t.meta.assign(t.ld, 0);
    t.seg_base.assign(t.nblocks + 1, 0);
    t.seg_delta.clear();
    t.aux.assign(t.ld, -1);
    std::vector<char> defined(Q, 0);
    int cur = -1;
    int nb[Q];
    for (int i = 0; i < n; ++i) {
        uint64_t mask = 0;
        for (int q = 0; q < Q; ++q) {
            nb[q] = q == L::REST ? i : ci.lookup(cx[i] + L::cx(q), cy[i] + L::cy(q), cz[i] + L::cz(q));
            if (nb[q] >= 0) mask |= 1ull << q;
        }
        bool fresh = cur < 0 || i % BLOCK_NODES == 0;
        if (!fresh)
            for (int q = 0; q < Q; ++q)
                if (nb[q] >= 0 && defined[q] && t.seg_delta[(size_t)cur * Q + q] != nb[q] - i) {
                    fresh = true;
                    break;
                }
        if (fresh) {
            cur = t.nseg++;
            t.seg_delta.resize((size_t)t.nseg * Q, 0);
            std::fill(defined.begin(), defined.end(), 0);
            if (i % BLOCK_NODES == 0) t.seg_base[i / BLOCK_NODES] = cur;
        }
        for (int q = 0; q < Q; ++q)
            if (nb[q] >= 0 && !defined[q]) {
                t.seg_delta[(size_t)cur * Q + q] = nb[q] - i;
                defined[q] = 1;
            }
        const uint64_t rel = (uint64_t)(cur - t.seg_base[i / BLOCK_NODES]);
        if (rel >> M::SEG_BITS) return "segment index overflow";
        t.meta[i] = mask | ((uint64_t)kind[i] << M::KIND_SHIFT) | (rel << M::SEG_SHIFT);
    }
    t.seg_base[t.nblocks] = t.nseg;
    for (int b = 0; b < t.nblocks; ++b) t.max_block_segs = std::max(t.max_block_segs, t.seg_base[b + 1] - t.seg_base[b]);

    auto node_of = [&](int64_t caller, int want_kind, const char* what, std::string& err) -> int {
        if (caller < 0 || caller >= n) {
            err = std::string(what) + " index out of range";
            return -1;
        }
        const int i = t.iperm[caller];
        if (kind[i] != want_kind) {
            err = std::string(what) + " list names a node of another kind";
            return -1;
        }
        return i;
    };
    std::string err;

    // inlet
    if (d.n_inlet < 0 || (d.n_inlet > 0 && !d.inlet)) return "bad inlet list";
    long long n_in_kind = 0, n_out_kind = 0;
    for (int i = 0; i < n; ++i) {
        n_in_kind += kind[i] == KIND_INLET;
        n_out_kind += kind[i] == KIND_OUTLET;
    }
    if (d.n_inlet != n_in_kind) return "inlet list does not match the inlet node count";
    for (int64_t k = 0; k < d.n_inlet; ++k) {
        const int i = node_of(d.inlet[k], KIND_INLET, "inlet", err);
        if (i < 0) return err;
        if (t.aux[i] >= 0) return "node listed twice in the inlet list";
        t.aux[i] = (int)k;
        t.in_node.push_back(i);
    }

    // outlets, with the reference's in-order copy sweep resolved to sources
    if (d.n_outlets < 0 || (d.n_outlets > 0 && (!d.outlet_offsets || !d.outlet_nodes || !d.outlet_normals)))
        return "bad outlet description";
    std::vector<int> src_of(n, -2);  // -2: not swept yet
    for (int o = 0; o < d.n_outlets; ++o) {
        const double* nr = d.outlet_normals + 3 * o;
        int dd[3] = {0, 0, 0};
        bool any = true;
        if (nr[0] > 0) dd[0] = -1;
        else if (nr[0] < 0) dd[0] = 1;
        else if (nr[1] > 0) dd[1] = -1;
        else if (nr[1] < 0) dd[1] = 1;
        else if (nr[2] > 0) dd[2] = -1;
        else if (nr[2] < 0) dd[2] = 1;
        else any = false;
        const int64_t b = d.outlet_offsets[o], e = d.outlet_offsets[o + 1];
        if (b < 0 || e < b) return "bad outlet offsets";
        if (o == 0) t.out_off.push_back(0);
        t.out_off.push_back((long long)(t.out_node.size() + (e - b)));
        for (int c = 0; c < 3; ++c) t.out_normal.push_back(nr[c]);
        for (int64_t k = b; k < e; ++k) {
            const int i = node_of(d.outlet_nodes[k], KIND_OUTLET, "outlet", err);
            if (i < 0) return err;
            if (src_of[i] != -2) return "node listed twice in the outlet lists";
            int src = -1;
            if (any) {
                const int m = ci.lookup(cx[i] + dd[0], cy[i] + dd[1], cz[i] + dd[2]);
                if (m >= 0) src = (src_of[m] >= 0) ? src_of[m] : m;
            }
            src_of[i] = src;
            t.aux[i] = (int)t.out_node.size();
            t.out_node.push_back(i);
            // a source that is an inlet node is encoded -(src + 2): the
            // boundary pass applies its Zou-He update before copying
            t.out_src.push_back(src >= 0 && kind[src] == KIND_INLET ? -(src + 2) : src);
            for (int c = 0; c < 3; ++c) t.out_nrm.push_back((float)nr[c]);
        }
    }
    if ((long long)t.out_node.size() != n_out_kind) return "outlet lists do not match the outlet node count";

    // walls: only checked; the kernels use the node kind
    if (d.n_wall < 0 || (d.n_wall > 0 && !d.wall)) return "bad wall list";
    for (int64_t k = 0; k < d.n_wall; ++k)
        if (node_of(d.wall[k], KIND_WALL, "wall", err) < 0) return err;

    // near-wall nodes keep the caller's list order; like the reference's
    // nextToTheWall set (Subdomain.cpp:475-493) they are plain fluid nodes,
    // each listed once
    if (d.n_nearwall < 0 || (d.n_nearwall > 0 && (!d.nearwall || !d.nearwall_normals))) return "bad near-wall list";
    for (int64_t k = 0; k < d.n_nearwall; ++k) {
        const int i = node_of(d.nearwall[k], KIND_FLUID, "near-wall", err);
        if (i < 0) return err;
        if ((t.meta[i] >> M::NW_SHIFT) & 1) return "node listed twice in the near-wall list";
        t.meta[i] |= 1ull << M::NW_SHIFT;
        t.aux[i] = (int)k;
        t.nw_node.push_back(i);
        for (int c = 0; c < 3; ++c) t.nw_normal.push_back(d.nearwall_normals[3 * k + c]);
    }
    return "";
}

// Inlet waveform of the reference (Simulation::getInletVelocity,
// Simulation.cpp:519-534, with the polynomial pieces of pulsatile.h:55-69),
// evaluated on the host with the same expressions so the per-step velocity
// equals the reference's.
double waveform_piece(int piece, double x) {
    if (piece == 1)
        return (-8.579e+08 * std::pow(x, 8) + 4.059e+08 * std::pow(x, 7) - 7.817e+07 * std::pow(x, 6) +
                7.994e+06 * std::pow(x, 5) - 4.835e+05 * std::pow(x, 4) + 1.782e+04 * std::pow(x, 3) -
                321.6 * std::pow(x, 2) + 3.215 * x + 0.1423);
    if (piece == 2)
        return (-4.32e+06 * std::pow(x, 8) + 7.94e+06 * std::pow(x, 7) - 6.298e+06 * std::pow(x, 6) +
                2.82e+06 * std::pow(x, 5) - 7.809e+05 * std::pow(x, 4) + 1.37e+05 * std::pow(x, 3) -
                1.484e+04 * std::pow(x, 2) + 901.9 * x - 22.87);
    return (-5.123 * std::pow(x, 4) + 14.15 * std::pow(x, 3) - 14.21 * std::pow(x, 2) + 5.865 * x - 0.5696);
}

double pulsatile_velocity(double t, double period) {
    const double x = std::fmod(t, period);
    if (x >= 0 && x < (0.1 * period)) return waveform_piece(1, x);
    if (x >= (0.1 * period) && x < (0.3 * period)) return waveform_piece(2, x);
    if (x >= (0.3 * period) && x < (0.9 * period)) return waveform_piece(3, x);
    return 0.0;
}

template <class S, int Q>
struct Tag {
    using St = S;
    static constexpr int q = Q;
};

}  // namespace

struct lbm_engine {
    std::string err = "no error";
    int Q = 19, storage = 0, bc = 0, device = 0;
    Topo t;
    double tau = 1, omega = 1, dt = 0, spacing = 1, wss_c = 0;
    double inlet_normal[3] = {0, 0, 0};
    int flow = LBM_FLOW_CONSTANT;
    bool pulse_custom = false;  // lbm_set_pulsatile pieces instead of the reference's
    lbm::Pulse pulse;
    double cte_vel = 0.0, out_rho = 1.0;
    int64_t step = 0;
    double runtime = 0.0;
    int phase = 1;
    bool observe = true;       // lbm_set_observation
    bool force_general = false;  // LBM_B200_PHASE1_GENERAL=1: phase-1 pair kernel without its twin path
    int64_t mom_step[2] = {-1, -1};  // step whose collision-input moments each obs_mom buffer holds
    int64_t pop_step = -1;           // step whose post-boundary populations obs_pop holds
    bool wss_pending = false;  // a step kernel handed near-wall populations not yet reduced to WSS
    bool fresh = false;        // no step since the last initialisation
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    size_t bytes = 0;
    std::vector<void*> allocs;
    // device buffers
    void* pop = nullptr;
    void* meta = nullptr;
    int* seg_base = nullptr;
    int* seg_delta = nullptr;
    int* seg_slot = nullptr;   // pair phase-1 kernel: [segments][Q] d * ld + delta (mod 2^32)
    int* aux = nullptr;
    int* out_src = nullptr;
    void* out_buf = nullptr;
    float* out_nrm = nullptr;
    int* nw_node = nullptr;
    double* nw_normal = nullptr;   // FP64 normals (adjoint)
    void* nw_normal_c = nullptr;   // normals in the compute type (wall shear stress)
    void* nw_mom = nullptr;        // [n_nw][4] in the compute type
    void* nw_s = nullptr;
    double* wss = nullptr;
    double* acc = nullptr;
    double* accmag = nullptr;
    double* obs_pop = nullptr;
    double* obs_mom[2] = {nullptr, nullptr};
    unsigned* flags = nullptr;
    int* tile_sched = nullptr;  // [2] phase-1 tile counter, CTAs done (zero between launches)
    double* in_vel = nullptr;
    int* in_node = nullptr;    // internal index per inlet-list entry
    int* out_node = nullptr;   // internal index per outlet-table entry
    double* io_u = nullptr;    // physics mode: outlet node velocities [n_out][3]
    // harmonic waveform: factor 1 + sum_k amp_k cos(2 pi k t / period + phase_k), t in steps
    double wave_period = 1.0;
    std::vector<double> wave_amp, wave_phase;
    int* perm = nullptr;
    // host copies for the result writers: caller-order coordinates, near-wall list
    std::vector<int32_t> host_coords;
    std::vector<int64_t> host_nearwall;
    long long* flux_nodes = nullptr;  // internal indices: the inlet list, then the outlet lists
    double* flux_partials = nullptr;
    double* flux_out = nullptr;
    double* staging = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> evpool;
    // numeric-fault detection (lbm_set_numeric_check): the device flags are
    // copied into pinned host memory behind the steps and read once that copy
    // has completed, so the check never waits for the GPU
    bool numeric_check = true;
    unsigned* flag_host = nullptr;     // pinned mirror of *flags
    cudaEvent_t flag_ev = nullptr;     // recorded after the mirror's copy
    bool flag_copy_pending = false;
    bool numeric_fault = false;        // a completed copy showed FLAG_NONFINITE
    // slab halo lists (lbm_halo_define): slot indices q * ld + internal node
    struct HaloList {
        int64_t n = -1;  // -1: not defined
        long long* slots = nullptr;
    };
    HaloList halo[64];

    template <class T>
    cudaError_t alloc(T** p, size_t count) {
        const size_t b = std::max<size_t>(count, 1) * sizeof(T);
        cudaError_t e = cudaMalloc((void**)p, b);
        if (e == cudaSuccess) {
            allocs.push_back(*p);
            bytes += b;
        }
        return e;
    }
    template <class T>
    cudaError_t upload(T** p, const std::vector<T>& h) {
        cudaError_t e = alloc(p, h.size());
        if (e != cudaSuccess || h.empty()) return e;
        return cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    }
    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* where) {
        err = std::string(where) + ": " + cudaGetErrorString(e);
        return LBM_ERR_CUDA;
    }
    bool shifted() const { return storage != LBM_STORE_F64; }
    int nw() const { return (int)t.nw_node.size(); }
    int nout() const { return (int)t.out_node.size(); }
    int nin() const { return (int)t.in_node.size(); }
};

namespace {

template <class F>
int dispatch(lbm_engine* e, F&& f) {
    const bool q19 = e->Q == 19;
    switch (e->storage) {
        case LBM_STORE_F64: return q19 ? f(Tag<double, 19>{}) : f(Tag<double, 27>{});
        case LBM_STORE_F32: return q19 ? f(Tag<float, 19>{}) : f(Tag<float, 27>{});
        case LBM_STORE_F16: return q19 ? f(Tag<__half, 19>{}) : f(Tag<__half, 27>{});
        default: return q19 ? f(Tag<__nv_bfloat16, 19>{}) : f(Tag<__nv_bfloat16, 27>{});
    }
}

template <class S, int Q>
StepArgs<S, Q> step_args(lbm_engine* e, double vel, double* mom) {
    using C = typename Store<S>::C;
    StepArgs<S, Q> a{};
    a.pop = (S*)e->pop;
    a.ld = e->t.ld;
    a.n = e->t.n;
    a.meta = (const typename Meta<Q>::T*)e->meta;
    a.seg_base = e->seg_base;
    a.seg_delta = e->seg_delta;
    a.seg_slot = e->seg_slot;
    a.seg_smem_bytes = e->t.max_block_segs * Q * (int)sizeof(int);
    a.aux = e->aux;
    a.omega = (C)e->omega;
    for (int c = 0; c < 3; ++c) a.inlet_normal[c] = e->inlet_normal[c];
    a.inlet_vel = vel;
    a.out_src = e->out_src;
    a.out_buf = (const C*)e->out_buf;
    a.io_u = e->io_u;
    a.nw_s = (C*)e->nw_s;
    a.n_nw = e->nw();
    a.obs_pop = e->obs_pop;
    a.obs_mom = mom;
    a.flags = e->flags;
    a.force_general = e->force_general ? 1 : 0;
    a.tile_sched = e->tile_sched;
    return a;
}

template <class S, int Q>
BoundaryArgs<S, Q> boundary_args(lbm_engine* e, double vel, bool with_wss, bool with_outlets) {
    using C = typename Store<S>::C;
    BoundaryArgs<S, Q> b{};
    b.pop = (const S*)e->pop;
    b.ld = e->t.ld;
    b.meta = (const typename Meta<Q>::T*)e->meta;
    b.seg_base = e->seg_base;
    b.seg_delta = e->seg_delta;
    b.n_wss = with_wss ? e->nw() : 0;
    b.n_nw = e->nw();
    b.nw_s = (const C*)e->nw_s;
    b.nw_normal = (const C*)e->nw_normal_c;
    b.nw_mom = (C*)e->nw_mom;
    b.wss = e->wss;
    b.acc = e->acc;
    b.accmag = e->accmag;
    b.wss_c = e->wss_c;
    b.n_out = (with_outlets && e->bc == LBM_BC_REFERENCE) ? e->nout() : 0;
    b.out_src = e->out_src;
    b.out_buf = (C*)e->out_buf;
    for (int c = 0; c < 3; ++c) b.inlet_normal[c] = e->inlet_normal[c];
    b.inlet_vel = vel;
    return b;
}

template <class S, int Q>
OpenArgs<S, Q> open_args(lbm_engine* e, double scale) {
    OpenArgs<S, Q> o{};
    o.pop = (S*)e->pop;
    o.ld = e->t.ld;
    o.meta = (const typename Meta<Q>::T*)e->meta;
    o.n_in = e->nin();
    o.in_node = e->in_node;
    o.in_vel = e->in_vel;
    o.in_scale = scale;
    for (int c = 0; c < 3; ++c) o.in_normal[c] = e->inlet_normal[c];
    o.n_out = e->nout();
    o.out_node = e->out_node;
    o.out_nrm = e->out_nrm;
    o.io_u = e->io_u;
    o.out_rho = e->out_rho;
    return o;
}

// Pulsatile inlet velocity at flow clock t: the reference's waveform, or the
// pieces given with lbm_set_pulsatile.
double pulsatile_at(const lbm_engine* e, double t) {
    return e->pulse_custom ? lbm::pulse_value(e->pulse, t) : pulsatile_velocity(t, 0.9);
}

// Inlet waveform factor of step k (0-based) whose flow clock reads runtime_k:
// 1 for constant flow, the reference waveform value for pulsatile flow, the
// harmonic factor for harmonic flow.
double inlet_factor(const lbm_engine* e, int64_t k, double runtime_k) {
    if (e->flow == LBM_FLOW_PULSATILE) return pulsatile_at(e, runtime_k);
    double f = 1.0;
    if (e->flow == LBM_FLOW_HARMONIC) {
        const double two_pi = 6.283185307179586;
        for (size_t h = 0; h < e->wave_amp.size(); ++h)
            f += e->wave_amp[h] * std::cos(two_pi * (double)(h + 1) * (double)k / e->wave_period + e->wave_phase[h]);
    }
    return f;
}

// Physics mode: corrects the open-boundary links of the store just issued,
// which streams into step k.
int open_pass(lbm_engine* e, int64_t k, double runtime_k) {
    if (e->bc != LBM_BC_PHYSICS || e->nin() + e->nout() == 0) return 0;
    const double scale = inlet_factor(e, k, runtime_k);
    return dispatch(e, [&](auto tag) {
        using S = typename decltype(tag)::St;
        constexpr int Q = decltype(tag)::q;
        cudaError_t ce = launch_open<S, Q>(open_args<S, Q>(e, scale), e->stream);
        return ce == cudaSuccess ? 0 : e->cuda_fail(ce, "open-boundary kernel");
    });
}

// Collides the natural-layout state in obs_pop into the AA buffer and primes
// the near-wall moments; the next step reads phase 1.
int init_from_obs(lbm_engine* e) {
    const int mb = (int)(e->step % 2);
    int rc = dispatch(e, [&](auto tag) {
        using S = typename decltype(tag)::St;
        constexpr int Q = decltype(tag)::q;
        auto a = step_args<S, Q>(e, 0.0, e->obs_mom[mb]);
        cudaError_t ce = launch_init<S, Q>(a, e->bc, e->stream);
        return ce == cudaSuccess ? 0 : e->cuda_fail(ce, "init kernel");
    });
    if (rc) return rc;
    if (int rc2 = open_pass(e, e->step, e->runtime)) return rc2;
    cudaError_t ce = launch_nearwall_moments(e->nw(), e->nw_node, e->obs_mom[mb], e->t.ld, e->shifted(),
                                             e->nw_mom, e->storage != LBM_STORE_F64, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "near-wall moments");
    e->phase = 1;
    e->wss_pending = false;
    e->mom_step[mb] = e->step;
    e->mom_step[1 - mb] = -1;
    e->pop_step = e->step;
    e->fresh = true;
    return 0;
}

// Reads the flag mirror if its copy has completed (never blocks).
void poll_flags(lbm_engine* e) {
    if (!e->flag_copy_pending) return;
    const cudaError_t q = cudaEventQuery(e->flag_ev);
    if (q == cudaErrorNotReady) return;
    if (q != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    e->flag_copy_pending = false;
    if (*e->flag_host & FLAG_NONFINITE) e->numeric_fault = true;
}

// Queues a copy of the device flags into the mirror behind the work issued so
// far (one copy in flight at a time).
void post_flags(lbm_engine* e) {
    if (e->flag_copy_pending) return;
    if (cudaMemcpyAsync(e->flag_host, e->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess ||
        cudaEventRecord(e->flag_ev, e->stream) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    e->flag_copy_pending = true;
}

// Steps between two flag copies inside one lbm_step call.
constexpr int64_t FLAG_POLL_STEPS = 256;

// LBM_ERR_NUMERIC once a completed copy of the device flags showed
// non-finite densities (when the check is on).
int numeric_status(lbm_engine* e) {
    if (!e->numeric_check) return 0;
    poll_flags(e);
    if (!e->numeric_fault) return 0;
    return e->fail(LBM_ERR_NUMERIC, "non-finite densities reported by the device by step " + std::to_string(e->step) +
                                        " (lbm_set_numeric_check(e, 0) runs on regardless)");
}

// Observation bits of a step followed by `left` more steps of its call: the
// last two steps write the moments, the last one the populations too.
int observe_bits(const lbm_engine* e, int64_t left) {
    if (!e->observe) return 0;
    return (left <= 1 ? 2 : 0) | (left == 0 ? 1 : 0);
}

// Timed runs (lbm_step_timed) record events around sampled steps only: the
// two steps (one of each phase) that begin every TIMING_STRIDE steps. An
// event between two kernels of a stream costs the stream about 5 us, which
// events around every step would add to the very time they measure (1.8 % of
// a step of the 21.4M-node vessel, 15-28 % on lattices of about a million
// nodes). The per-class sums are the sampled steps' averages times the
// step count; each sampled step uses three events.
constexpr int64_t TIMING_STRIDE = 32;
bool timing_sample(int64_t i) { return i % TIMING_STRIDE < 2; }
int64_t timing_samples(int64_t n) { return (n / TIMING_STRIDE) * 2 + std::min<int64_t>(n % TIMING_STRIDE, 2); }

// Physics mode: per step the stream+collide kernel, then one post-pass with
// that step's wall shear stress and the open-boundary corrections of its
// store (which streams into the next step). No pre-pass: physics mode has no
// outlet copy sources. A sampled step of a timed run records events before
// its step kernel, before its post-pass and after it. A WSS hand-off left
// pending by an earlier reference-style sequence is reduced first (never the
// case in physics mode, where every post-pass reduces it).
int run_steps_physics(lbm_engine* e, int64_t n_steps, int64_t after, double* t_step, double* t_bnd) {
    const bool timed = t_step || t_bnd;
    const bool pulsatile = e->flow == LBM_FLOW_PULSATILE;
    int64_t sample = 0;
    for (int64_t i = 0; i < n_steps; ++i) {
        const int64_t t = e->step + 1;
        const int obs = observe_bits(e, n_steps - 1 - i + after);
        double* mom = e->obs_mom[t % 2];
        const int phase = e->phase;
        const double scale = inlet_factor(e, e->step + 1, pulsatile ? e->runtime + e->dt : e->runtime);
        cudaEvent_t* ev = timed && timing_sample(i) ? &e->evpool[3 * sample++] : nullptr;
        int rc = dispatch(e, [&](auto tag) {
            using S = typename decltype(tag)::St;
            constexpr int Q = decltype(tag)::q;
            cudaError_t ce = cudaSuccess;
            if (e->wss_pending) {
                ce = launch_boundary<S, Q>(boundary_args<S, Q>(e, 0.0, true, false), phase, e->stream);
                if (ce != cudaSuccess) return e->cuda_fail(ce, "wall shear kernel");
                e->wss_pending = false;
            }
            if (ev) cudaEventRecord(ev[0], e->stream);
            ce = launch_step<S, Q>(step_args<S, Q>(e, 0.0, mom), phase, e->bc, obs, e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "step kernel");
            if (ev) cudaEventRecord(ev[1], e->stream);
            ce = launch_post<S, Q>(boundary_args<S, Q>(e, 0.0, e->nw() > 0, false), open_args<S, Q>(e, scale),
                                   e->stream);
            if (ev) cudaEventRecord(ev[2], e->stream);
            return ce == cudaSuccess ? 0 : e->cuda_fail(ce, "post-step kernel");
        });
        if (rc) return rc;
        if (obs & 2) e->mom_step[t % 2] = t;
        if (obs & 1) e->pop_step = t;
        e->phase ^= 1;
        e->step = t;
        if (pulsatile) e->runtime += e->dt;
        e->fresh = false;
    }
    if (timed && sample > 0) {
        cudaError_t ce = cudaEventSynchronize(e->evpool[3 * sample - 1]);
        if (ce != cudaSuccess) return e->cuda_fail(ce, "timed steps");
        double ms_step = 0, ms_bnd = 0;
        for (int64_t j = 0; j < sample; ++j) {
            float a = 0, b = 0;
            cudaEventElapsedTime(&a, e->evpool[3 * j], e->evpool[3 * j + 1]);
            cudaEventElapsedTime(&b, e->evpool[3 * j + 1], e->evpool[3 * j + 2]);
            ms_step += a;
            ms_bnd += b;
        }
        const double scale = (double)n_steps / (double)sample;
        if (t_step) *t_step = ms_step * scale;
        if (t_bnd) *t_bnd = ms_bnd * scale;
    }
    return 0;
}

int run_steps_checked(lbm_engine* e, int64_t n_steps, int64_t after, double* t_step, double* t_bnd);

// Runs n_steps steps in chunks of FLAG_POLL_STEPS with a flag copy behind each
// chunk; with the numeric check on, stops before the next chunk once a copy
// that has completed shows non-finite densities.
int run_steps(lbm_engine* e, int64_t n_steps, double* t_step, double* t_bnd) {
    if (n_steps < 0) return e->fail(LBM_ERR_ARGUMENT, "negative step count");
    if (int rc = numeric_status(e)) return rc;
    if (t_step || t_bnd) {
        // timed runs are one chunk: their events are read once at the end
        const int rc = run_steps_checked(e, n_steps, 0, t_step, t_bnd);
        post_flags(e);
        return rc;
    }
    for (int64_t done = 0; done < n_steps;) {
        const int64_t chunk = std::min<int64_t>(FLAG_POLL_STEPS, n_steps - done);
        if (int rc = run_steps_checked(e, chunk, n_steps - done - chunk, nullptr, nullptr)) return rc;
        done += chunk;
        post_flags(e);
        if (done < n_steps)
            if (int rc = numeric_status(e)) return rc;
    }
    return 0;
}

// `after`: steps of the same lbm_step call that follow these (the call's
// last two steps are the observed ones).
int run_steps_checked(lbm_engine* e, int64_t n_steps, int64_t after, double* t_step, double* t_bnd) {
    if (n_steps == 0) return 0;
    if (t_step) *t_step = 0;
    if (t_bnd) *t_bnd = 0;
    const bool timed = t_step || t_bnd;
    // timed runs: three events per sampled step (timing_sample) and two
    // around the last step's wall-shear pass in reference mode, read once at
    // the end so timing adds no host round trip between steps
    if (timed) {
        if (n_steps > (1 << 24)) return e->fail(LBM_ERR_ARGUMENT, "too many timed steps in one call");
        while ((int64_t)e->evpool.size() < 3 * timing_samples(n_steps) + 2) {
            cudaEvent_t ev;
            cudaError_t ce = cudaEventCreate(&ev);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "event");
            e->evpool.push_back(ev);
        }
    }
    if (e->bc == LBM_BC_PHYSICS) return run_steps_physics(e, n_steps, after, t_step, t_bnd);
    int64_t sample = 0;
    for (int64_t i = 0; i < n_steps; ++i) {
        const int64_t t = e->step + 1;
        const bool pulsatile = e->flow == LBM_FLOW_PULSATILE;
        // reference-mode inlet velocity of this step (Simulation.cpp:558-562)
        const double vel = pulsatile ? pulsatile_at(e, e->runtime)
                                     : e->cte_vel * inlet_factor(e, e->step, e->runtime);
        const int obs = observe_bits(e, n_steps - 1 - i + after);
        double* mom = e->obs_mom[t % 2];
        const int phase = e->phase;
        cudaEvent_t* ev = timed && timing_sample(i) ? &e->evpool[3 * sample++] : nullptr;
        int rc = dispatch(e, [&](auto tag) {
            using S = typename decltype(tag)::St;
            constexpr int Q = decltype(tag)::q;
            if (ev) cudaEventRecord(ev[0], e->stream);
            cudaError_t ce =
                launch_boundary<S, Q>(boundary_args<S, Q>(e, vel, e->wss_pending, true), phase, e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "boundary kernel");
            if (ev) cudaEventRecord(ev[1], e->stream);
            ce = launch_step<S, Q>(step_args<S, Q>(e, vel, mom), phase, e->bc, obs, e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "step kernel");
            if (ev) cudaEventRecord(ev[2], e->stream);
            return 0;
        });
        if (rc) return rc;
        // physics mode: this store streams into the next step
        if (int rc2 = open_pass(e, e->step + 1, pulsatile ? e->runtime + e->dt : e->runtime)) return rc2;
        if (obs & 2) e->mom_step[t % 2] = t;
        if (obs & 1) e->pop_step = t;
        e->wss_pending = e->nw() > 0;
        e->phase ^= 1;
        e->step = t;
        if (pulsatile) e->runtime += e->dt;
        e->fresh = false;
    }
    // wall shear stress of the last step
    cudaEvent_t* last_ev = timed ? &e->evpool[3 * sample] : nullptr;
    if (last_ev) cudaEventRecord(last_ev[0], e->stream);
    if (e->wss_pending) {
        int rc = dispatch(e, [&](auto tag) {
            using S = typename decltype(tag)::St;
            constexpr int Q = decltype(tag)::q;
            cudaError_t ce = launch_boundary<S, Q>(boundary_args<S, Q>(e, 0.0, true, false), e->phase, e->stream);
            return ce == cudaSuccess ? 0 : e->cuda_fail(ce, "wall shear kernel");
        });
        if (rc) return rc;
        e->wss_pending = false;
    }
    if (timed) {
        cudaEventRecord(last_ev[1], e->stream);
        cudaError_t ce = cudaEventSynchronize(last_ev[1]);
        if (ce != cudaSuccess) return e->cuda_fail(ce, "timed steps");
        double ms_step = 0, ms_bnd = 0;
        for (int64_t j = 0; j < sample; ++j) {
            float a = 0, b = 0;
            cudaEventElapsedTime(&a, e->evpool[3 * j], e->evpool[3 * j + 1]);
            cudaEventElapsedTime(&b, e->evpool[3 * j + 1], e->evpool[3 * j + 2]);
            ms_bnd += a;
            ms_step += b;
        }
        const double scale = sample > 0 ? (double)n_steps / (double)sample : 0.0;
        ms_step *= scale;
        ms_bnd *= scale;
        float last = 0;
        cudaEventElapsedTime(&last, last_ev[0], last_ev[1]);
        ms_bnd += last;
        if (t_step) *t_step = ms_step;
        if (t_bnd) *t_bnd = ms_bnd;
    }
    return 0;
}

int ensure_staging(lbm_engine* e) {
    if (e->staging) return 0;
    cudaError_t ce = e->alloc(&e->staging, (size_t)e->t.n * e->Q);
    return ce == cudaSuccess ? 0 : e->cuda_fail(ce, "staging buffer");
}

int sync(lbm_engine* e) {
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? 0 : e->cuda_fail(ce, "stream synchronize");
}


int create(const lbm_desc* d, lbm_engine** out) {
    if (!d || !out) {
        g_create_error = "null descriptor or output pointer";
        return LBM_ERR_ARGUMENT;
    }
    *out = nullptr;
    if (d->lattice != 19 && d->lattice != 27) {
        g_create_error = "lattice must be 19 or 27";
        return LBM_ERR_ARGUMENT;
    }
    if (d->storage < 0 || d->storage > 3) {
        g_create_error = "storage must be 0..3";
        return LBM_ERR_ARGUMENT;
    }
    if (d->bc_mode != LBM_BC_REFERENCE && d->bc_mode != LBM_BC_PHYSICS) {
        g_create_error = "bc_mode must be 0 or 1";
        return LBM_ERR_ARGUMENT;
    }
    if (d->bc_mode == LBM_BC_REFERENCE && d->lattice != 19) {
        g_create_error = "reference boundaries are defined for D3Q19 only (Boundary.cpp uses D3Q19 indices)";
        return LBM_ERR_ARGUMENT;
    }
    if (!(d->tau > 0.5)) {
        g_create_error = "tau must exceed 0.5";
        return LBM_ERR_ARGUMENT;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_create_error = "no CUDA device";
        return LBM_ERR_NO_DEVICE;
    }
    if (d->device < 0 || d->device >= ndev) {
        g_create_error = "device ordinal out of range";
        return LBM_ERR_ARGUMENT;
    }
    lbm_engine* e = new lbm_engine();
    e->Q = d->lattice;
    e->storage = d->storage;
    e->bc = d->bc_mode;
    e->device = d->device;
    e->tau = d->tau;
    e->omega = 1.0 / d->tau;
    e->dt = d->dt;
    e->spacing = d->spacing;
    {
        // tests compare the phase-1 pair kernel's twin and per-node paths
        const char* g = getenv("LBM_B200_PHASE1_GENERAL");
        e->force_general = g && !strcmp(g, "1");
    }
    {
        // Simulation::ComputeWallShearStress, Simulation.cpp:768-771
        const double phys_den = 1060;
        const double dtdt = d->dt * d->dt;
        const double dxdx = d->spacing * d->spacing * 1e-6;
        e->wss_c = phys_den * dtdt / dxdx;
    }
    for (int c = 0; c < 3; ++c) e->inlet_normal[c] = d->inlet_normal[c];
    std::string msg = e->Q == 19 ? build_topology<19>(*d, e->t) : build_topology<27>(*d, e->t);
    if (!msg.empty()) {
        g_create_error = msg;
        delete e;
        return LBM_ERR_ARGUMENT;
    }
    e->host_coords.assign(d->coords, d->coords + 3 * d->n_nodes);
    if (d->n_nearwall > 0) e->host_nearwall.assign(d->nearwall, d->nearwall + d->n_nearwall);
    auto bail = [&](cudaError_t ce, const char* where) {
        g_create_error = std::string(where) + ": " + cudaGetErrorString(ce);
        lbm_destroy(e);
        return LBM_ERR_CUDA;
    };
    cudaError_t ce = cudaSetDevice(e->device);
    if (ce != cudaSuccess) return bail(ce, "cudaSetDevice");
    ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return bail(ce, "stream");
    e->own_stream = true;
    for (auto& ev : e->ev)
        if ((ce = cudaEventCreate(&ev)) != cudaSuccess) return bail(ce, "event");
    if ((ce = cudaEventCreateWithFlags(&e->flag_ev, cudaEventDisableTiming)) != cudaSuccess) return bail(ce, "event");
    if ((ce = cudaHostAlloc((void**)&e->flag_host, sizeof(unsigned), cudaHostAllocDefault)) != cudaSuccess)
        return bail(ce, "flag mirror");
    *e->flag_host = 0;

    const Topo& t = e->t;
    const size_t elem = e->storage == LBM_STORE_F64 ? 8 : (e->storage == LBM_STORE_F32 ? 4 : 2);
    const size_t celem = e->storage == LBM_STORE_F64 ? 8 : 4;
    char* p = nullptr;
    if ((ce = e->alloc(&p, (size_t)e->Q * t.ld * elem)) != cudaSuccess) return bail(ce, "population buffer");
    e->pop = p;
    if (e->Q == 19) {
        std::vector<uint32_t> m32(t.meta.begin(), t.meta.end());
        uint32_t* mp = nullptr;
        if ((ce = e->upload(&mp, m32)) != cudaSuccess) return bail(ce, "metadata");
        e->meta = mp;
    } else {
        std::vector<unsigned long long> m64(t.meta.begin(), t.meta.end());
        unsigned long long* mp = nullptr;
        if ((ce = e->upload(&mp, m64)) != cudaSuccess) return bail(ce, "metadata");
        e->meta = mp;
    }
    if ((ce = e->upload(&e->seg_base, t.seg_base)) != cudaSuccess) return bail(ce, "segments");
    if ((ce = e->upload(&e->seg_delta, t.seg_delta)) != cudaSuccess) return bail(ce, "segments");
    if (e->shifted() && e->bc == LBM_BC_PHYSICS && (long long)e->Q * t.ld < (1LL << 32)) {
        // the pair phase-1 kernel's row entry for direction d is the slot
        // offset d * ld + delta, taken modulo 2^32 (its slot indices are
        // 32-bit; the launcher runs it only when Q * ld < 2^32)
        std::vector<int> slot(t.seg_delta.size());
        for (size_t i = 0; i < slot.size(); ++i) {
            const uint32_t d = (uint32_t)(i % (size_t)e->Q);
            slot[i] = (int)(d * (uint32_t)t.ld + (uint32_t)t.seg_delta[i]);
        }
        if ((ce = e->upload(&e->seg_slot, slot)) != cudaSuccess) return bail(ce, "segments");
    }
    if ((ce = e->upload(&e->aux, t.aux)) != cudaSuccess) return bail(ce, "aux");
    if ((ce = e->upload(&e->out_src, t.out_src)) != cudaSuccess) return bail(ce, "outlets");
    if ((ce = e->upload(&e->out_nrm, t.out_nrm)) != cudaSuccess) return bail(ce, "outlets");
    char* ob = nullptr;
    if ((ce = e->alloc(&ob, (size_t)std::max(1, e->nout()) * e->Q * celem)) != cudaSuccess)
        return bail(ce, "outlet buffer");
    e->out_buf = ob;
    if ((ce = e->upload(&e->nw_node, t.nw_node)) != cudaSuccess) return bail(ce, "near-wall");
    if ((ce = e->upload(&e->nw_normal, t.nw_normal)) != cudaSuccess) return bail(ce, "near-wall");
    if (celem == 8) {
        e->nw_normal_c = e->nw_normal;
    } else {
        std::vector<float> nf(t.nw_normal.begin(), t.nw_normal.end());
        float* d_nf = nullptr;
        if ((ce = e->upload(&d_nf, nf)) != cudaSuccess) return bail(ce, "near-wall");
        e->nw_normal_c = d_nf;
    }
    char* nwm = nullptr;
    if ((ce = e->alloc(&nwm, (size_t)4 * std::max(1, e->nw()) * celem)) != cudaSuccess) return bail(ce, "near-wall");
    e->nw_mom = nwm;
    char* nws = nullptr;
    const size_t rows = celem == 8 ? (size_t)e->Q : (size_t)lbm::handoff_rows<float, 19>();
    if ((ce = e->alloc(&nws, rows * std::max(1, e->nw()) * celem)) != cudaSuccess) return bail(ce, "near-wall");
    e->nw_s = nws;
    if ((ce = e->alloc(&e->wss, (size_t)e->nw())) != cudaSuccess) return bail(ce, "wss");
    if ((ce = e->alloc(&e->acc, (size_t)3 * e->nw())) != cudaSuccess) return bail(ce, "wss");
    if ((ce = e->alloc(&e->accmag, (size_t)e->nw())) != cudaSuccess) return bail(ce, "wss");
    if ((ce = e->alloc(&e->obs_pop, (size_t)e->Q * t.ld)) != cudaSuccess) return bail(ce, "observation buffer");
    for (auto& m : e->obs_mom)
        if ((ce = e->alloc(&m, (size_t)4 * t.ld)) != cudaSuccess) return bail(ce, "observation buffer");
    if ((ce = e->alloc(&e->flags, 1)) != cudaSuccess) return bail(ce, "flags");
    if ((ce = e->alloc(&e->tile_sched, 2)) != cudaSuccess) return bail(ce, "tile counter");
    std::vector<double> zero_in((size_t)3 * std::max(1, e->nin()), 0.0);
    if ((ce = e->upload(&e->in_vel, zero_in)) != cudaSuccess) return bail(ce, "inlet profile");
    if ((ce = e->upload(&e->in_node, t.in_node)) != cudaSuccess) return bail(ce, "inlet list");
    if ((ce = e->upload(&e->out_node, t.out_node)) != cudaSuccess) return bail(ce, "outlet list");
    if ((ce = e->alloc(&e->io_u, (size_t)3 * std::max(1, e->nout()))) != cudaSuccess) return bail(ce, "outlet velocity");
    if ((ce = e->upload(&e->perm, t.perm)) != cudaSuccess) return bail(ce, "permutation");
    {
        std::vector<long long> fl;
        for (int i : t.in_node) fl.push_back(i);
        for (int i : t.out_node) fl.push_back(i);
        if ((ce = e->upload(&e->flux_nodes, fl)) != cudaSuccess) return bail(ce, "flux lists");
        const size_t blocks = (fl.size() + FLUX_THREADS - 1) / FLUX_THREADS + 1;
        if ((ce = e->alloc(&e->flux_partials, blocks)) != cudaSuccess) return bail(ce, "flux scratch");
        if ((ce = e->alloc(&e->flux_out, (size_t)d->n_outlets + 1)) != cudaSuccess) return bail(ce, "flux scratch");
    }

    cudaMemsetAsync(e->wss, 0, sizeof(double) * std::max(1, e->nw()), e->stream);
    cudaMemsetAsync(e->acc, 0, sizeof(double) * 3 * std::max(1, e->nw()), e->stream);
    cudaMemsetAsync(e->accmag, 0, sizeof(double) * std::max(1, e->nw()), e->stream);
    cudaMemsetAsync(e->flags, 0, sizeof(unsigned), e->stream);
    cudaMemsetAsync(e->tile_sched, 0, 2 * sizeof(int), e->stream);
    // pad slots of the population buffer stay zero
    cudaMemsetAsync(e->pop, 0, (size_t)e->Q * t.ld * elem, e->stream);
    if ((ce = launch_fill_weights(e->obs_pop, t.ld, t.n, e->Q, e->stream)) != cudaSuccess)
        return bail(ce, "initial state");
    if (int rc = init_from_obs(e)) {
        g_create_error = e->err;
        lbm_destroy(e);
        return rc;
    }
    if ((ce = cudaStreamSynchronize(e->stream)) != cudaSuccess) return bail(ce, "initialisation");
    *out = e;
    return 0;
}

}  // namespace

extern "C" {

int lbm_create(const lbm_desc* desc, lbm_engine** out) {
    try {
        return create(desc, out);
    } catch (const std::exception& ex) {
        g_create_error = ex.what();
        return LBM_ERR_ARGUMENT;
    }
}

int lbm_destroy(lbm_engine* e) {
    if (!e) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (void* p : e->allocs) cudaFree(p);
    for (auto& ev : e->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : e->evpool) cudaEventDestroy(ev);
    if (e->flag_ev) cudaEventDestroy(e->flag_ev);
    if (e->flag_host) cudaFreeHost(e->flag_host);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return 0;
}

int lbm_set_stream(lbm_engine* e, void* stream) {
    if (!e) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    e->own_stream = false;
    e->stream = (cudaStream_t)stream;
    return 0;
}

// Physics mode applies the inlet and outlet conditions when it stores a step's
// populations; a parameter set before the first step must reach the store of
// the initialisation too, so that store is redone.
static int reapply_initial_store(lbm_engine* e) {
    if (e->bc != LBM_BC_PHYSICS || !e->fresh) return 0;
    cudaSetDevice(e->device);
    if (int rc = init_from_obs(e)) return rc;
    return sync(e);
}

int lbm_set_pulsatile(lbm_engine* e, const lbm_pulse_desc* w) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (!w) {
        e->pulse_custom = false;
        return reapply_initial_store(e);
    }
    lbm::Pulse p;
    const std::string err = lbm::pulse_from_desc(*w, p);
    if (!err.empty()) return e->fail(LBM_ERR_ARGUMENT, err);
    e->pulse = std::move(p);
    e->pulse_custom = true;
    // the inlet correction of the initial store reads the waveform at t = 0
    return reapply_initial_store(e);
}

int lbm_set_waveform(lbm_engine* e, double period_steps, int32_t n_harmonics, const double* amplitude,
                     const double* phase) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (!(period_steps > 0) || n_harmonics < 0 || (n_harmonics > 0 && (!amplitude || !phase)))
        return e->fail(LBM_ERR_ARGUMENT, "bad waveform");
    e->wave_period = period_steps;
    e->wave_amp.assign(amplitude, amplitude + n_harmonics);
    e->wave_phase.assign(phase, phase + n_harmonics);
    return reapply_initial_store(e);
}

int lbm_set_flow(lbm_engine* e, int32_t flow, double cte_vel) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (flow != LBM_FLOW_CONSTANT && flow != LBM_FLOW_PULSATILE && flow != LBM_FLOW_HARMONIC)
        return e->fail(LBM_ERR_ARGUMENT, "unknown flow type");
    e->flow = flow;
    e->cte_vel = cte_vel;
    return reapply_initial_store(e);
}

int lbm_set_inlet_profile(lbm_engine* e, const double* velocity) {
    if (!e || !velocity) return LBM_ERR_ARGUMENT;
    std::vector<double> v(velocity, velocity + (size_t)3 * e->nin());
    if (v.empty()) return 0;
    cudaSetDevice(e->device);
    cudaError_t ce = cudaMemcpyAsync(e->in_vel, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "inlet profile");
    if (int rc = sync(e)) return rc;
    return reapply_initial_store(e);
}

int lbm_set_outlet_density(lbm_engine* e, double rho) {
    if (!e) return LBM_ERR_ARGUMENT;
    e->out_rho = rho;
    return reapply_initial_store(e);
}

int lbm_set_numeric_check(lbm_engine* e, int32_t enabled) {
    if (!e) return LBM_ERR_ARGUMENT;
    e->numeric_check = enabled != 0;
    return 0;
}

int lbm_set_observation(lbm_engine* e, int32_t enabled) {
    if (!e) return LBM_ERR_ARGUMENT;
    e->observe = enabled != 0;
    return 0;
}

int lbm_step(lbm_engine* e, int64_t n_steps) {
    if (!e) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    return run_steps(e, n_steps, nullptr, nullptr);
}

int lbm_step_timed(lbm_engine* e, int64_t n_steps, double* step_kernel_ms, double* boundary_kernel_ms) {
    if (!e) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    double a = 0, b = 0;
    int rc = run_steps(e, n_steps, &a, &b);
    if (step_kernel_ms) *step_kernel_ms = a;
    if (boundary_kernel_ms) *boundary_kernel_ms = b;
    return rc;
}

int lbm_get_time(lbm_engine* e, int64_t* steps, double* runtime) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (steps) *steps = e->step;
    if (runtime) *runtime = e->runtime;
    return 0;
}

}  // extern "C"

// Restart support: the state the next step reads, as one host blob.
namespace {
struct StateHeader {
    uint32_t magic, version;
    int32_t lattice, storage, bc, phase;
    int64_t n, ld, n_nw, n_segments, step;
    double runtime;
    int64_t pop_bytes, mom_bytes;
};
constexpr uint32_t STATE_MAGIC = 0x534d424cu;  // "LBMS"
constexpr uint32_t STATE_VERSION = 1;

StateHeader state_header(const lbm_engine* e) {
    StateHeader h{};
    h.magic = STATE_MAGIC;
    h.version = STATE_VERSION;
    h.lattice = e->Q;
    h.storage = e->storage;
    h.bc = e->bc;
    h.phase = e->phase;
    h.n = e->t.n;
    h.ld = e->t.ld;
    h.n_nw = e->nw();
    h.n_segments = e->t.nseg;
    h.step = e->step;
    h.runtime = e->runtime;
    const int64_t elem = e->storage == LBM_STORE_F64 ? 8 : (e->storage == LBM_STORE_F32 ? 4 : 2);
    h.pop_bytes = (int64_t)e->Q * e->t.ld * elem;
    h.mom_bytes = 4 * h.n_nw * (e->storage == LBM_STORE_F64 ? 8 : 4);
    return h;
}

int64_t state_bytes(const StateHeader& h) {
    return (int64_t)sizeof(StateHeader) + h.pop_bytes + h.mom_bytes + 5 * 8 * h.n_nw;
}
}  // namespace

extern "C" {

int lbm_state_size(lbm_engine* e, int64_t* bytes) {
    if (!e || !bytes) return LBM_ERR_ARGUMENT;
    *bytes = state_bytes(state_header(e));
    return 0;
}

int lbm_get_state(lbm_engine* e, void* dst, int64_t bytes) {
    if (!e || !dst) return LBM_ERR_ARGUMENT;
    if (e->wss_pending) return e->fail(LBM_ERR_STATE, "lbm_get_state: a wall shear stress reduction is pending");
    const StateHeader h = state_header(e);
    if (bytes < state_bytes(h))
        return e->fail(LBM_ERR_ARGUMENT, "lbm_get_state: buffer of " + std::to_string(bytes) +
                                             " bytes, the state needs " + std::to_string(state_bytes(h)));
    cudaSetDevice(e->device);
    char* p = static_cast<char*>(dst);
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    const size_t m = (size_t)h.n_nw;
    struct Part { const void* src; size_t bytes; } parts[] = {
        {e->pop, (size_t)h.pop_bytes}, {e->nw_mom, (size_t)h.mom_bytes}, {e->wss, 8 * m},
        {e->acc, 24 * m}, {e->accmag, 8 * m}};
    for (const Part& part : parts) {
        if (part.bytes) {
            cudaError_t ce = cudaMemcpyAsync(p, part.src, part.bytes, cudaMemcpyDeviceToHost, e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "state download");
        }
        p += part.bytes;
    }
    return sync(e);
}

int lbm_set_state(lbm_engine* e, const void* src, int64_t bytes) {
    if (!e || !src) return LBM_ERR_ARGUMENT;
    const StateHeader mine = state_header(e);
    if (bytes != state_bytes(mine))
        return e->fail(LBM_ERR_ARGUMENT, "lbm_set_state: blob of " + std::to_string(bytes) +
                                             " bytes, this engine's state has " + std::to_string(state_bytes(mine)));
    StateHeader h;
    std::memcpy(&h, src, sizeof h);
    if (h.magic != STATE_MAGIC || h.version != STATE_VERSION)
        return e->fail(LBM_ERR_ARGUMENT, "lbm_set_state: not a state blob of this version");
    if (h.lattice != mine.lattice || h.storage != mine.storage || h.bc != mine.bc || h.n != mine.n ||
        h.ld != mine.ld || h.n_nw != mine.n_nw || h.n_segments != mine.n_segments ||
        h.pop_bytes != mine.pop_bytes || h.mom_bytes != mine.mom_bytes)
        return e->fail(LBM_ERR_ARGUMENT,
                       "lbm_set_state: the state comes from an engine with another node set, lattice, "
                       "storage type or boundary mode");
    if ((h.phase != 0 && h.phase != 1) || h.step < 0 || !std::isfinite(h.runtime))
        return e->fail(LBM_ERR_ARGUMENT, "lbm_set_state: bad phase, step or clock");
    cudaSetDevice(e->device);
    if (int rc = sync(e)) return rc;
    const char* p = static_cast<const char*>(src) + sizeof h;
    const size_t m = (size_t)h.n_nw;
    struct Part { void* dst; size_t bytes; } parts[] = {
        {e->pop, (size_t)h.pop_bytes}, {e->nw_mom, (size_t)h.mom_bytes}, {e->wss, 8 * m},
        {e->acc, 24 * m}, {e->accmag, 8 * m}};
    for (const Part& part : parts) {
        if (part.bytes) {
            cudaError_t ce = cudaMemcpyAsync(part.dst, p, part.bytes, cudaMemcpyHostToDevice, e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "state upload");
        }
        p += part.bytes;
    }
    cudaError_t cm = cudaMemsetAsync(e->flags, 0, sizeof(unsigned), e->stream);
    if (cm != cudaSuccess) return e->cuda_fail(cm, "flags");
    if (int rc = sync(e)) return rc;
    e->step = h.step;
    e->runtime = h.runtime;
    e->phase = h.phase;
    e->flag_copy_pending = false;
    e->numeric_fault = false;
    e->wss_pending = false;
    // the observation buffers hold nothing of the restored state: populations,
    // moments and fluxes are available again after the next step
    e->pop_step = -1;
    e->mom_step[0] = e->mom_step[1] = -1;
    // a restored state is not an initialisation: setters must not redo it
    e->fresh = false;
    return 0;
}

int lbm_get_populations(lbm_engine* e, double* f) {
    if (!e || !f) return LBM_ERR_ARGUMENT;
    if (e->pop_step != e->step) return e->fail(LBM_ERR_STATE, "populations of the last step were not observed");
    cudaSetDevice(e->device);
    if (int rc = ensure_staging(e)) return rc;
    cudaError_t ce = launch_pop_to_caller(e->obs_pop, e->perm, e->t.n, e->Q, e->t.ld, e->staging, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "reorder");
    ce = cudaMemcpyAsync(f, e->staging, sizeof(double) * e->t.n * e->Q, cudaMemcpyDeviceToHost, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "download");
    return sync(e);
}

int lbm_set_populations(lbm_engine* e, const double* f) {
    if (!e || !f) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    if (int rc = ensure_staging(e)) return rc;
    // a new state: the device flags and the numeric-fault state start afresh
    if (int rc = sync(e)) return rc;
    e->flag_copy_pending = false;
    e->numeric_fault = false;
    cudaError_t cm = cudaMemsetAsync(e->flags, 0, sizeof(unsigned), e->stream);
    if (cm != cudaSuccess) return e->cuda_fail(cm, "flags");
    cudaError_t ce = cudaMemcpyAsync(e->staging, f, sizeof(double) * e->t.n * e->Q, cudaMemcpyHostToDevice, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "upload");
    ce = launch_pop_from_caller(e->staging, e->perm, e->t.n, e->Q, e->t.ld, e->obs_pop, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "reorder");
    if (int rc = init_from_obs(e)) return rc;
    return sync(e);
}

int lbm_get_macros(lbm_engine* e, double* rho, double* u) {
    if (!e) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    if (int rc = ensure_staging(e)) return rc;
    const int n = e->t.n;
    double* r = e->staging;
    double* uu = e->staging + n;
    // the moments the last step's collision used (those of the previous
    // step's state); right after initialisation, those of the initial state
    int b = (int)((e->step + 1) % 2);
    if (e->step == 0 || e->mom_step[b] != e->step - 1) {
        b = (int)(e->step % 2);
        if (e->mom_step[b] != e->step || e->pop_step != e->step)
            return e->fail(LBM_ERR_STATE, "moments of the last step were not observed");
    }
    cudaError_t ce = launch_mom_to_caller(e->obs_mom[b], e->perm, n, e->t.ld, r, uu, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "reorder");
    if (rho && (ce = cudaMemcpyAsync(rho, r, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess)
        return e->cuda_fail(ce, "download");
    if (u && (ce = cudaMemcpyAsync(u, uu, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess)
        return e->cuda_fail(ce, "download");
    return sync(e);
}

int lbm_get_wss(lbm_engine* e, double* wss, double* acc, double* accmag) {
    if (!e) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    const size_t m = (size_t)e->nw();
    cudaError_t ce = cudaSuccess;
    if (wss && m) ce = cudaMemcpyAsync(wss, e->wss, sizeof(double) * m, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess && acc && m) ce = cudaMemcpyAsync(acc, e->acc, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess && accmag && m)
        ce = cudaMemcpyAsync(accmag, e->accmag, sizeof(double) * m, cudaMemcpyDeviceToHost, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "download");
    return sync(e);
}

int lbm_get_osi_tawss(lbm_engine* e, double* osi, double* tawss) {
    if (!e) return LBM_ERR_ARGUMENT;
    const size_t m = (size_t)e->nw();
    std::vector<double> acc(3 * m), accmag(m);
    if (int rc = lbm_get_wss(e, nullptr, acc.data(), accmag.data())) return rc;
    // Simulation::ComputeOSIAndTAWSS, Simulation.cpp:804-826 (period 0.9)
    const double period = 0.9;
    for (size_t k = 0; k < m; ++k) {
        const double ta = accmag[k] / period;
        const double norm = std::sqrt(std::pow(acc[3 * k], 2) + std::pow(acc[3 * k + 1], 2) + std::pow(acc[3 * k + 2], 2));
        if (osi) osi[k] = 0.5 * (1.0 - (norm / accmag[k]));
        if (tawss) tawss[k] = ta * e->dt;
    }
    return 0;
}

int lbm_get_flux(lbm_engine* e, double* inlet, double* outlets) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (e->pop_step != e->step) return e->fail(LBM_ERR_STATE, "populations of the last step were not observed");
    cudaSetDevice(e->device);
    const int n_out = (int)e->t.out_normal.size() / 3;
    cudaError_t ce = launch_flux(e->Q, e->obs_pop, 1, e->t.ld, e->t.n, e->flux_nodes, e->nin(), e->inlet_normal,
                                 e->flux_partials, e->flux_out, e->stream);
    for (int o = 0; o < n_out && ce == cudaSuccess; ++o) {
        const long long b = e->t.out_off[o], n = e->t.out_off[o + 1] - b;
        ce = launch_flux(e->Q, e->obs_pop, 1, e->t.ld, e->t.n, e->flux_nodes + e->nin() + b, n, &e->t.out_normal[3 * o],
                         e->flux_partials, e->flux_out + 1 + o, e->stream);
    }
    if (ce != cudaSuccess) return e->cuda_fail(ce, "flux kernels");
    std::vector<double> h((size_t)n_out + 1);
    ce = cudaMemcpyAsync(h.data(), e->flux_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "download");
    if (int rc = sync(e)) return rc;
    if (inlet) *inlet = h[0];
    if (outlets)
        for (int o = 0; o < n_out; ++o) outlets[o] = h[1 + o];
    return 0;
}

int lbm_get_flags(lbm_engine* e, uint32_t* flags) {
    if (!e || !flags) return LBM_ERR_ARGUMENT;
    cudaSetDevice(e->device);
    unsigned v = 0;
    cudaError_t ce = cudaMemcpyAsync(&v, e->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "download");
    if (int rc = sync(e)) return rc;
    *flags = v;
    return 0;
}

int lbm_adjoint_run(lbm_engine* e, const lbm_adjoint_desc* d, int32_t gradient, lbm_adjoint_result* r) {
    if (!e || !d || !r) return LBM_ERR_ARGUMENT;
    if (e->bc != LBM_BC_PHYSICS) return e->fail(LBM_ERR_STATE, "the adjoint needs physics boundaries");
    if (d->precision != LBM_STORE_F64 && d->precision != LBM_STORE_F32)
        return e->fail(LBM_ERR_ARGUMENT, "adjoint precision must be LBM_STORE_F64 or LBM_STORE_F32");
    if (d->n_steps < 1) return e->fail(LBM_ERR_ARGUMENT, "adjoint needs at least one step");
    if (gradient && d->checkpoint_every < 1) return e->fail(LBM_ERR_ARGUMENT, "checkpoint interval below 1");
    if (d->n_target < 0 || (d->n_target > 0 && !d->target)) return e->fail(LBM_ERR_ARGUMENT, "bad target list");
    const int n_in = e->nin();
    if (d->n_coeffs < 0 || (d->n_coeffs > 0 && (!d->coeffs || (n_in > 0 && !d->basis))))
        return e->fail(LBM_ERR_ARGUMENT, "bad inlet coefficients or basis");
    if (d->objective != LBM_ADJOINT_WSS2 && d->objective != LBM_ADJOINT_OSI)
        return e->fail(LBM_ERR_ARGUMENT, "unknown adjoint objective");
    if (e->pop_step != e->step) return e->fail(LBM_ERR_STATE, "populations of the last step were not observed");
    cudaSetDevice(e->device);
    AdjointSetup s;
    s.objective = d->objective;
    s.Q = e->Q;
    s.fp64 = d->precision == LBM_STORE_F64;
    s.gradient = gradient != 0;
    s.n = e->t.n;
    s.ld = e->t.ld;
    s.meta = e->meta;
    s.seg_base = e->seg_base;
    s.seg_delta = e->seg_delta;
    s.max_block_segs = e->t.max_block_segs;
    s.aux = e->aux;
    for (int c = 0; c < 3; ++c) s.in_normal[c] = e->inlet_normal[c];
    s.n_in = n_in;
    s.out_nrm = e->out_nrm;
    s.out_rho = e->out_rho;
    s.n_nw = e->nw();
    s.nw_node = e->nw_node;
    s.nw_normal = e->nw_normal;
    s.wss_c = e->wss_c;
    s.tau = e->tau;
    s.f0 = e->obs_pop;
    s.n_steps = d->n_steps;
    s.checkpoint_every = d->checkpoint_every;
    s.stream = e->stream;
    // waveform factor of each step, as the engine's own steps from here would use it
    const bool pulsatile = e->flow == LBM_FLOW_PULSATILE;
    s.factors.resize((size_t)d->n_steps);
    for (int64_t i = 0; i < d->n_steps; ++i)
        s.factors[(size_t)i] = inlet_factor(e, e->step + i, pulsatile ? e->runtime + (double)i * e->dt : e->runtime);
    s.speed.assign(n_in, 0.0);
    for (int j = 0; j < d->n_coeffs; ++j)
        for (int i = 0; i < n_in; ++i) s.speed[i] += d->coeffs[j] * d->basis[(size_t)j * n_in + i];
    s.targets.resize(d->n_target);
    for (int k = 0; k < d->n_target; ++k) {
        if (d->target[k] < 0 || d->target[k] >= e->nw()) return e->fail(LBM_ERR_ARGUMENT, "target outside the near-wall list");
        s.targets[k] = (int)d->target[k];
    }
    double* fin = nullptr;
    if (r->final_populations) {
        cudaError_t ce = cudaMalloc(&fin, sizeof(double) * (size_t)e->Q * e->t.ld);
        if (ce != cudaSuccess) return e->cuda_fail(ce, "adjoint output buffer");
        s.final_pop = fin;
    }
    AdjointOut o;
    const int rc = adjoint_run(s, o);
    int status = 0;
    if (rc == -1) status = e->fail(LBM_ERR_ARGUMENT, o.err);
    else if (rc != 0) status = e->fail(LBM_ERR_CUDA, o.err);
    if (!status && fin) {
        status = ensure_staging(e);
        if (!status) {
            cudaError_t ce = launch_pop_to_caller(fin, e->perm, e->t.n, e->Q, e->t.ld, e->staging, e->stream);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(r->final_populations, e->staging, sizeof(double) * e->t.n * e->Q,
                                     cudaMemcpyDeviceToHost, e->stream);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
            if (ce != cudaSuccess) status = e->cuda_fail(ce, "adjoint populations");
        }
    }
    if (fin) cudaFree(fin);
    if (status) return status;
    r->objective = o.J;
    r->dJ_dtau = s.gradient ? -o.dJ_domega / (e->tau * e->tau) : 0.0;
    if (r->grad_coeffs)
        for (int j = 0; j < d->n_coeffs; ++j) {
            double g = 0.0;
            for (int i = 0; i < n_in; ++i) g += d->basis[(size_t)j * n_in + i] * o.dJ_dspeed[i];
            r->grad_coeffs[j] = g;
        }
    if (r->grad_inlet)
        for (int i = 0; i < n_in; ++i) r->grad_inlet[i] = o.dJ_dspeed[i];
    r->forward_ms = o.forward_ms;
    r->reverse_ms = o.reverse_ms;
    r->steps_recomputed = o.steps_recomputed;
    r->device_bytes = (int64_t)o.bytes;
    return 0;
}

int lbm_get_info(lbm_engine* e, int64_t* n_nodes, int64_t* ld, int64_t* n_segments, int64_t* n_nearwall,
                 int64_t* n_outlet_nodes, int64_t* device_bytes) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (n_nodes) *n_nodes = e->t.n;
    if (ld) *ld = e->t.ld;
    if (n_segments) *n_segments = e->t.nseg;
    if (n_nearwall) *n_nearwall = e->nw();
    if (n_outlet_nodes) *n_outlet_nodes = e->nout();
    if (device_bytes) *device_bytes = (int64_t)e->bytes;
    return 0;
}

// ------------------------------------------------------ slab halo lists ---
}  // extern "C"

namespace {

template <class T>
__global__ void halo_pack_kernel(const T* __restrict__ pop, const long long* __restrict__ slots, long long n,
                                 T* __restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = pop[slots[i]];
}

template <class T>
__global__ void halo_unpack_kernel(T* __restrict__ pop, const long long* __restrict__ slots, long long n,
                                   const T* __restrict__ src) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pop[slots[i]] = src[i];
}

size_t storage_bytes(int storage) {
    return storage == LBM_STORE_F64 ? 8 : storage == LBM_STORE_F32 ? 4 : 2;
}

int halo_copy(lbm_engine* e, int32_t id, void* buf, bool pack) {
    if (!e || !buf || id < 0 || id >= 64) return LBM_ERR_ARGUMENT;
    const auto& h = e->halo[id];
    if (h.n < 0) return e->fail(LBM_ERR_STATE, "halo list " + std::to_string(id) + " is not defined");
    if (h.n == 0) return 0;
    cudaSetDevice(e->device);
    const unsigned grid = (unsigned)((h.n + 255) / 256);
    switch (storage_bytes(e->storage)) {
        case 8:
            if (pack) halo_pack_kernel<<<grid, 256, 0, e->stream>>>((const unsigned long long*)e->pop, h.slots, h.n,
                                                                   (unsigned long long*)buf);
            else halo_unpack_kernel<<<grid, 256, 0, e->stream>>>((unsigned long long*)e->pop, h.slots, h.n,
                                                                (const unsigned long long*)buf);
            break;
        case 4:
            if (pack) halo_pack_kernel<<<grid, 256, 0, e->stream>>>((const unsigned*)e->pop, h.slots, h.n,
                                                                   (unsigned*)buf);
            else halo_unpack_kernel<<<grid, 256, 0, e->stream>>>((unsigned*)e->pop, h.slots, h.n,
                                                                (const unsigned*)buf);
            break;
        default:
            if (pack) halo_pack_kernel<<<grid, 256, 0, e->stream>>>((const unsigned short*)e->pop, h.slots, h.n,
                                                                   (unsigned short*)buf);
            else halo_unpack_kernel<<<grid, 256, 0, e->stream>>>((unsigned short*)e->pop, h.slots, h.n,
                                                                (const unsigned short*)buf);
            break;
    }
    const cudaError_t ce = cudaGetLastError();
    return ce == cudaSuccess ? 0 : e->cuda_fail(ce, pack ? "halo pack" : "halo unpack");
}

}  // namespace

extern "C" {

int lbm_halo_define(lbm_engine* e, int32_t id, int64_t n, const int64_t* node, const int32_t* dir) {
    if (!e) return LBM_ERR_ARGUMENT;
    if (id < 0 || id >= 64) return e->fail(LBM_ERR_ARGUMENT, "halo list id out of range (0..63)");
    if (e->halo[id].n >= 0) return e->fail(LBM_ERR_STATE, "halo list " + std::to_string(id) + " is already defined");
    if (n < 0 || (n > 0 && (!node || !dir))) return e->fail(LBM_ERR_ARGUMENT, "bad halo list");
    if (e->bc != LBM_BC_PHYSICS) return e->fail(LBM_ERR_STATE, "slab halo exchange needs physics boundaries");
    std::vector<long long> slots((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        if (node[i] < 0 || node[i] >= e->t.n) return e->fail(LBM_ERR_ARGUMENT, "halo node index out of range");
        if (dir[i] < 0 || dir[i] >= e->Q) return e->fail(LBM_ERR_ARGUMENT, "halo direction out of range");
        slots[(size_t)i] = (long long)dir[i] * e->t.ld + e->t.iperm[(size_t)node[i]];
    }
    cudaSetDevice(e->device);
    long long* d = nullptr;
    const cudaError_t ce = e->upload(&d, slots);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "halo list");
    e->halo[id].n = n;
    e->halo[id].slots = d;
    return 0;
}

int lbm_halo_pack(lbm_engine* e, int32_t id, void* dst) { return halo_copy(e, id, dst, true); }

int lbm_halo_unpack(lbm_engine* e, int32_t id, const void* src) {
    return halo_copy(e, id, const_cast<void*>(src), false);
}

int lbm_get_phase(lbm_engine* e, int32_t* next_phase) {
    if (!e || !next_phase) return LBM_ERR_ARGUMENT;
    *next_phase = e->phase;
    return 0;
}

const char* lbm_last_error(const lbm_engine* e) { return e ? e->err.c_str() : g_create_error.c_str(); }

}  // extern "C"

void lbm::set_global_error(const std::string& msg) { g_create_error = msg; }

namespace lbm {
// Caller-order node coordinates and near-wall list of an engine, for the
// result writers (output.cu).
bool engine_view(const lbm_engine* e, EngineView& v) {
    if (!e) return false;
    v.n = (int64_t)(e->host_coords.size() / 3);
    v.coords = e->host_coords.data();
    v.n_nw = (int64_t)e->host_nearwall.size();
    v.nearwall = e->host_nearwall.data();
    v.Q = e->Q;
    return true;
}
}  // namespace lbm
