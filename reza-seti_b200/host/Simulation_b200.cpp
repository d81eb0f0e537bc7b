/*
 * Drop-in replacement of the reference solver's Simulation.cpp: implements the
 * unchanged Simulation.h (Simulation.h:54-90) on the B200 engine through its
 * C ABI (include/lbm_b200.h). Link it instead of the reference's Simulation.cpp;
 * everything else (LBM.cpp main, Geometry, SubDomain, OutputFile) stays as is.
 *
 * Construction flattens SubDomain_ (Involved_Lat_ order, the inlet / outlet /
 * wall lists and the near-wall list with normals) into an lbm_desc and creates
 * the engine (FP64 storage and reference boundaries by default; environment
 * variable LBM_B200_STORAGE = f32 | f16 | bf16 selects another storage type).
 * Iterate() keeps the reference's loop rules (Simulation.cpp:549-616): MaxIter
 * steps for constant flow, total_runtime <= 2.7 for pulsatile flow, outputs
 * every IterToWrite steps or at systole / diastole, one progress line per
 * step. Between outputs it runs the steps in one engine call without
 * materialising state; before each output it copies populations, density,
 * velocity, |u|, WSS, its accumulators and OSI / TAWSS into the Node fields
 * the reference's OutputFile reads.
 *
 * The per-phase members keep their names and call order. The engine fuses a
 * whole step, so Collision() ... ApplyWallBc() only check the order and
 * ComputeWallShearStress(iter), the last phase of a reference step, runs the
 * step with the current InletVelocity_ and refreshes the Node fields. The
 * fields a reference phase would have changed by then hold NaN from that
 * phase on, so that a caller reading them mid-step sees that they are not
 * there instead of the previous step's values: Collision() sets density,
 * velocity, velMag, m_eqdistributions and m_newDistributions; Streaming()
 * m_distributions. ComputeWallShearStress restores all but
 * m_newDistributions (the engine keeps no post-collision copy).
 *
 * LBM_B200_DUMP=<path>: after Iterate(), write the final Node fields in the
 * record format of the reference harness (oracle/refharness/harness.cpp), for
 * end-to-end comparison with the reference.
 */
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "Simulation.h"
#include "lbm_b200.h"

namespace {

struct EngineState {
    lbm_engine* e = nullptr;
    std::vector<std::shared_ptr<Node>> nodes;  // Involved_Lat_ order (engine node order)
    std::vector<std::shared_ptr<Node>> nearwall;
    int phase = 0;  // next expected phase of a caller-driven step (0 = Collision)
};

std::unordered_map<const Simulation*, EngineState>& registry() {
    static std::unordered_map<const Simulation*, EngineState> r;
    return r;
}

void check(int rc, lbm_engine* e, const char* what) {
    if (rc != LBM_OK) {
        std::cerr << "B200 engine: " << what << " failed (" << rc << "): " << lbm_last_error(e) << std::endl;
        throw std::runtime_error(what);
    }
}

// Storage type: LBM_B200_STORAGE if set, else the config's storage key.
int storage_from_env(int configured) {
    const char* s = std::getenv("LBM_B200_STORAGE");
    if (!s) return configured;
    if (!std::strcmp(s, "f64")) return LBM_STORE_F64;
    if (!std::strcmp(s, "f32")) return LBM_STORE_F32;
    if (!std::strcmp(s, "f16")) return LBM_STORE_F16;
    if (!std::strcmp(s, "bf16")) return LBM_STORE_BF16;
    return configured;
}

// The extension keys of config.txt (lbm_config_parse on the file LBM.cpp's
// main read, "config.txt" in the working directory). The drop-in links the
// reference's D3Q19 SubDomain and reproduces its boundary rules, so it
// accepts only lattice D3Q19 and boundary reference; physics mode and D3Q27
// run through the library's own config runner. A file this parser rejects
// (where the reference reads undefined values) leaves the defaults.
lbm_config config_extensions() {
    lbm_config c{};
    c.lattice = LBM_D3Q19;
    c.storage = LBM_STORE_F64;
    c.bc_mode = LBM_BC_REFERENCE;
    c.period = 0.9;
    if (lbm_config_parse("config.txt", &c) != LBM_OK) {
        std::cerr << "B200 engine: config.txt extensions not read: " << lbm_last_error(nullptr) << std::endl;
        c = lbm_config{};
        c.lattice = LBM_D3Q19;
        c.storage = LBM_STORE_F64;
        c.bc_mode = LBM_BC_REFERENCE;
        c.period = 0.9;
        return c;
    }
    if (c.lattice != LBM_D3Q19 || c.bc_mode != LBM_BC_REFERENCE) {
        std::cerr << "B200 engine: the drop-in runs lattice D3Q19 with the reference's boundary rules; "
                     "use the library's config runner for D3Q27 or physics boundaries"
                  << std::endl;
        std::exit(1);
    }
    return c;
}

// Pulsatile pieces from the config's equations: when they describe a whole
// waveform (three equations, the reference's piece bounds; or as many as
// equation_bounds has intervals). The reference parses equations: but its
// waveform is fixed (pulsatile.h:55-69); with its own coefficients both agree.
void set_waveform_from_equations(lbm_engine* e, const SimulationParameters& sp, const lbm_config& c) {
    const size_t n = sp.equations.size();
    if (n == 0) return;
    for (const auto& q : sp.equations)
        if (q.coeffs.empty() || q.coeffs.size() > LBM_PULSE_MAX_COEFFS) return;
    std::vector<double> bounds;
    if (c.n_bounds > 0) {
        if ((size_t)c.n_bounds != n + 1) return;
        bounds.assign(c.equation_bounds, c.equation_bounds + c.n_bounds);
    } else if (n == 3) {
        bounds = {0.0, 0.1, 0.3, 0.9};
    } else {
        return;
    }
    std::vector<int32_t> counts;
    std::vector<double> coeffs;
    for (const auto& q : sp.equations) {
        counts.push_back((int32_t)q.coeffs.size());
        coeffs.insert(coeffs.end(), q.coeffs.begin(), q.coeffs.end());
    }
    lbm_pulse_desc w{};
    w.period = c.period;
    w.n_pieces = (int32_t)n;
    w.bounds = bounds.data();
    w.n_coeffs = counts.data();
    w.coeffs = coeffs.data();
    check(lbm_set_pulsatile(e, &w), e, "lbm_set_pulsatile");
}

int kind_of(const Node& n) {
    if (n.NodeType_ == NodeType::Fluid) return LBM_NODE_FLUID;
    switch (n.BoundaryType_) {
        case BoundaryType::Inlet: return LBM_NODE_INLET;
        case BoundaryType::Outlet: return LBM_NODE_OUTLET;
        default: return LBM_NODE_WALL;
    }
}

// Copies the engine's observed state into the Node fields the reference's
// output code reads (Node.h:53-71).
void pull_state(EngineState& st, const Simulation& sim) {
    const int64_t n = (int64_t)st.nodes.size();
    const int Q = _nLatNodes;
    std::vector<double> f((size_t)n * Q), rho(n), u(3 * (size_t)n);
    check(lbm_get_populations(st.e, f.data()), st.e, "lbm_get_populations");
    check(lbm_get_macros(st.e, rho.data(), u.data()), st.e, "lbm_get_macros");
    for (int64_t i = 0; i < n; ++i) {
        Node& nd = *st.nodes[i];
        for (int q = 0; q < Q; ++q) nd.m_distributions[q] = f[(size_t)i * Q + q];
        nd.density = rho[i];
        for (int c = 0; c < 3; ++c) nd.velocity[c] = u[3 * (size_t)i + c];
        if (nd.BoundaryType_ != BoundaryType::Wall || nd.NodeType_ == NodeType::Fluid)
            nd.velMag = std::sqrt(std::pow(nd.velocity[0], 2) + std::pow(nd.velocity[1], 2) +
                                  std::pow(nd.velocity[2], 2));
        // f_eq of the last collision, from its moments (Simulation.cpp:212-224)
        for (int q = 0; q < Q; ++q) {
            const auto c = sim.SubDomain_.m_velSet->GetDirection(q);
            const double du = nd.velocity[0] * c[0] + nd.velocity[1] * c[1] + nd.velocity[2] * c[2];
            const double usq = nd.velocity[0] * nd.velocity[0] + nd.velocity[1] * nd.velocity[1] +
                               nd.velocity[2] * nd.velocity[2];
            nd.m_eqdistributions[q] =
                sim.SubDomain_.m_velSet->GetWeight(q) * nd.density * (1.0 + 3.0 * du + 4.5 * du * du - 1.5 * usq);
        }
    }
    const size_t m = st.nearwall.size();
    std::vector<double> wss(m), acc(3 * m), accm(m), osi(m), tawss(m);
    check(lbm_get_wss(st.e, wss.data(), acc.data(), accm.data()), st.e, "lbm_get_wss");
    check(lbm_get_osi_tawss(st.e, osi.data(), tawss.data()), st.e, "lbm_get_osi_tawss");
    const bool pulsatile = sim.simParams.FlowType == "Pulsatile";
    for (size_t k = 0; k < m; ++k) {
        Node& nd = *st.nearwall[k];
        nd.wall_shear_stress = wss[k];
        nd.accumulated_shear_stress = {acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]};
        nd.accumulated_shear_stress_magnitude = accm[k];
        if (pulsatile) {
            nd.osi = osi[k];
            nd.tawss = tawss[k];
        }
    }
}

// Runs n steps; with observe, the state after the last step is materialised
// and copied into the Node fields.
void run(EngineState& st, const Simulation& sim, int64_t n, bool observe) {
    check(lbm_set_observation(st.e, observe ? 1 : 0), st.e, "lbm_set_observation");
    check(lbm_step(st.e, n), st.e, "lbm_step");
    if (observe) pull_state(st, sim);
}

void dump_if_requested(EngineState& st, const Simulation& sim);

}  // namespace

Simulation::Simulation(SubDomain& SubDomain, SimulationParameters& simParams) : SubDomain_(SubDomain) {
    MPI_Comm_rank(MPI_COMM_WORLD, &myrank_);
    MPI_Comm_size(MPI_COMM_WORLD, &num_procs_);
    this->simParams = simParams;
    SetRelaxation(simParams.tau);
    pressure_ = simParams.pressure;
    m_dt = simParams.dt;
    m_omega = 1.0 / m_relaxation;
    InitializeShearStressAccumulators();

    EngineState& st = registry()[this];
    st.nodes = SubDomain_.Involved_Lat_;
    std::unordered_map<const Node*, int64_t> index;
    for (size_t i = 0; i < st.nodes.size(); ++i) index[st.nodes[i].get()] = (int64_t)i;
    const int64_t n = (int64_t)st.nodes.size();
    std::vector<int32_t> coords(3 * (size_t)n);
    std::vector<uint8_t> kind(n);
    for (int64_t i = 0; i < n; ++i) {
        coords[3 * i] = st.nodes[i]->x_position;
        coords[3 * i + 1] = st.nodes[i]->y_position;
        coords[3 * i + 2] = st.nodes[i]->z_position;
        kind[i] = (uint8_t)kind_of(*st.nodes[i]);
    }
    auto indices = [&](const std::vector<std::shared_ptr<Node>>& v) {
        std::vector<int64_t> r;
        for (const auto& p : v) r.push_back(index.at(p.get()));
        return r;
    };
    std::vector<int64_t> inlet = indices(SubDomain_.InletBoundaryNode_.first);
    std::vector<int64_t> out_off = {0}, out_nodes;
    std::vector<double> out_normals;
    for (const auto& o : SubDomain_.OutletBoundaryNodes_) {
        for (const auto& p : o.first) out_nodes.push_back(index.at(p.get()));
        out_off.push_back((int64_t)out_nodes.size());
        for (int c = 0; c < 3; ++c) out_normals.push_back(c < (int)o.second.size() ? o.second[c] : 0.0);
    }
    std::vector<int64_t> wall = indices(SubDomain_.WallBoundaryNode_);
    st.nearwall = SubDomain_.nextToTheWall;
    std::vector<int64_t> nearwall = indices(st.nearwall);
    std::vector<double> normals;
    for (const auto& p : st.nearwall)
        for (int c = 0; c < 3; ++c) normals.push_back(p->normal[c]);

    lbm_desc d{};
    d.lattice = _nLatNodes;
    const lbm_config ext = config_extensions();
    d.storage = storage_from_env(ext.storage);
    d.bc_mode = LBM_BC_REFERENCE;
    d.device = 0;
    d.n_nodes = n;
    d.coords = coords.data();
    d.kind = kind.data();
    d.n_inlet = (int64_t)inlet.size();
    d.inlet = inlet.data();
    for (int c = 0; c < 3; ++c)
        d.inlet_normal[c] = c < (int)SubDomain_.InletBoundaryNode_.second.size() ? SubDomain_.InletBoundaryNode_.second[c] : 0.0;
    d.n_outlets = (int32_t)SubDomain_.OutletBoundaryNodes_.size();
    d.outlet_offsets = out_off.data();
    d.outlet_nodes = out_nodes.data();
    d.outlet_normals = out_normals.data();
    d.n_wall = (int64_t)wall.size();
    d.wall = wall.data();
    d.n_nearwall = (int64_t)nearwall.size();
    d.nearwall = nearwall.data();
    d.nearwall_normals = normals.data();
    d.tau = m_relaxation;
    d.dt = m_dt;
    d.spacing = SubDomain_.Geometry_.spacing;
    check(lbm_create(&d, &st.e), nullptr, "lbm_create");
    // the reference runs on through non-finite values (no check in Iterate)
    check(lbm_set_numeric_check(st.e, 0), st.e, "lbm_set_numeric_check");
    if (simParams.FlowType == "Pulsatile") set_waveform_from_equations(st.e, simParams, ext);
    Iterate();
}

Simulation::~Simulation() {
    auto& r = registry();
    auto it = r.find(this);
    if (it != r.end()) {
        if (it->second.e) lbm_destroy(it->second.e);
        r.erase(it);
    }
}

void Simulation::InitializeShearStressAccumulators() {
    for (auto& node : SubDomain_.nextToTheWall) {
        node->accumulated_shear_stress = {0.0, 0.0, 0.0};
        node->accumulated_shear_stress_magnitude = 0.0;
    }
}

// ---- per-phase members: order check; the step runs in ComputeWallShearStress
static void expect_phase(const Simulation* s, int want, int next, const char* name) {
    EngineState& st = registry().at(s);
    if (st.phase != want) {
        std::cerr << "B200 engine: " << name << " called out of the reference step order" << std::endl;
        throw std::logic_error(name);
    }
    st.phase = next;
}

// Fields that the reference's phases change before the step's end: NaN
// until ComputeWallShearStress has run the fused step.
static void invalidate(const Simulation* s, bool collision) {
    const double nan = std::nan("");
    for (const auto& p : registry().at(s).nodes) {
        Node& nd = *p;
        if (collision) {
            nd.density = nan;
            for (int c = 0; c < 3; ++c) nd.velocity[c] = nan;
            nd.velMag = nan;
            for (auto& v : nd.m_eqdistributions) v = nan;
            for (auto& v : nd.m_newDistributions) v = nan;
        } else {
            for (auto& v : nd.m_distributions) v = nan;
        }
    }
}

void Simulation::Collision() {
    expect_phase(this, 0, 1, "Collision");
    invalidate(this, true);
}
void Simulation::Communicate() {}
void Simulation::Streaming() {
    expect_phase(this, 1, 2, "Streaming");
    invalidate(this, false);
}
void Simulation::ApplyZouHeBc() { expect_phase(this, 2, 3, "ApplyZouHeBc"); }
void Simulation::ApplyInBc() {
    std::cerr << "B200 engine: ApplyInBc (never called by the reference loop) is not provided" << std::endl;
    throw std::logic_error("ApplyInBc");
}
void Simulation::ApplyOutletBc() { expect_phase(this, 3, 4, "ApplyOutletBc"); }
void Simulation::ApplyWallBc() { expect_phase(this, 4, 5, "ApplyWallBc"); }

void Simulation::ComputeWallShearStress(int) {
    expect_phase(this, 5, 0, "ComputeWallShearStress");
    EngineState& st = registry().at(this);
    check(lbm_set_flow(st.e, LBM_FLOW_CONSTANT, InletVelocity_), st.e, "lbm_set_flow");
    run(st, *this, 1, true);
}

void Simulation::ComputeOSIAndTAWSS(int) {
    EngineState& st = registry().at(this);
    const size_t m = st.nearwall.size();
    std::vector<double> osi(m), tawss(m);
    check(lbm_get_osi_tawss(st.e, osi.data(), tawss.data()), st.e, "lbm_get_osi_tawss");
    for (size_t k = 0; k < m; ++k) {
        st.nearwall[k]->osi = osi[k];
        st.nearwall[k]->tawss = tawss[k];
    }
}

double Simulation::getInletVelocity(double x, double period) {
    // Simulation.cpp:519-534; the engine evaluates the same waveform itself
    double vel = 0.0;
    const double t = std::fmod(x, period);
    if (t >= 0 && t < (0.1 * period)) vel = Pulsatile_.InletVelequation1(t);
    else if (t >= (0.1 * period) && t < (0.3 * period)) vel = Pulsatile_.InletVelequation2(t);
    else if (t >= (0.3 * period) && t < (0.9 * period)) vel = Pulsatile_.InletVelequation3(t);
    return vel;
}

void Simulation::Iterate() {
    EngineState& st = registry().at(this);
    const bool pulsatile = simParams.FlowType == "Pulsatile";
    const bool constant = simParams.FlowType == "Constant";
    check(lbm_set_flow(st.e, pulsatile ? LBM_FLOW_PULSATILE : LBM_FLOW_CONSTANT, simParams.CteVel), st.e,
          "lbm_set_flow");
    InletVelocity_ = constant ? simParams.CteVel : 0.0;
    auto progress = [&](int64_t a, int64_t b) {
        if (myrank_ == 0)
            for (int64_t it = a; it < b; ++it)
                std::cout << "Iteration " << it << " has been performed successfully" << std::endl;
    };
    if (constant) {
        const int64_t total = simParams.MaxIter;
        const int64_t every = simParams.IterToWrite;
        int64_t done = 0;
        while (done < total) {
            // next output: after the step with index iter > 0, iter % IterToWrite == 0
            int64_t next = total;
            if (every > 0) {
                int64_t cand = (done / every) * every;
                if (cand == 0 || cand < done) cand += every;
                if (cand < total) next = cand + 1;
            }
            const int64_t chunk = next - done;
            const int64_t iter = next - 1;
            const bool output = every > 0 && iter > 0 && iter % every == 0 && next <= total;
            run(st, *this, chunk, output || next == total);
            progress(done, next);
            done = next;
            if (output) {
                std::string name = "Iteration_" + std::to_string(iter);
                WriteOutput((int)iter, name);
                if (myrank_ == 0) std::cout << "Iteration output written: " << name << std::endl;
            }
        }
    } else if (pulsatile) {
        // the reference's clock (Simulation.cpp:541-607), replayed on the host
        // to place the systole / diastole outputs between engine calls
        const double period = 0.9, tol = m_dt / 2;
        double runtime = 0.0;
        int64_t iter = 0, last = 0;
        int systole = 0, diastole = 0;
        while (runtime <= 2.7) {
            const double cyc = std::fmod(runtime, period);
            std::string name;
            if (std::fabs(cyc - simParams.Systole) < tol) name = "Systole_" + std::to_string(++systole);
            else if (std::fabs(cyc - simParams.Diastole) < tol) name = "Diastole_" + std::to_string(++diastole);
            runtime += m_dt;
            ++iter;
            if (!name.empty()) {
                run(st, *this, iter - last, true);
                progress(last, iter);
                last = iter;
                WriteOutput((int)(iter - 1), name);
                if (myrank_ == 0) std::cout << name.substr(0, name.find('_')) << " output written: " << name << std::endl;
            }
        }
        if (iter > last) {
            run(st, *this, iter - last, true);
            progress(last, iter);
        }
    }
    dump_if_requested(st, *this);
}

void Simulation::SetRelaxation(double tau) { m_relaxation = tau; }

void Simulation::WriteOutput(int iter, const std::string& phase_name) {
    // the reference's output sequence (Simulation.cpp:835-856), unchanged
    const std::string input = std::to_string(iter) + "_FlowHemodynamics.csv";
    const std::string folder = "FlowHemodynamics";
    const std::string output = folder + "/" + phase_name + "_" + std::to_string(iter) + "_FlowHemodynamics.csv";
    if (mkdir(folder.c_str(), 0777) != 0 && errno != EEXIST) {
        perror("Error creating directory");
        return;
    }
    OutputFile file(iter);
    file.WriteVTK_Collective(SubDomain_);
    file.WriteSurfaceAttribute(SubDomain_, iter);
    file.processFlowData(input, output, 0.25, simParams.FlowType);
}

namespace {

// Record writer in the reference harness's format: u32 name length, name,
// u8 dtype, u32 ndim, u64 dims, data.
struct Records {
    std::ofstream out;
    void put(const std::string& name, char dt, std::vector<uint64_t> dims, const void* data, size_t elem) {
        uint32_t n = (uint32_t)name.size(), nd = (uint32_t)dims.size();
        out.write((const char*)&n, 4);
        out.write(name.data(), n);
        out.write(&dt, 1);
        out.write((const char*)&nd, 4);
        uint64_t cnt = 1;
        for (uint64_t d : dims) {
            out.write((const char*)&d, 8);
            cnt *= d;
        }
        out.write((const char*)data, (std::streamsize)(cnt * elem));
    }
};

void dump_if_requested(EngineState& st, const Simulation& sim) {
    const char* path = std::getenv("LBM_B200_DUMP");
    if (!path) return;
    Records r;
    r.out.open(path, std::ios::binary);
    const size_t n = st.nodes.size();
    const int Q = _nLatNodes;
    std::vector<double> f(n * Q), rho(n), u(3 * n), vm(n);
    for (size_t i = 0; i < n; ++i) {
        const Node& nd = *st.nodes[i];
        for (int q = 0; q < Q; ++q) f[i * Q + q] = nd.m_distributions[q];
        rho[i] = nd.density;
        for (int c = 0; c < 3; ++c) u[3 * i + c] = nd.velocity[c];
        vm[i] = nd.velMag;
    }
    r.put("final/f", 'd', {n, (uint64_t)Q}, f.data(), 8);
    r.put("final/rho", 'd', {n}, rho.data(), 8);
    r.put("final/u", 'd', {n, 3}, u.data(), 8);
    r.put("final/velmag", 'd', {n}, vm.data(), 8);
    const size_t m = st.nearwall.size();
    std::vector<double> wss(m), acc(3 * m), accm(m);
    std::vector<int64_t> nw(m);
    std::unordered_map<const Node*, int64_t> index;
    for (size_t i = 0; i < n; ++i) index[st.nodes[i].get()] = (int64_t)i;
    for (size_t k = 0; k < m; ++k) {
        const Node& nd = *st.nearwall[k];
        wss[k] = nd.wall_shear_stress;
        for (int c = 0; c < 3; ++c) acc[3 * k + c] = nd.accumulated_shear_stress[c];
        accm[k] = nd.accumulated_shear_stress_magnitude;
        nw[k] = index.at(st.nearwall[k].get());
    }
    r.put("nearwall", 'q', {m}, nw.data(), 8);
    r.put("final/wss", 'd', {m}, wss.data(), 8);
    r.put("final/acc", 'd', {m, 3}, acc.data(), 8);
    r.put("final/accmag", 'd', {m}, accm.data(), 8);
    (void)sim;
}

}  // namespace
