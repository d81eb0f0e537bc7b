/*
 * Reference harness: drives the reference solver's own step methods and dumps
 * its state, so the oracle restatement and the CUDA engine can be pinned to
 * the reference's real output. Test infrastructure only; built by
 * oracle/Makefile into oracle/_ref/ from the reference sources where they lie.
 *
 * Geometry sources
 *   stl <config.txt>                  : the reference's own pipeline,
 *        Geometry(velSet, params) (ComplexGeometry.cpp:48-73) then
 *        SubDomain(Geometry) (Subdomain.cpp:43-62). Paths in the config are
 *        relative to the config's directory.
 *   nodemap <config.txt> <map.bin>    : a voxel class map written by the test
 *        tools. The SubDomain is assembled from it with the reference's own
 *        Create_cart_comm / Connectivity / Initialize /
 *        IdentifyNextToWallLattices / GetFluidHaloLat
 *        (Subdomain.cpp:96,447,578,475,598); node creation follows
 *        CreateNodes' classification order (Subdomain.cpp:364-442) with O(1)
 *        lookups instead of point-list scans, and near-wall normals come from
 *        the map instead of the O(N*T) triangle sum (Subdomain.cpp:499-572).
 *
 * Step loop
 *   Mirrors Simulation::Iterate (Simulation.cpp:549-616) call for call:
 *   Collision, Communicate, Streaming, inlet velocity, ApplyZouHeBc,
 *   ApplyOutletBc, ApplyWallBc, ComputeWallShearStress, and for pulsatile
 *   flow ComputeOSIAndTAWSS and the time advance. Output and per-step prints
 *   are left out. With --iterate the reference's own Iterate() runs instead
 *   (output goes through the no-op OutputFile).
 *
 * Config
 *   config <config.txt>: runs the reference's parseInputFile (LBM.h:81-188)
 *   and prints what it read, one item per line ("key value", doubles with 17
 *   significant digits; "inlet"/"outlet" lines: plane, coordinate, then each
 *   range's values and the normal's, each list prefixed by its length;
 *   "equation" lines: name, count, coefficients). Parse errors print
 *   "error <what>" and exit 3.
 *
 * Usage
 *   refharness stl <config> <steps> <out.bin> [--phases] [--time] [--iterate]
 *   refharness nodemap <config> <map.bin> <steps> <out.bin> [--phases] [--time]
 *   refharness config <config>
 *   <out.bin> may be "-" for no dump (timing runs).
 */
#include <array>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include <unistd.h>

#include "LBM.h"
#include "LatticeModel.h"
#include "Simulation.h"
#include "Subdomain.h"

namespace {

// ---- dump container -------------------------------------------------------
// Records: u32 name_len | name | u8 dtype | u32 ndim | u64 dims[ndim] | data.
// dtype: 'd' float64, 'i' int32, 'q' int64, 'b' uint8.
class Dump {
public:
    explicit Dump(const std::string& path) {
        if (path != "-") out_.open(path, std::ios::binary);
    }
    bool active() const { return out_.is_open(); }

    template <class T>
    void put(const std::string& name, char dtype, const std::vector<uint64_t>& dims,
             const T* data) {
        if (!active()) return;
        uint32_t n = (uint32_t)name.size();
        out_.write((const char*)&n, 4);
        out_.write(name.data(), n);
        out_.write(&dtype, 1);
        uint32_t nd = (uint32_t)dims.size();
        out_.write((const char*)&nd, 4);
        uint64_t count = 1;
        for (uint64_t d : dims) {
            out_.write((const char*)&d, 8);
            count *= d;
        }
        out_.write((const char*)data, (std::streamsize)(count * sizeof(T)));
    }
    void putd(const std::string& name, const std::vector<double>& v,
              std::vector<uint64_t> dims = {}) {
        if (dims.empty()) dims = {v.size()};
        put(name, 'd', dims, v.data());
    }
    void putq(const std::string& name, const std::vector<int64_t>& v) {
        put(name, 'q', {v.size()}, v.data());
    }

private:
    std::ofstream out_;
};

struct Index {
    std::unordered_map<const Node*, int64_t> of;
    std::vector<std::shared_ptr<Node>> nodes;
};

Index build_index(SubDomain& sd) {
    Index ix;
    ix.nodes = sd.Involved_Lat_;
    for (size_t n = 0; n < ix.nodes.size(); ++n) ix.of[ix.nodes[n].get()] = (int64_t)n;
    return ix;
}

std::vector<int64_t> indices_of(const Index& ix, const std::vector<std::shared_ptr<Node>>& v) {
    std::vector<int64_t> r;
    r.reserve(v.size());
    for (const auto& p : v) r.push_back(ix.of.at(p.get()));
    return r;
}

uint8_t kind_of(const Node& n) {
    if (n.NodeType_ == NodeType::Fluid) return 0;
    switch (n.BoundaryType_) {
        case BoundaryType::Inlet: return 1;
        case BoundaryType::Outlet: return 2;
        case BoundaryType::Wall: return 3;
        default: return 9;
    }
}

void dump_topology(Dump& d, SubDomain& sd, const Index& ix, double tau, double dt,
                   const SimulationParameters& sp) {
    const int64_t N = (int64_t)ix.nodes.size();
    std::vector<int32_t> coords(3 * N);
    std::vector<uint8_t> kind(N);
    int64_t fluid_marked_wall = 0;
    for (int64_t n = 0; n < N; ++n) {
        const Node& nd = *ix.nodes[n];
        coords[3 * n + 0] = nd.x_position;
        coords[3 * n + 1] = nd.y_position;
        coords[3 * n + 2] = nd.z_position;
        kind[n] = kind_of(nd);
        if (nd.NodeType_ == NodeType::Fluid && nd.BoundaryType_ == BoundaryType::Wall)
            ++fluid_marked_wall;
    }
    const double spacing = sd.Geometry_.spacing;
    const double C = 1060 * (dt * dt) / (spacing * spacing * 1e-6);
    std::vector<int64_t> meta_i = {N,
                                   (int64_t)_nLatNodes,
                                   (int64_t)sd.my_Nx_,
                                   (int64_t)sd.my_Ny_,
                                   (int64_t)sd.my_Nz_,
                                   (int64_t)sd.OutletBoundaryNodes_.size(),
                                   fluid_marked_wall,
                                   sp.FlowType == "Pulsatile" ? 1 : 0};
    d.putq("meta_i", meta_i);
    double ox = 0, oy = 0, oz = 0;
    if (!sd.Geometry_.pointsBox.empty()) {
        ox = sd.Geometry_.pointsBox[0][0][0].x;
        oy = sd.Geometry_.pointsBox[0][0][0].y;
        oz = sd.Geometry_.pointsBox[0][0][0].z;
    }
    d.putd("meta_d", {tau, dt, spacing, C, sp.CteVel, ox, oy, oz});
    d.put("coords", 'i', {(uint64_t)N, 3}, coords.data());
    d.put("kind", 'b', {(uint64_t)N}, kind.data());
    d.putq("inlet", indices_of(ix, sd.InletBoundaryNode_.first));
    d.putd("inlet_normal", sd.InletBoundaryNode_.second);
    for (size_t k = 0; k < sd.OutletBoundaryNodes_.size(); ++k) {
        d.putq("outlet_" + std::to_string(k), indices_of(ix, sd.OutletBoundaryNodes_[k].first));
        d.putd("outlet_normal_" + std::to_string(k), sd.OutletBoundaryNodes_[k].second);
    }
    d.putq("wall", indices_of(ix, sd.WallBoundaryNode_));
    d.putq("nearwall", indices_of(ix, sd.nextToTheWall));
    std::vector<double> nrm;
    for (const auto& p : sd.nextToTheWall)
        for (int c = 0; c < 3; ++c) nrm.push_back(p->normal[c]);
    d.putd("nearwall_normal", nrm, {sd.nextToTheWall.size(), 3});
}

void dump_state(Dump& d, const std::string& tag, SubDomain& sd, const Index& ix, double inlet_vel) {
    if (!d.active()) return;
    const int64_t N = (int64_t)ix.nodes.size();
    const int Q = _nLatNodes;
    std::vector<double> f(N * Q), fn(N * Q), fe(N * Q), rho(N), u(3 * N), vm(N);
    for (int64_t n = 0; n < N; ++n) {
        const Node& nd = *ix.nodes[n];
        for (int q = 0; q < Q; ++q) {
            f[n * Q + q] = nd.m_distributions[q];
            fn[n * Q + q] = nd.m_newDistributions[q];
            fe[n * Q + q] = nd.m_eqdistributions[q];
        }
        rho[n] = nd.density;
        for (int c = 0; c < 3; ++c) u[3 * n + c] = nd.velocity[c];
        vm[n] = nd.velMag;
    }
    d.putd(tag + "/f", f, {(uint64_t)N, (uint64_t)Q});
    d.putd(tag + "/fnew", fn, {(uint64_t)N, (uint64_t)Q});
    d.putd(tag + "/feq", fe, {(uint64_t)N, (uint64_t)Q});
    d.putd(tag + "/rho", rho);
    d.putd(tag + "/u", u, {(uint64_t)N, 3});
    d.putd(tag + "/velmag", vm);
    std::vector<double> wss, acc, accm, osi, tawss;
    for (const auto& p : sd.nextToTheWall) {
        wss.push_back(p->wall_shear_stress);
        for (int c = 0; c < 3; ++c) acc.push_back(p->accumulated_shear_stress[c]);
        accm.push_back(p->accumulated_shear_stress_magnitude);
        osi.push_back(p->osi);
        tawss.push_back(p->tawss);
    }
    d.putd(tag + "/wss", wss);
    d.putd(tag + "/acc", acc, {sd.nextToTheWall.size(), 3});
    d.putd(tag + "/accmag", accm);
    d.putd(tag + "/osi", osi);
    d.putd(tag + "/tawss", tawss);
    d.putd(tag + "/inletvel", {inlet_vel});
}

// ---- node-map geometry ------------------------------------------------------
// Format (little endian): "NMAP" | i32 nx, ny, nz, n_outlets | f64 spacing |
// f64 origin[3] | f64 inlet_normal[3] | f64 outlet_normal[n_outlets][3] |
// u8 cls[nx*ny*nz] (index (i*ny + j)*nz + k; 0 solid, 1 fluid, 2 inlet,
// 3 wall, 4+k outlet k) | i64 n_normals | n_normals x {i32 x,y,z; i32 pad;
// f64 nx,ny,nz}.
struct NodeMap {
    int nx = 0, ny = 0, nz = 0, n_out = 0;
    double spacing = 1, origin[3] = {0, 0, 0}, inlet_normal[3] = {0, 0, 0};
    std::vector<double> outlet_normals;
    std::vector<uint8_t> cls;
    std::unordered_map<int64_t, std::array<double, 3>> normals;
};

bool read_nodemap(const std::string& path, NodeMap& m) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    char magic[4];
    in.read(magic, 4);
    if (std::memcmp(magic, "NMAP", 4) != 0) return false;
    int32_t hdr[4];
    in.read((char*)hdr, 16);
    m.nx = hdr[0];
    m.ny = hdr[1];
    m.nz = hdr[2];
    m.n_out = hdr[3];
    in.read((char*)&m.spacing, 8);
    in.read((char*)m.origin, 24);
    in.read((char*)m.inlet_normal, 24);
    m.outlet_normals.resize(3 * (size_t)m.n_out);
    in.read((char*)m.outlet_normals.data(), 24 * (std::streamsize)m.n_out);
    m.cls.resize((size_t)m.nx * m.ny * m.nz);
    in.read((char*)m.cls.data(), (std::streamsize)m.cls.size());
    int64_t nn = 0;
    in.read((char*)&nn, 8);
    for (int64_t r = 0; r < nn; ++r) {
        int32_t c[4];
        double v[3];
        in.read((char*)c, 16);
        in.read((char*)v, 24);
        const int64_t key = ((int64_t)c[0] * m.ny + c[1]) * m.nz + c[2];
        m.normals[key] = {v[0], v[1], v[2]};
    }
    return (bool)in;
}

void assemble_from_nodemap(SubDomain& sd, const NodeMap& m, std::shared_ptr<VelocitySet> vs) {
    sd.Geometry_.spacing = m.spacing;
    sd.m_velSet = vs;
    sd.gridSize_ = {m.nx, m.ny, m.nz};
    sd.Create_cart_comm();
    sd.m_lattice.assign(m.nx, std::vector<std::vector<std::shared_ptr<Node>>>(
                                   m.ny, std::vector<std::shared_ptr<Node>>(m.nz, nullptr)));
    sd.OutletBoundaryNodes_.resize(m.n_out);
    for (int i = 0; i < m.nx; ++i)
        for (int j = 0; j < m.ny; ++j)
            for (int k = 0; k < m.nz; ++k) {
                const uint8_t c = m.cls[((size_t)i * m.ny + j) * m.nz + k];
                if (c == 0) continue;
                std::shared_ptr<Node> p;
                if (c == 1) {
                    p = std::make_shared<Node>(i, j, k, NodeType::Fluid);
                    p->BoundaryType_ = BoundaryType::None;
                } else {
                    p = std::make_shared<Boundary>(i, j, k, vs, NodeType::Boundary);
                    if (c == 2) {
                        p->BoundaryType_ = BoundaryType::Inlet;
                        sd.InletBoundaryNode_.first.push_back(p);
                    } else if (c == 3) {
                        p->BoundaryType_ = BoundaryType::Wall;
                        sd.WallBoundaryNode_.push_back(p);
                    } else {
                        p->BoundaryType_ = BoundaryType::Outlet;
                        sd.OutletBoundaryNodes_[c - 4].first.push_back(p);
                    }
                }
                sd.m_lattice[i][j][k] = p;
            }
    sd.InletBoundaryNode_.second = {m.inlet_normal[0], m.inlet_normal[1], m.inlet_normal[2]};
    for (int o = 0; o < m.n_out; ++o)
        sd.OutletBoundaryNodes_[o].second = {m.outlet_normals[3 * o], m.outlet_normals[3 * o + 1],
                                             m.outlet_normals[3 * o + 2]};
    sd.Connectivity();
    sd.Initialize();
    sd.IdentifyNextToWallLattices();
    for (auto& p : sd.nextToTheWall) {
        const int64_t key = ((int64_t)p->x_position * m.ny + p->y_position) * m.nz + p->z_position;
        auto it = m.normals.find(key);
        p->normal = {0.0, 0.0, 0.0};
        if (it != m.normals.end()) p->normal = {it->second[0], it->second[1], it->second[2]};
    }
    sd.GetFluidHaloLat();
}

// ---- step loop -------------------------------------------------------------
struct Clock {
    double total_runtime = 0.0;
    int iter = 0;
};

void run_steps(Simulation& sim, int steps, Dump& d, const Index& ix, bool phases, Clock& clk) {
    const bool pulsatile = sim.simParams.FlowType == "Pulsatile";
    const double period = 0.9;
    for (int s = 0; s < steps; ++s) {
        const bool dump_phases = phases && clk.iter == 0;
        sim.Collision();
        if (dump_phases) dump_state(d, "p1_collide", sim.SubDomain_, ix, 0.0);
        sim.Communicate();
        sim.Streaming();
        if (dump_phases) dump_state(d, "p1_stream", sim.SubDomain_, ix, 0.0);
        if (sim.simParams.FlowType == "Constant")
            sim.InletVelocity_ = sim.simParams.CteVel;
        else if (pulsatile)
            sim.InletVelocity_ = sim.getInletVelocity(clk.total_runtime, period);
        sim.ApplyZouHeBc();
        if (dump_phases) dump_state(d, "p1_inlet", sim.SubDomain_, ix, sim.InletVelocity_);
        sim.ApplyOutletBc();
        if (dump_phases) dump_state(d, "p1_outlet", sim.SubDomain_, ix, sim.InletVelocity_);
        sim.ApplyWallBc();
        if (dump_phases) dump_state(d, "p1_wall", sim.SubDomain_, ix, sim.InletVelocity_);
        sim.ComputeWallShearStress(clk.iter);
        if (pulsatile) sim.ComputeOSIAndTAWSS(clk.iter);
        if (dump_phases) dump_state(d, "p1_wss", sim.SubDomain_, ix, sim.InletVelocity_);
        if (pulsatile) clk.total_runtime += sim.m_dt;
        clk.iter++;
    }
}

int usage() {
    std::fprintf(stderr,
                 "usage: refharness stl <config> <steps> <out.bin> [--phases] [--time] [--iterate]\n"
                 "       refharness nodemap <config> <map.bin> <steps> <out.bin> [--phases] "
                 "[--time]\n"
                 "       refharness config <config>\n");
    return 2;
}

void print_list(const std::vector<double>& v) {
    std::printf(" %zu", v.size());
    for (double x : v) std::printf(" %.17g", x);
}

int print_config(const std::string& path) {
    SimulationParameters sp;
    try {
        parseInputFile(path, sp);
    } catch (const std::exception& ex) {
        std::printf("error %s\n", ex.what());
        return 3;
    }
    std::printf("stl_file %s\n", sp.stlFile.c_str());
    std::printf("FlowType %s\n", sp.FlowType.c_str());
    std::printf("dt %.17g\nrho %.17g\nnu_blood %.17g\ntau %.17g\ngrid_size %.17g\npressure %.17g\n", sp.dt,
                sp.rho, sp.nu_blood, sp.tau, sp.dx, sp.pressure);
    std::printf("CteVel %.17g\nreynolds_number %.17g\nSystole %.17g\nDiastole %.17g\n", sp.CteVel,
                sp.reynoldsNumber, sp.Systole, sp.Diastole);
    std::printf("number_of_outlets %d\nMaxIter %d\nIterToWrite %d\nNumCycle %d\n", sp.num_Out, sp.MaxIter,
                sp.IterToWrite, (int)sp.NumCycle);
    auto opening = [](const char* kind, const std::string& plane, double coordinate, const std::vector<double>& rx,
                      const std::vector<double>& ry, const std::vector<double>& rz, const std::vector<double>& n) {
        std::printf("%s %s %.17g", kind, plane.c_str(), coordinate);
        print_list(rx);
        print_list(ry);
        print_list(rz);
        print_list(n);
        std::printf("\n");
    };
    for (const auto& o : sp.inlets) opening("inlet", o.plane, o.coordinate, o.range_x, o.range_y, o.range_z, o.normal);
    for (const auto& o : sp.outlets) opening("outlet", o.plane, o.coordinate, o.range_x, o.range_y, o.range_z, o.normal);
    for (const auto& q : sp.equations) {
        std::printf("equation %s", q.name.c_str());
        print_list(q.coeffs);
        std::printf("\n");
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc == 3 && std::string(argv[1]) == "config") return print_config(argv[2]);
    if (argc < 5) return usage();
    const std::string mode = argv[1];
    std::string config = argv[2], mappath, out;
    int steps = 0, argi = 0;
    if (mode == "stl") {
        steps = std::atoi(argv[3]);
        out = argv[4];
        argi = 5;
    } else if (mode == "nodemap") {
        if (argc < 6) return usage();
        mappath = argv[3];
        steps = std::atoi(argv[4]);
        out = argv[5];
        argi = 6;
    } else {
        return usage();
    }
    bool phases = false, timing = false, iterate = false;
    for (int a = argi; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--phases")) phases = true;
        else if (!std::strcmp(argv[a], "--time")) timing = true;
        else if (!std::strcmp(argv[a], "--iterate")) iterate = true;
        else return usage();
    }

    // Resolve output/map paths before changing directory to the config's.
    auto absolute = [](const std::string& p) {
        if (p == "-" || p.empty() || p[0] == '/') return p;
        char buf[4096];
        if (!getcwd(buf, sizeof buf)) return p;
        return std::string(buf) + "/" + p;
    };
    out = absolute(out);
    mappath = absolute(mappath);
    config = absolute(config);
    const std::string dir = config.substr(0, config.find_last_of('/'));
    if (chdir(dir.c_str()) != 0) {
        std::perror("chdir");
        return 1;
    }

    int ac = 1;
    MPI_Init(&ac, &argv);
    SimulationParameters sp;
    parseInputFile(config, sp);

    std::shared_ptr<LatticeModel> velSet = std::make_shared<LatticeModel>();
    SubDomain sd;
    const auto t_setup0 = std::chrono::steady_clock::now();
    if (mode == "stl") {
        Geometry geo(velSet, sp);
        sd = SubDomain(geo);
    } else {
        NodeMap m;
        if (!read_nodemap(mappath, m)) {
            std::fprintf(stderr, "cannot read node map %s\n", mappath.c_str());
            return 1;
        }
        assemble_from_nodemap(sd, m, velSet);
    }
    const auto t_setup1 = std::chrono::steady_clock::now();

    Simulation sim;
    sim.myrank_ = 0;
    sim.num_procs_ = 1;
    sim.SubDomain_ = sd;
    sim.simParams = sp;
    sim.SetRelaxation(sp.tau);
    sim.pressure_ = sp.pressure;
    sim.m_dt = sp.dt;
    sim.m_omega = 1.0 / sim.m_relaxation;
    sim.InletVelocity_ = 0.0;
    sim.InitializeShearStressAccumulators();

    Index ix = build_index(sim.SubDomain_);
    Dump d(out);
    dump_topology(d, sim.SubDomain_, ix, sp.tau, sp.dt, sp);
    dump_state(d, "init", sim.SubDomain_, ix, 0.0);

    Clock clk;
    const auto t0 = std::chrono::steady_clock::now();
    if (iterate) {
        sim.Iterate();
        clk.iter = -1;
    } else {
        run_steps(sim, steps, d, ix, phases, clk);
    }
    const auto t1 = std::chrono::steady_clock::now();
    dump_state(d, "final", sim.SubDomain_, ix, sim.InletVelocity_);

    const double secs = std::chrono::duration<double>(t1 - t0).count();
    const double setup = std::chrono::duration<double>(t_setup1 - t_setup0).count();
    if (timing) {
        const double n = (double)ix.nodes.size();
        std::printf("{\"nodes\": %.0f, \"steps\": %d, \"seconds\": %.6f, \"mlups\": %.6f, "
                    "\"setup_seconds\": %.3f}\n",
                    n, steps, secs, steps > 0 ? n * steps / secs / 1e6 : 0.0, setup);
    }
    MPI_Finalize();
    return 0;
}
