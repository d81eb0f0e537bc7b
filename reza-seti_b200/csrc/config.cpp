// config.txt parser and the piecewise-polynomial pulsatile waveform.
//
// lbm_config_parse restates parseInputFile (LBM.h:81-188): the same trimming
// (spaces and tabs only), the same section rule (a line ending in ':'), the
// same key splitting through std::getline and the same number conversion
// (std::stod / std::stoi, which read a numeric prefix, so "1.0 # note" is 1.0),
// so a file reads the same here as in the reference. Cases where the
// reference would read an uninitialised coordinate or index past a short
// vector are reported as errors.
//
// The waveform evaluates Simulation::getInletVelocity (Simulation.cpp:519-534)
// with given pieces. Each term is formed as pulsatile.h:55-69 forms it: the
// coefficient times std::pow(x, k) for k >= 3, x * x for the square (which is
// what the compiler makes of std::pow(x, 2)), x, and the bare constant, summed
// from the highest power down, so the reference's coefficients reproduce its
// waveform exactly.
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "errors.h"
#include "lbm_b200.h"
#include "pulse.h"

namespace lbm {

namespace {

double power(double x, int k) {
    if (k == 0) return 1.0;
    if (k == 1) return x;
    if (k == 2) return x * x;
    return std::pow(x, (double)k);
}

double piece_value(const double* c, int n, double x) {
    const int d = n - 1;
    double v = c[0] * power(x, d);
    for (int k = 1; k < n; ++k) v = v + c[k] * power(x, d - k);
    return v;
}

}  // namespace

std::string pulse_from_desc(const lbm_pulse_desc& d, Pulse& p) {
    if (!(d.period > 0) || !std::isfinite(d.period)) return "waveform period must be positive";
    if (d.n_pieces < 1 || d.n_pieces > LBM_CONFIG_MAX_EQUATIONS) return "waveform needs 1..16 pieces";
    if (!d.bounds || !d.n_coeffs || !d.coeffs) return "waveform arrays are required";
    Pulse q;
    q.period = d.period;
    q.bounds.assign(d.bounds, d.bounds + d.n_pieces + 1);
    for (int k = 0; k < d.n_pieces; ++k)
        if (!(q.bounds[k] <= q.bounds[k + 1])) return "waveform bounds must ascend";
    size_t total = 0;
    for (int k = 0; k < d.n_pieces; ++k) {
        if (d.n_coeffs[k] < 1 || d.n_coeffs[k] > LBM_PULSE_MAX_COEFFS) return "waveform piece needs 1..16 coefficients";
        q.n_coeffs.push_back(d.n_coeffs[k]);
        total += (size_t)d.n_coeffs[k];
    }
    q.coeffs.assign(d.coeffs, d.coeffs + total);
    p = std::move(q);
    return "";
}

double pulse_value(const Pulse& p, double t) {
    const double x = std::fmod(t, p.period);
    const double* c = p.coeffs.data();
    for (size_t k = 0; k + 1 < p.bounds.size(); ++k) {
        if (x >= p.bounds[k] * p.period && x < p.bounds[k + 1] * p.period) return piece_value(c, p.n_coeffs[k], x);
        c += p.n_coeffs[k];
    }
    return 0.0;
}

const Pulse& reference_pulse() {
    static const Pulse p = [] {
        Pulse r;
        r.period = 0.9;
        r.bounds = {0.0, 0.1, 0.3, 0.9};
        r.n_coeffs = {9, 9, 5};
        r.coeffs = {-8.579e+08, 4.059e+08, -7.817e+07, 7.994e+06, -4.835e+05, 1.782e+04, -321.6, 3.215, 0.1423,
                    -4.32e+06, 7.94e+06, -6.298e+06, 2.82e+06, -7.809e+05, 1.37e+05, -1.484e+04, 901.9, -22.87,
                    -5.123, 14.15, -14.21, 5.865, -0.5696};
        return r;
    }();
    return p;
}

}  // namespace lbm

namespace {

// trim of LBM.h: spaces and tabs
std::string trim(const std::string& s) {
    const size_t first = s.find_first_not_of(" \t");
    const size_t last = s.find_last_not_of(" \t");
    return (first == std::string::npos || last == std::string::npos) ? "" : s.substr(first, last - first + 1);
}

// parseRange of LBM.h: the comma-separated numbers between '[' and ']'
std::vector<double> parse_range(const std::string& value) {
    std::vector<double> r;
    const size_t a = value.find('['), b = value.find(']');
    if (a != std::string::npos && b != std::string::npos) {
        std::istringstream in(value.substr(a + 1, b - a - 1));
        std::string number;
        while (std::getline(in, number, ',')) r.push_back(std::stod(trim(number)));
    }
    return r;
}

std::string unquote(std::string v) {
    std::string r;
    for (char c : v)
        if (c != '"') r += c;
    return r;
}

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void copy_string(char* dst, size_t cap, const std::string& s, const char* what) {
    if (s.size() + 1 > cap) throw ParseError(std::string(what) + " is too long");
    std::memcpy(dst, s.c_str(), s.size() + 1);
}

int storage_of(const std::string& v) {
    if (v == "f64") return LBM_STORE_F64;
    if (v == "f32") return LBM_STORE_F32;
    if (v == "f16") return LBM_STORE_F16;
    if (v == "bf16") return LBM_STORE_BF16;
    throw ParseError("storage must be f64, f32, f16 or bf16");
}

void parse(std::ifstream& file, lbm_config& c) {
    int n_in = 0, n_out = 0;
    lbm_opening ins[LBM_CONFIG_MAX_OPENINGS], outs[LBM_CONFIG_MAX_OPENINGS];
    std::vector<double> amps, phases;
    bool have_phases = false;
    std::string line, section;
    while (std::getline(file, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        if (line.back() == ':') {
            section = line.substr(0, line.size() - 1);
            continue;
        }
        if (section == "parameters") {
            std::istringstream iss(line);
            std::string key, value;
            if (!(std::getline(iss, key, ':') && std::getline(iss, value))) continue;
            key = trim(key);
            value = trim(value);
            // the reference's keys (LBM.h:108-131)
            if (key == "time_resolution") c.dt = std::stod(value);
            else if (key == "density") c.rho = std::stod(value);
            else if (key == "kinematic_viscosity") c.nu_blood = std::stod(value);
            else if (key == "relaxation_factor") c.tau = std::stod(value);
            else if (key == "grid_size") c.grid_size = std::stod(value);
            else if (key == "pressure") c.pressure = std::stod(value);
            else if (key == "CteVel") c.cte_vel = std::stod(value);
            else if (key == "reynolds_number") c.reynolds_number = std::stod(value);
            else if (key == "number_of_outlets") c.number_of_outlets = std::stoi(value);
            else if (key == "IterToWrite") c.iter_to_write = std::stoi(value);
            else if (key == "MaxIter") c.max_iter = std::stoi(value);
            else if (key == "Systole") c.systole = std::stod(value);
            else if (key == "Diastole") c.diastole = std::stod(value);
            else if (key == "NumCycle") c.num_cycle = (int32_t)std::stod(value);  // an int field set from stod
            else if (key == "FlowType") copy_string(c.flow_type, sizeof c.flow_type, unquote(value), "FlowType");
            else if (key == "stl_file") copy_string(c.stl_file, sizeof c.stl_file, unquote(value), "stl_file");
            // extensions
            else if (key == "lattice") {
                const std::string v = unquote(value);
                if (v == "D3Q19" || v == "19") c.lattice = LBM_D3Q19;
                else if (v == "D3Q27" || v == "27") c.lattice = LBM_D3Q27;
                else throw ParseError("lattice must be D3Q19 or D3Q27");
            } else if (key == "storage") c.storage = storage_of(unquote(value));
            else if (key == "boundary") {
                const std::string v = unquote(value);
                if (v == "reference") c.bc_mode = LBM_BC_REFERENCE;
                else if (v == "physics") c.bc_mode = LBM_BC_PHYSICS;
                else throw ParseError("boundary must be reference or physics");
            } else if (key == "period") c.period = std::stod(value);
            else if (key == "equation_bounds") {
                const std::vector<double> b = parse_range(value);
                if (b.size() < 2 || b.size() > LBM_CONFIG_MAX_EQUATIONS + 1)
                    throw ParseError("equation_bounds needs 2..17 values");
                c.n_bounds = (int32_t)b.size();
                for (size_t k = 0; k < b.size(); ++k) c.equation_bounds[k] = b[k];
            } else if (key == "outlet_density") c.outlet_density = std::stod(value);
            else if (key == "harmonic_period_steps") c.harmonic_period_steps = std::stod(value);
            else if (key == "harmonic_amplitudes") amps = parse_range(value);
            else if (key == "harmonic_phases") {
                phases = parse_range(value);
                have_phases = true;
            } else if (key == "device") c.device = std::stoi(value);
        } else if (section == "inlets" || section == "outlets") {
            // one block: this line and the following ones up to an empty line
            std::string plane;
            double coordinate = 0.0;
            bool have_coordinate = false;
            std::vector<double> rx, ry, rz, normal;
            do {
                line = trim(line);
                if (line.empty()) continue;
                const size_t pos = line.find(':');
                if (pos == std::string::npos) continue;
                const std::string key = trim(line.substr(0, pos));
                const std::string value = trim(line.substr(pos + 1));
                if (key == "plane") plane = value;
                else if (key == "coordinate") {
                    coordinate = std::stod(value);
                    have_coordinate = true;
                } else if (key == "range_x") rx = parse_range(value);
                else if (key == "range_y") ry = parse_range(value);
                else if (key == "range_z") rz = parse_range(value);
                else if (key == "normal") normal = parse_range(value);
            } while (std::getline(file, line) && !line.empty());
            const bool outlet = section == "outlets";
            const std::string what = outlet ? "outlet " + std::to_string(n_out + 1) : "inlet " + std::to_string(n_in + 1);
            lbm_opening o{};
            o.outlet = outlet ? 1 : 0;
            if (plane == "x") o.axis = 0;
            else if (plane == "y") o.axis = 1;
            else if (plane == "z") o.axis = 2;
            else throw ParseError(what + ": plane must be x, y or z");
            if (!have_coordinate) throw ParseError(what + ": no coordinate");
            o.coordinate = coordinate;
            if (normal.size() < 3) throw ParseError(what + ": normal needs three values");
            for (int a = 0; a < 3; ++a) o.normal[a] = normal[a];
            const std::vector<double>* r[3] = {&rx, &ry, &rz};
            const double inf = std::numeric_limits<double>::infinity();
            for (int a = 0; a < 3; ++a) {
                if (r[a]->empty()) {
                    o.range[a][0] = -inf;
                    o.range[a][1] = inf;
                } else if (r[a]->size() < 2) {
                    throw ParseError(what + ": a range needs two values");
                } else {
                    o.range[a][0] = (*r[a])[0];
                    o.range[a][1] = (*r[a])[1];
                }
            }
            if (n_in + n_out >= LBM_CONFIG_MAX_OPENINGS) throw ParseError("more than 64 inlets and outlets");
            if (outlet) outs[n_out++] = o;
            else ins[n_in++] = o;
        } else if (section == "equations") {
            const size_t pos = line.find(':');
            if (pos == std::string::npos) continue;
            const std::string name = trim(line.substr(0, pos));
            const std::vector<double> co = parse_range(trim(line.substr(pos + 1)));
            if (c.n_equations >= LBM_CONFIG_MAX_EQUATIONS) throw ParseError("more than 16 equations");
            if (co.size() > LBM_PULSE_MAX_COEFFS) throw ParseError("equation " + name + " has more than 16 coefficients");
            lbm_equation& q = c.equations[c.n_equations++];
            copy_string(q.name, sizeof q.name, name, "equation name");
            q.n_coeffs = (int32_t)co.size();
            for (size_t k = 0; k < co.size(); ++k) q.coeffs[k] = co[k];
        }
    }
    c.n_inlets = n_in;
    c.n_outlets = n_out;
    for (int k = 0; k < n_in; ++k) c.openings[k] = ins[k];
    for (int k = 0; k < n_out; ++k) c.openings[n_in + k] = outs[k];
    if (!amps.empty()) {
        if (amps.size() > LBM_CONFIG_MAX_HARMONICS) throw ParseError("more than 16 harmonics");
        if (have_phases && phases.size() != amps.size())
            throw ParseError("harmonic_phases needs as many values as harmonic_amplitudes");
        c.n_harmonics = (int32_t)amps.size();
        for (size_t k = 0; k < amps.size(); ++k) {
            c.harmonic_amplitudes[k] = amps[k];
            c.harmonic_phases[k] = have_phases ? phases[k] : 0.0;
        }
    }
    const std::string ft = c.flow_type;
    c.flow = ft == "Constant" ? LBM_FLOW_CONSTANT : ft == "Pulsatile" ? LBM_FLOW_PULSATILE
             : ft == "Harmonic" ? LBM_FLOW_HARMONIC : -1;
}

}  // namespace

extern "C" {

int lbm_config_parse(const char* path, lbm_config* out) {
    if (!path || !out) {
        lbm::set_global_error("lbm_config_parse: path and out are required");
        return LBM_ERR_ARGUMENT;
    }
    std::ifstream file(path);
    if (!file.is_open()) {
        lbm::set_global_error(std::string("Unable to open input file: ") + path);
        return LBM_ERR_ARGUMENT;
    }
    lbm_config c;
    std::memset(&c, 0, sizeof c);
    c.lattice = LBM_D3Q19;
    c.storage = LBM_STORE_F64;
    c.bc_mode = LBM_BC_REFERENCE;
    c.period = 0.9;
    c.outlet_density = 1.0;
    c.flow = -1;
    try {
        parse(file, c);
    } catch (const ParseError& ex) {
        lbm::set_global_error(std::string("config ") + path + ": " + ex.what());
        return LBM_ERR_ARGUMENT;
    } catch (const std::exception& ex) {
        // std::stod / std::stoi on a value that is not a number
        lbm::set_global_error(std::string("config ") + path + ": bad number (" + ex.what() + ")");
        return LBM_ERR_ARGUMENT;
    }
    *out = c;
    return LBM_OK;
}

int lbm_pulse_eval(const lbm_pulse_desc* w, double t, double* value) {
    if (!value) {
        lbm::set_global_error("lbm_pulse_eval: value is required");
        return LBM_ERR_ARGUMENT;
    }
    if (!w) {
        *value = lbm::pulse_value(lbm::reference_pulse(), t);
        return LBM_OK;
    }
    lbm::Pulse p;
    const std::string err = lbm::pulse_from_desc(*w, p);
    if (!err.empty()) {
        lbm::set_global_error("lbm_pulse_eval: " + err);
        return LBM_ERR_ARGUMENT;
    }
    *value = lbm::pulse_value(p, t);
    return LBM_OK;
}

}  // extern "C"
