// Piecewise-polynomial inlet waveform (lbm_pulse_desc) held by an engine.
#pragma once

#include <string>
#include <vector>

#include "lbm_b200.h"

namespace lbm {

struct Pulse {
    double period = 0.9;
    std::vector<double> bounds;  // [pieces + 1], fractions of the period
    std::vector<int> n_coeffs;   // [pieces]
    std::vector<double> coeffs;  // concatenated, highest power first
};

// Validates d and copies it into p; returns an error message or "".
std::string pulse_from_desc(const lbm_pulse_desc& d, Pulse& p);

// Waveform value at time t (Simulation::getInletVelocity with p's pieces).
double pulse_value(const Pulse& p, double t);

// The reference's waveform (pulsatile.h:55-69 pieces, period 0.9).
const Pulse& reference_pulse();

}  // namespace lbm
