// Time derivatives of SORD's source time functions (sord/utilities.f90:223-281),
// for the adjoint's origin-time gradient.  Plain C++: the library and a CPU
// test (tests/timefn_rate.cpp) both include it.
#pragma once

#include <cmath>
#include <string>

namespace sordgpu {

// d/dt of each time function, in double (zero for const, delta and step).
inline double host_time_function_rate(const std::string& pulse, double t, double tau) {
    const double pi = 3.14159265358979323846;
    double f = 0, a, b;
    if (pulse == "brune") {
        if (0.0 < t) { a = 1.0 / tau; f = std::exp(-a * t) * a * a * (1.0 - a * t); }
    } else if (pulse == "integral_brune") {
        if (0.0 < t) { a = 1.0 / tau; f = std::exp(-a * t) * a * a * t; }
    } else if (pulse == "hann") {
        b = pi * tau;
        if (-b < t && t < b) { a = 1.0 / tau; f = -0.5 / pi * a * a * std::sin(a * t); }
    } else if (pulse == "integral_hann") {
        b = pi * tau;
        if (-b < t && t < b) { a = 1.0 / tau; f = 0.5 / pi * a * (1.0 + std::cos(a * t)); }
    } else if (pulse == "gaussian" || pulse == "integral_ricker1") {
        a = 0.5 / (tau * tau); b = std::sqrt(a / pi); f = -2.0 * a * t * std::exp(-a * t * t) * b;
    } else if (pulse == "ricker1" || pulse == "integral_ricker2") {
        a = 0.5 / (tau * tau); b = std::sqrt(a / pi) * 2.0 * a; f = -std::exp(-a * t * t) * b * (1.0 - 2.0 * a * t * t);
    } else if (pulse == "ricker2") {
        a = 0.5 / (tau * tau); b = std::sqrt(a / pi) * 4.0 * a; f = std::exp(-a * t * t) * b * 2.0 * a * t * (1.5 - a * t * t);
    }
    return f;
}


}  // namespace sordgpu
