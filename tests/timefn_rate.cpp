// Checks host_time_function_rate (coseis_b200/csrc/timefn.h), the time
// derivatives of the source time functions used by the adjoint's delay
// gradient, against central differences of the time functions of
// sord/utilities.f90:223-281 evaluated in double.  Prints the largest error
// relative to the largest |rate| of each pulse.  Built and run by
// tests/test_stencil.py.
#include <cmath>
#include <cstdio>
#include <string>

#include "../coseis_b200/csrc/timefn.h"

static double tf(const std::string& pulse, double t, double tau) {
    const double pi = 3.14159265358979323846;
    double f = 0, a, b;
    if (pulse == "brune") {
        if (0.0 < t) { a = 1.0 / tau; f = std::exp(-a * t) * a * a * t; }
    } else if (pulse == "integral_brune") {
        if (0.0 < t) { a = 1.0 / tau; f = 1.0 - std::exp(-a * t) * (a * t + 1.0); }
    } else if (pulse == "hann") {
        b = pi * tau;
        if (-b < t && t < b) { a = 1.0 / tau; f = 0.5 / pi * a * (1.0 + std::cos(a * t)); }
    } else if (pulse == "integral_hann") {
        b = pi * tau;
        if (-b < t && t < b) { a = 1.0 / tau; f = 0.5 + 0.5 / pi * (a * t + std::sin(a * t)); }
        else if (0.0 < t) f = 1;
    } else if (pulse == "gaussian" || pulse == "integral_ricker1") {
        a = 0.5 / (tau * tau); b = std::sqrt(a / pi); f = std::exp(-a * t * t) * b;
    } else if (pulse == "ricker1" || pulse == "integral_ricker2") {
        a = 0.5 / (tau * tau); b = std::sqrt(a / pi) * 2.0 * a; f = -std::exp(-a * t * t) * b * t;
    } else if (pulse == "ricker2") {
        a = 0.5 / (tau * tau); b = std::sqrt(a / pi) * 4.0 * a; f = std::exp(-a * t * t) * b * (a * t * t - 0.5);
    }
    return f;
}

int main() {
    const char* pulses[] = {"brune", "integral_brune", "hann", "integral_hann", "gaussian", "integral_ricker1",
                            "ricker1", "integral_ricker2", "ricker2"};
    const double tau = 0.07;
    double worst = 0;
    for (const char* p : pulses) {
        double err = 0, big = 0;
        for (int i = 1; i < 400; i++) {
            // avoid the kinks at the ends of the supports (0 and +-pi tau)
            const double t = -0.5 + 1.0 * i / 400.0 + 1.3e-4;
            const double h = 1e-6 * tau;
            const double fd = (tf(p, t + h, tau) - tf(p, t - h, tau)) / (2 * h);
            const double an = sordgpu::host_time_function_rate(p, t, tau);
            err = std::fmax(err, std::fabs(an - fd));
            big = std::fmax(big, std::fabs(an));
        }
        const double rel = err / (big > 0 ? big : 1.0);
        if (rel > worst) worst = rel;
        printf("%s %.3e\n", p, rel);
    }
    printf("worst %.3e\n", worst);
    return 0;
}
