// pulse_case.cpp -- a NekWave driver in the manner of the reference's examples
// (examples/3dboxper/3dboxper.cpp): loads a case file, sets a Gaussian pulse
// through the Case's initial-condition hook, and runs preprocess, simulate and
// postprocess.  The reference's CLI cannot set an initial wave (a case file's
// wave_type is ignored, src/config.hpp:145-149), so the tests and timings that
// compare front ends on a nonzero wave use this driver, built three ways:
//   oracle/_ref/pulse-case-ref       the reference's Case on its own CUDA build
//   build/dropin/pulse-case          the reference's Case on libnwb (drop-in)
//   build/dropin/pulse-case-devdiag  the device-diagnostics Case on libnwb
//
//   pulse-case <case.json> <component 0..5> <x0> <y0> <z0> <sigma>
// sets u_c = exp(-|r - r0|^2 / sigma^2), all other components zero.
#include "case.hpp"
#include "comm.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

int main(int argc, char* argv[]) {
    Comm::init(&argc, &argv);
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s <case.json> <component 0..5> <x0> <y0> <z0> <sigma>\n", argv[0]);
        Comm::finalize();
        return 2;
    }
    const int comp = std::atoi(argv[2]);
    const double x0 = std::atof(argv[3]), y0 = std::atof(argv[4]), z0 = std::atof(argv[5]);
    const double sig = std::atof(argv[6]);
    if (comp < 0 || comp > 5 || !(sig > 0.0)) {
        std::fprintf(stderr, "pulse-case: component must be 0..5 and sigma > 0\n");
        Comm::finalize();
        return 2;
    }
    Case c;
    c.loadConfig(argv[1]);
    c.setWaveType("pulse");
    c.setInitialConditionHook([=](double x, double y, double z, double& ex, double& ey, double& ez,
                                  double& hx, double& hy, double& hz) {
        const double v = std::exp(-((x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0)) /
                                  (sig * sig));
        double* f[6] = {&ex, &ey, &ez, &hx, &hy, &hz};
        for (int k = 0; k < 6; ++k) *f[k] = k == comp ? v : 0.0;
    });
    c.preprocess();
    const auto t0 = std::chrono::steady_clock::now();
    c.simulate();
    const auto t1 = std::chrono::steady_clock::now();
    c.postprocess();
    std::printf("[pulse-case] simulate_s %.6f\n", std::chrono::duration<double>(t1 - t0).count());
    Comm::finalize();
    return 0;
}
