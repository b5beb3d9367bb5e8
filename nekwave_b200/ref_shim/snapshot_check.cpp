// snapshot_check.cpp -- checks nwb_dropin::SnapshotWriter against synchronous
// downloads on the drop-in DgSolver (dg_solver.cpp on libnwb).
//
//   snapshot-check <N> <nel> <steps> <save_every>
//
// A periodic nel^3 box (the reference's Mesh::createBoxMesh), a seeded state,
// central flux, dt = 0.5 dxmin.  Run A saves every save_every steps through the
// writer; each job copies its snapshot and then sleeps 2 ms, so the writer lags the
// time loop and both snapshot buffers are in use.  Run B downloads the state
// synchronously at the same steps (DgSolver::downloadState, what the reference's
// Case::simulate does).  Prints the saves, their steps and times, and the largest
// difference; exits 0 when every saved state, step and time is equal bit for bit.
#include "dg_solver.hpp"
#include "device_diag.hpp"
#include "mesh.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include <utility>
#include <vector>

namespace {

struct Saved {
    int step;
    double time;
    std::vector<double> state;
};

}  // namespace

int main(int argc, char* argv[]) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s <N> <nel> <steps> <save_every>\n", argv[0]);
        return 2;
    }
    const int N = std::atoi(argv[1]), nel = std::atoi(argv[2]);
    const int steps = std::atoi(argv[3]), every = std::atoi(argv[4]);
    if (N < 2 || nel < 1 || steps < 1 || every < 1) {
        std::fprintf(stderr, "snapshot-check: N >= 2, nel, steps, save_every >= 1\n");
        return 2;
    }
    Mesh mesh(N, 1);
    if (!mesh.createBoxMesh(nel, nel, nel, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, true, true, true)) {
        std::fprintf(stderr, "snapshot-check: createBoxMesh failed\n");
        return 1;
    }
    const size_t n = 6 * static_cast<size_t>(mesh.getTotalPoints());
    std::vector<double> u0(n);
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    for (double& v : u0) v = uni(rng);
    const double dt = 0.5 * mesh.computeMinNodeDistance();

    std::vector<Saved> a, b;
    {  // A: background writer
        DgSolver s;
        s.initialize(mesh, 0.0);
        s.uploadState(u0.data(), n);
        nwb_dropin::SnapshotWriter w;
        double t = 0.0;
        for (int step = 1; step <= steps; ++step) {
            s.step(dt, t);
            t += dt;
            if (step % every == 0)
                w.save(s, step, t, [&a, n](int st, double tt, const double* p) {
                    a.push_back(Saved{st, tt, std::vector<double>(p, p + n)});
                    std::this_thread::sleep_for(std::chrono::milliseconds(2));
                });
        }
        w.finish();
        s.finalize();
    }
    {  // B: synchronous downloads
        DgSolver s;
        s.initialize(mesh, 0.0);
        s.uploadState(u0.data(), n);
        double t = 0.0;
        for (int step = 1; step <= steps; ++step) {
            s.step(dt, t);
            t += dt;
            if (step % every == 0) {
                b.push_back(Saved{step, t, std::vector<double>(n)});
                s.downloadState(b.back().state.data(), n);
            }
        }
        s.finalize();
    }
    bool ok = a.size() == b.size() && !a.empty();
    double maxdiff = 0.0;
    for (size_t i = 0; ok && i < a.size(); ++i) {
        ok = a[i].step == b[i].step && std::memcmp(&a[i].time, &b[i].time, sizeof(double)) == 0;
        for (size_t j = 0; j < n; ++j) {
            const double d = std::abs(a[i].state[j] - b[i].state[j]);
            if (d > maxdiff) maxdiff = d;
        }
        ok = ok && std::memcmp(a[i].state.data(), b[i].state.data(), n * sizeof(double)) == 0;
    }
    std::printf("[snapshot-check] saves %zu / %zu steps", a.size(), b.size());
    for (const Saved& x : a) std::printf(" %d", x.step);
    std::printf(" max_abs_diff %.3e %s\n", maxdiff, ok ? "equal" : "DIFFERENT");
    return ok ? 0 : 1;
}
