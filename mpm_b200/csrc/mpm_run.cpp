// mpm_run.cpp -- headless driver: the reference's demo loop without the GUI.
//
//   mpm-run <config.yaml> [--steps N] [--apic] [--out positions.f32]
//
// parseYAML -> build{,APIC}MPMSolver3DFromYAML -> simulateOneStep() N times
// (src/demo/mpm-pic-flip/main.cu:47-215 with the GL/ImGui/VDB parts replaced
// by an optional raw float32 (x, y, z, 1) dump of the final positions), and
// one JSON line with the timing.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/chains/mpm_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s config.yaml [--steps N] [--apic] [--out file]\n", argv[0]);
        return 2;
    }
    std::string cfg_path = argv[1], out;
    int steps = 100;
    bool apic = false;
    for (int i = 2; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--steps") && i + 1 < argc) steps = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--apic")) apic = true;
        else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) out = argv[++i];
        else {
            std::fprintf(stderr, "unknown argument %s\n", argv[i]);
            return 2;
        }
    }
    try {
        chains::MPM3DConfiguration config = chains::parseYAML(cfg_path);
        int n = 0;
        auto run = [&](auto& solver) {
            solver.synchronize();
            auto t0 = std::chrono::steady_clock::now();
            for (int s = 0; s < steps; ++s) solver.simulateOneStep();
            solver.synchronize();
            double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (!out.empty()) {
                std::vector<float> p = solver.positions4();
                FILE* f = std::fopen(out.c_str(), "wb");
                if (!f) throw std::runtime_error("cannot write " + out);
                std::fwrite(p.data(), sizeof(float), p.size(), f);
                std::fclose(f);
            }
            std::printf("{\"particles\": %d, \"steps\": %d, \"seconds\": %.6f, \"particle_steps_per_s\": %.6e}\n", n,
                        steps, sec, sec > 0 ? (double)n * steps / sec : 0.0);
        };
        if (apic) {
            chains::APICMPMSolver3D solver = chains::buildAPICMPMSolver3DFromYAML(config, n);
            run(solver);
        } else {
            chains::MPMSolver3D solver = chains::buildMPMSolver3DFromYAML(config, n);
            run(solver);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[ERROR] %s\n", e.what());
        return 1;
    }
    return 0;
}
