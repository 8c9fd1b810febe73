// mpm_run.cpp -- headless driver: the reference's demo loop without the GUI.
//
//   mpm-run <config.yaml> [--steps N] [--apic] [--out positions.f32]
//           [--density density.f32] [--vdb density.vdb] [--cfl C]
//           [--integration explicit|semi-implicit|implicit] [--max-iter N] [--tol T]
//
// parseYAML -> build{,APIC}MPMSolver3DFromYAML -> simulateOneStep() N times
// (src/demo/mpm-pic-flip/main.cu:47-215 with the GL/ImGui parts replaced by
// an optional raw float32 (x, y, z, 1) dump of the final positions, and the
// VDB frame by an OpenVDB file of the final density grid (writeToOpenVDB) or
// a raw float32 density grid, res_z x res_y x res_x), and one JSON line with
// the timing.  --integration
// picks the IntegrationType (include/enums.h:17-21), --cfl a CFL time step.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/chains/mpm_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr,
                     "usage: %s config.yaml [--steps N] [--apic] [--out file] [--density file] [--vdb file] [--cfl C]\n"
                     "       [--integration explicit|semi-implicit|implicit] [--max-iter N] [--tol T]\n",
                     argv[0]);
        return 2;
    }
    std::string cfg_path = argv[1], out, density, vdb;
    int steps = 100, max_iter = 50;
    float cfl = 0.f, tol = 1e-5f;
    bool apic = false;
    chains::IntegrationType integration = chains::IntegrationType::EXPLICIT;
    for (int i = 2; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--steps") && i + 1 < argc) steps = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--apic")) apic = true;
        else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) out = argv[++i];
        else if (!std::strcmp(argv[i], "--density") && i + 1 < argc) density = argv[++i];
        else if (!std::strcmp(argv[i], "--vdb") && i + 1 < argc) vdb = argv[++i];
        else if (!std::strcmp(argv[i], "--cfl") && i + 1 < argc) cfl = (float)std::atof(argv[++i]);
        else if (!std::strcmp(argv[i], "--max-iter") && i + 1 < argc) max_iter = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--tol") && i + 1 < argc) tol = (float)std::atof(argv[++i]);
        else if (!std::strcmp(argv[i], "--integration") && i + 1 < argc) {
            const char* v = argv[++i];
            if (!std::strcmp(v, "explicit")) integration = chains::IntegrationType::EXPLICIT;
            else if (!std::strcmp(v, "semi-implicit")) integration = chains::IntegrationType::SEMI_IMPLICIT;
            else if (!std::strcmp(v, "implicit")) integration = chains::IntegrationType::FULL_IMPLICIT;
            else {
                std::fprintf(stderr, "unknown integration %s\n", v);
                return 2;
            }
        } else {
            std::fprintf(stderr, "unknown argument %s\n", argv[i]);
            return 2;
        }
    }
    try {
        chains::MPM3DConfiguration config = chains::parseYAML(cfg_path);
        int n = 0;
        auto write = [](const std::string& path, const std::vector<float>& v) {
            FILE* f = std::fopen(path.c_str(), "wb");
            if (!f) throw std::runtime_error("cannot write " + path);
            const bool ok = std::fwrite(v.data(), sizeof(float), v.size(), f) == v.size();
            if (std::fclose(f) != 0 || !ok) throw std::runtime_error("write failed: " + path);
        };
        auto run = [&](auto& solver) {
            if (integration != chains::IntegrationType::EXPLICIT) solver.setIntegrationType(integration, max_iter, tol);
            if (cfl > 0.f) solver.setCfl(cfl);
            solver.synchronize();
            auto t0 = std::chrono::steady_clock::now();
            for (int s = 0; s < steps; ++s) solver.simulateOneStep();
            solver.synchronize();
            double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (!out.empty()) write(out, solver.positions4());
            if (!density.empty()) write(density, solver.density());
            if (!vdb.empty()) solver.writeToOpenVDB(vdb);
            std::printf(
                "{\"particles\": %d, \"steps\": %d, \"seconds\": %.6f, \"particle_steps_per_s\": %.6e, "
                "\"simulated_time\": %.9g}\n",
                n, steps, sec, sec > 0 ? (double)n * steps / sec : 0.0, solver.simulatedTime());
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
