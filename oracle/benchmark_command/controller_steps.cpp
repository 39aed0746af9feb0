// Test driver for the reference's simulation controller built with the two new
// force algorithms (the sed recipes beside this file): generate a preset the way
// the `benchmark` command does, take STEPS controller steps with the chosen
// algorithm, and write the state as a checkpoint through the controller's own
// save path, so a test can compare it with the CPU oracle.  Test infrastructure
// only; it links the reference engine compiled from its sources and the B200
// library.
//
//   controller_steps PRESET N SEED ALGORITHM THETA SOFTENING TIMESTEP STEPS OUT
//     ALGORITHM: cuda | barnes_hut_cuda | all_pairs | barnes_hut, or
//     cuda_resident | barnes_hut_cuda_resident: the controller's device-resident
//     step, with no download before the checkpoint's own
#include "simulation/SimulationController.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>

int main(int argc, char** argv) {
    if (argc != 10) {
        std::fprintf(stderr,
                     "usage: %s PRESET N SEED ALGORITHM THETA SOFTENING TIMESTEP STEPS OUT\n",
                     argv[0]);
        return 2;
    }
    int preset = -1;
    for (int p = 0; p < N_BODY_SIM_PRO_PRESET_COUNT; ++p)
        if (std::strcmp(argv[1], n_body_sim_pro_preset_string((NBodySimProSimulationPreset)p)) == 0)
            preset = p;
    if (preset < 0) {
        std::fprintf(stderr, "unknown preset %s\n", argv[1]);
        return 2;
    }
    const std::size_t n = (std::size_t)std::strtoull(argv[2], nullptr, 10);
    const std::uint64_t seed = (std::uint64_t)std::strtoull(argv[3], nullptr, 10);
    const char* algorithm = argv[4];
    try {
        n_body_sim_pro::SimulationController sim;
        sim.running = false;
        sim.use_cuda = std::strstr(algorithm, "cuda") != nullptr;
        sim.cuda_resident = std::strstr(algorithm, "_resident") != nullptr;
        sim.barnes_hut_enabled = std::strncmp(algorithm, "barnes_hut", 10) == 0;
        sim.barnes_hut_theta = std::atof(argv[5]);
        sim.set_softening_length(std::atof(argv[6]));
        sim.timestep = std::atof(argv[7]);
        sim.apply_preset((NBodySimProSimulationPreset)preset, n, seed);
        const int steps = std::atoi(argv[8]);
        sim.cuda_download_interval = steps + 1;  // (resident) the checkpoint downloads
        for (int s = 0; s < steps; ++s) sim.step();
        sim.save_checkpoint(argv[9]);
        std::printf("{\"steps\":%d,\"last_step_ms\":%.6f,\"force_evaluation_ms\":%.6f}\n", steps,
                    sim.last_step_ms(), sim.last_force_evaluation_ms());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "controller_steps: %s\n", e.what());
        return 1;
    }
    return 0;
}
