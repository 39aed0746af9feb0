# The two new arms of the force selection, ahead of the CPU ones, and the tree
# statistics read from the device context when it computed them.  Addresses are
# lines of src/cpp/simulation/SimulationController.cpp.
/^NBodySimProForceFunction SimulationController::select_force_function(void\*& force_context) const {$/a\
    if (use_cuda) {\
        if (!cuda_) {\
            NBodySimProError error;\
            n_body_sim_pro_error_clear(&error);\
            cuda_.reset(n_body_sim_pro_cuda_context_create(&error));\
            if (!cuda_) {\
                throw std::runtime_error(std::string("SimulationController: failed to create "\
                                                     "CUDA context: ") + error.message);\
            }\
        }\
        n_body_sim_pro_cuda_context_set_theta(cuda_.get(), barnes_hut_theta);\
        force_context = cuda_.get();\
        return barnes_hut_enabled ? n_body_sim_pro_barnes_hut_compute_acceleration_cuda\
                                  : n_body_sim_pro_gravity_compute_acceleration_cuda;\
    }
s/^        if (n_body_sim_pro_barnes_hut_tree_stats(tree_.get(), &stats)) {$/        if (use_cuda ? n_body_sim_pro_cuda_context_stats(cuda_.get(), \&stats)\n                     : n_body_sim_pro_barnes_hut_tree_stats(tree_.get(), \&stats)) {/
# The device-resident step (cuda_resident): the state stays on the device and
# the host copy is refreshed every cuda_download_interval steps; a new preset or
# loaded checkpoint is uploaded at the next step, a checkpoint is written from a
# fresh download.
/^void SimulationController::step() {$/a\
    if (use_cuda && cuda_resident) {\
        step_on_device();\
        return;\
    }
/^    particles_ = std::move(replacement);$/a\
    cuda_on_device_ = false;
/^void SimulationController::save_checkpoint(const char\* path) {$/a\
    sync_from_device();
/^void SimulationController::refresh_energy_diagnostics() {$/i\
void SimulationController::step_on_device() {\
    void* force_context = nullptr;\
    select_force_function(force_context);  /* creates the device context, sets theta */\
    NBodySimProCudaContext* context = cuda_.get();\
    NBodySimProError error;\
    n_body_sim_pro_error_clear(&error);\
    if (!cuda_on_device_) {\
        NBodySimProParticleSystemView view = particles_.view();\
        if (n_body_sim_pro_cuda_upload(context, &view, &error) != N_BODY_SIM_PRO_STATUS_OK) {\
            throw std::runtime_error(std::string("SimulationController: upload failed: ") +\
                                     error.message);\
        }\
        cuda_on_device_ = true;\
        cuda_pending_steps_ = 0;\
    }\
    const auto step_start = std::chrono::steady_clock::now();\
    const NBodySimProStatus status = n_body_sim_pro_cuda_advance(\
        context, &gravity_, integrator, timestep, 1,\
        barnes_hut_enabled ? N_BODY_SIM_PRO_CUDA_ALGORITHM_BARNES_HUT\
                           : N_BODY_SIM_PRO_CUDA_ALGORITHM_ALL_PAIRS,\
        &error);\
    const auto step_end = std::chrono::steady_clock::now();\
    if (status != N_BODY_SIM_PRO_STATUS_OK) {\
        throw std::runtime_error(std::string("SimulationController: device step failed: ") +\
                                 error.message);\
    }\
    last_step_ms_ = std::chrono::duration<double, std::milli>(step_end - step_start).count();\
    NBodySimProBarnesHutStats stats;\
    if (barnes_hut_enabled && n_body_sim_pro_cuda_context_stats(context, &stats) == 0) {\
        last_tree_build_ms_ = stats.build_time_seconds * 1000.0;\
        last_force_evaluation_ms_ = stats.evaluation_time_seconds * 1000.0;\
    } else {\
        last_tree_build_ms_ = 0.0;\
        last_force_evaluation_ms_ = last_step_ms_;\
    }\
    simulation_time += timestep;\
    ++cuda_pending_steps_;\
    if (cuda_pending_steps_ >= (cuda_download_interval > 0 ? cuda_download_interval : 1)) {\
        sync_from_device();\
        refresh_numerical_diagnostics();\
        if (preset_ == N_BODY_SIM_PRO_PRESET_TWO_BODY) {\
            record_trail_positions();\
        }\
    }\
}\
\
void SimulationController::sync_from_device() {\
    if (!cuda_on_device_ || cuda_pending_steps_ == 0) {\
        return;\
    }\
    NBodySimProParticleSystemView view = particles_.view();\
    NBodySimProError error;\
    n_body_sim_pro_error_clear(&error);\
    if (n_body_sim_pro_cuda_download(cuda_.get(), &view, &error) != N_BODY_SIM_PRO_STATUS_OK) {\
        throw std::runtime_error(std::string("SimulationController: download failed: ") +\
                                 error.message);\
    }\
    cuda_pending_steps_ = 0;\
}\

