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
