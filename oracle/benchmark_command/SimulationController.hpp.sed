# The controller's device switch and the device context it owns (created on
# first use, destroyed with the controller, as the tree is).  Addresses are
# lines of src/cpp/simulation/SimulationController.hpp.
/^#include <n_body_sim_pro\/n_body_sim_pro.h>$/a\
#include <n_body_sim_pro_cuda.h>
/^    bool use_simd_barnes_hut = false;$/a\
\
    /* Evaluate forces on the B200 (n_body_sim_pro_gravity_compute_acceleration_cuda,\
     * or n_body_sim_pro_barnes_hut_compute_acceleration_cuda with barnes_hut_enabled);\
     * the integrator keeps running on the host, as for every force function. */\
    bool use_cuda = false;
/^        nullptr, n_body_sim_pro_barnes_hut_tree_destroy};$/a\
    mutable std::unique_ptr<NBodySimProCudaContext, void (*)(NBodySimProCudaContext*)> cuda_{\
        nullptr, n_body_sim_pro_cuda_context_destroy};
