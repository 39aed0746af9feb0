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
    bool use_cuda = false;\
    /* With use_cuda: keep the state on the device between steps\
     * (n_body_sim_pro_cuda_upload once, n_body_sim_pro_cuda_advance per step, the\
     * integrator fused with the force pass) and refresh this particle system from\
     * the device every cuda_download_interval steps and before a checkpoint is\
     * saved.  A preset or a loaded checkpoint replaces the device state at the\
     * next step. */\
    bool cuda_resident = false;\
    int cuda_download_interval = 1;
/^        nullptr, n_body_sim_pro_barnes_hut_tree_destroy};$/a\
    mutable std::unique_ptr<NBodySimProCudaContext, void (*)(NBodySimProCudaContext*)> cuda_{\
        nullptr, n_body_sim_pro_cuda_context_destroy};\
    bool cuda_on_device_ = false;  /* the device holds the newest state */\
    int cuda_pending_steps_ = 0;   /* device steps not yet downloaded */
/^    NBodySimProBarnesHutTree\* barnes_hut_tree();$/a\
    void step_on_device();\
    void sync_from_device();
