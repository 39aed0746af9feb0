# The reference's command-line entry (src/main.cpp) built headless with the two
# new force algorithms.  Every address is a line of the reference file; every
# inserted line is new code.  The interactive application (SDL3/OpenGL/ImGui)
# cannot be built on these machines, so its include and its launch are the only
# lines taken out; every command of the CLI (benchmark, hardware, save, resume,
# distributed) is the reference's own.

# the application header pulls in SDL3: a headless build includes the
# controller it brought in (the `save` command uses it) directly
s/^#include "application\/Application.hpp"$/#include "simulation\/SimulationController.hpp"/

# the two names in the usage text
s/--algorithm A       all_pairs | barnes_hut\\n/--algorithm A       all_pairs | barnes_hut | cuda | barnes_hut_cuda\\n/

# the `benchmark` command's --algorithm: two more arms before the error arm
/^            } else if (std::strcmp(value, "all_pairs") == 0) {$/i\
            } else if (std::strcmp(value, "cuda") == 0) {\
                options.barnes_hut = false;\
                options.cuda = true;\
                barnes_hut_override = true;\
            } else if (std::strcmp(value, "barnes_hut_cuda") == 0) {\
                options.barnes_hut = true;\
                options.cuda = true;\
                barnes_hut_override = true;

# no interactive application in a headless build
/^        n_body_sim_pro::application::Application application;$/c\
        std::fprintf(stderr, "N-Body Sim Pro: this headless build has no interactive application\\n");
s/^        return application.run();$/        return 1;/
