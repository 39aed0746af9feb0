# The two new algorithms of the reference's force benchmark, `cuda` and
# `barnes_hut_cuda`, added to a build copy of benchmarks/benchmark_force.c
# exactly as a maintainer would add them.  Used by `make -C oracle integrated`;
# the result links the reference engine and libn_body_sim_pro_cuda.so.  Each
# address below is a line of the reference file; every inserted line is new
# code.

# the library's header, after the engine's own headers
/#include "n_body_sim_pro\/threading\/threading.h"/a\
#include "n_body_sim_pro_cuda.h"

# the two names in the usage text
s/barnes_hut_openmp_neon\] \[--theta T\]/barnes_hut_openmp_neon|cuda|barnes_hut_cuda] [--theta T]/

# a CUDA context in place of the tree for the two new algorithms
/^    NBodySimProBarnesHutTree\* tree = NULL;$/a\
    NBodySimProCudaContext* cuda = NULL;\
    if (strcmp(algorithm, "cuda") == 0 || strcmp(algorithm, "barnes_hut_cuda") == 0) {\
        cuda = n_body_sim_pro_cuda_context_create(&error);\
        if (cuda == NULL) {\
            fprintf(stderr, "failed to create CUDA context: %s\\n", error.message);\
            return -1.0;\
        }\
        n_body_sim_pro_cuda_context_set_theta(cuda, theta);\
    }

# two more arms of the strcmp chain, before its last arm
/^        } else if (strcmp(algorithm, "barnes_hut") == 0) {$/i\
        } else if (strcmp(algorithm, "cuda") == 0) {\
            status = n_body_sim_pro_gravity_compute_acceleration_cuda(view, gravity, cuda, &error);\
        } else if (strcmp(algorithm, "barnes_hut_cuda") == 0) {\
            status = n_body_sim_pro_barnes_hut_compute_acceleration_cuda(view, gravity, cuda, &error);

# the context is released wherever the tree is
/n_body_sim_pro_barnes_hut_tree_destroy(tree);/a\
    n_body_sim_pro_cuda_context_destroy(cuda);
