/*
 * Test-only accessor compiled INTO oracle/_ref/libnbody_ref.so together with the
 * reference engine's own sources.  It reads the private tree fields that the
 * reference keeps behind src/c/barnes_hut/barnes_hut_internal.h:23-48 so the
 * parity tests can compare Morton keys and the sort permutation bit for bit.
 *
 * Nothing here computes anything: it calls the reference's own
 * n_body_sim_pro_barnes_hut_build_tree (src/c/barnes_hut/barnes_hut.c:442-528)
 * and copies out what that function left in the tree.
 */
#include "n_body_sim_pro/barnes_hut/barnes_hut.h"
#include "barnes_hut/barnes_hut_internal.h"

#include <stdint.h>
#include <string.h>

/*
 * Build the reference tree for `view` and copy out:
 *   keys_sorted[i]  = morton key of the particle at sorted position i
 *   permutation[i]  = original index of the particle at sorted position i
 *   root[4]         = root centre x, y, z and root half size
 * Returns the reference status code.  The keys and permutation are copied also
 * when the insertion phase fails with OVERFLOW (duplicate positions): the
 * reference computes them before inserting (barnes_hut.c:487 vs :503-520).
 */
int ref_shim_morton_order(const NBodySimProParticleSystemView* view, uint64_t* keys_sorted,
                          uint64_t* permutation, double* root, size_t* node_count) {
    NBodySimProError error;
    n_body_sim_pro_error_clear(&error);
    NBodySimProBarnesHutTree* tree = n_body_sim_pro_barnes_hut_tree_create(&error);
    if (tree == NULL) {
        return (int)N_BODY_SIM_PRO_STATUS_OUT_OF_MEMORY;
    }
    NBodySimProStatus status = n_body_sim_pro_barnes_hut_build_tree(tree, view, &error);
    if (status == N_BODY_SIM_PRO_STATUS_OK || status == N_BODY_SIM_PRO_STATUS_OVERFLOW) {
        for (size_t i = 0; i < view->particle_count; ++i) {
            const size_t original = tree->permutation[i];
            permutation[i] = (uint64_t)original;
            keys_sorted[i] = tree->morton_keys[original];
        }
        root[0] = tree->root_center_x;
        root[1] = tree->root_center_y;
        root[2] = tree->root_center_z;
        root[3] = tree->root_half_size;
        if (node_count != NULL) {
            *node_count = tree->node_count;
        }
    }
    n_body_sim_pro_barnes_hut_tree_destroy(tree);
    return (int)status;
}
