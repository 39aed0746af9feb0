# HeadlessOptions gains the device switch: with `cuda` set, `barnes_hut`
# selects barnes_hut_cuda, otherwise cuda (all-pairs).  Addresses are lines of
# src/cpp/benchmark/HeadlessRunner.hpp; inserted lines are new code.
/^    bool barnes_hut = true;$/a\
    bool cuda = false; /* forces on the B200 through libn_body_sim_pro_cuda */
