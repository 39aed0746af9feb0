# run_headless hands the device switch to the controller; the report names the
# two new algorithms.  Addresses are lines of src/cpp/benchmark/HeadlessRunner.cpp.
/^    simulation.barnes_hut_enabled = options.barnes_hut;$/a\
    simulation.use_cuda = options.cuda;
s/options.barnes_hut ? "barnes_hut" : "all-pairs"/options.cuda ? (options.barnes_hut ? "barnes_hut_cuda" : "cuda") : options.barnes_hut ? "barnes_hut" : "all-pairs"/
