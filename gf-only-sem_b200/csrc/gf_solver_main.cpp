// gf_solver_main.cpp -- gf_solver_elastic_cuda: the process entry of the
// forward solve, over libgfb's C ABI (forward/elastic/src/main.cpp:32-137).
//
//   gf_solver_elastic_cuda --direction {x,y,z} [--resume]
//
// Same flags, messages and exit codes as the reference: no GPU -> exit 1;
// a direction other than x, y, z -> message, usage, exit 1; otherwise the
// exit code of the solve (0 success, 1 failure).  One process runs every
// partition (the reference's single-GPU path); there is no MPI.
#include <cstdint>
#include <cstring>
#include <iostream>
#include <string>

#include "../../include/gfb.h"

static void print_usage(const char* prog) {
    std::cerr << "Usage: " << prog << " --direction {x,y,z} [--resume]\n"
              << "  All I/O paths are frozen relative to CWD:\n"
              << "    Output: wavefields/{direction}/record_{r}_{step}.h5\n"
              << "    Restart: restart/{direction}/restart_{r}.h5\n";
}

int main(int argc, char** argv) {
    int32_t n_devices = 0;
    if (gfb_device_count(&n_devices) != GFB_OK || n_devices == 0) {
        std::cerr << "Error: no CUDA-capable GPU found.\n";
        return 1;
    }
    std::string direction;
    bool resume = false;
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "--direction") == 0 && i + 1 < argc)
            direction = argv[++i];
        else if (std::strcmp(argv[i], "--resume") == 0)
            resume = true;
    }
    if (direction != "x" && direction != "y" && direction != "z") {
        std::cerr << "Error: --direction must be x, y, or z, got '" << direction << "'\n";
        print_usage(argv[0]);
        return 1;
    }
    std::cout << "gf_solver: direction=" << direction;
    if (resume) std::cout << " (resume mode)";
    std::cout << std::endl;
    std::cout << "  input:  config.h5 + partitions/partition_{r}.h5\n"
              << "  output: wavefields/" << direction << "/record_{r}_{step}.h5" << std::endl;
    return gfb_run_forward(direction.c_str(), resume ? 1 : 0, 0);
}
