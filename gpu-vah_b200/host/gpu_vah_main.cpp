// gpu_vah_main.cpp -- the gpu-vah executable (rhic/src/Run.cpp:38-102 and
// CommandLineArguments.cpp:17-107): same flags, same configuration files,
// same printout, the run() plugin on the GPU.
//
//   gpu-vah -c|--config DIR  -o|--output DIR  [-h|--hydro[=ARG]]  [-t|--test[=ARG]]
#include <getopt.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>

#include "vah_plugin.h"

int main(int argc, char **argv) {
    const char *configDirectory = nullptr, *outputDirectory = nullptr;
    bool runHydro = false, runTest = false;
    static const option longopts[] = {{"test", optional_argument, nullptr, 't'},
                                      {"hydro", optional_argument, nullptr, 'h'},
                                      {"output", required_argument, nullptr, 'o'},
                                      {"config", required_argument, nullptr, 'c'},
                                      {nullptr, 0, nullptr, 0}};
    int ch;
    while ((ch = getopt_long(argc, argv, "t::h::o:c:", longopts, nullptr)) != -1) {
        switch (ch) {
        case 't': runTest = true; break;
        case 'h': runHydro = true; break;
        case 'o': outputDirectory = optarg; break;
        case 'c': configDirectory = optarg; break;
        default:
            std::fprintf(stderr, "usage: %s [-c DIR] [-o DIR] [-h] [-t]\n", argv[0]);
            return 64;
        }
    }
    char *rootDirectory = getcwd(nullptr, 0);
    std::printf("configDirectory = %s\n", configDirectory ? configDirectory : "(null)");
    std::printf("outputDirectory = %s\n", outputDirectory ? outputDirectory : "(null)");
    std::printf(runHydro ? "runHydro = True\n" : "runHydro = False\n");
    std::printf(runTest ? "runTest = True\n" : "runTest = False\n");

    LatticeParameters lattice;
    InitialConditionParameters ic;
    HydroParameters hydro;
    vah_load_lattice_parameters(configDirectory, &lattice);
    vah_load_initial_condition_parameters(configDirectory, &ic);
    vah_load_hydro_parameters(configDirectory, &hydro);

    int rc = 0;
    if (runHydro) {
        rc = vah_run_plugin(&lattice, &ic, &hydro, rootDirectory, outputDirectory);
        std::printf("Done hydro.\n");
    }
    std::free(rootDirectory);
    return rc == 0 ? 0 : 1;
}
