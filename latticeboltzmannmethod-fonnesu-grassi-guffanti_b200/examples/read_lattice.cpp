// Reads a lattice file through Lattice<LLB_POLICY>(path) -- the reference's
// reader for SerialPolicy, the O(R*C) one for CUDAPolicy -- and writes the
// lattice's node vectors with print_lattice_structure(out, true).
//
//   read_lattice <lattice-file> <structure-out>
//
// Prints the seconds the constructor took on stderr.  No GPU is used: the
// CUDA lattice creates its device state at its first perform_lbm.
#include <llalbm.hpp>
#include <llalbm_cuda/CUDAPolicy.hpp>

#include <chrono>
#include <cstdio>
#include <fstream>

#ifndef LLB_POLICY
#define LLB_POLICY CUDAPolicy
#endif

int main(int argc, char** argv) {
    using namespace llalbm::core;
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s lattice-file structure-out\n", argv[0]);
        return 2;
    }
    using Configuration = LatticeConfiguration<2, collisions::BGKCollisionPolicy<2>, boundaries::BounceBackPolicy<2>,
                                               boundaries::BounceBackPolicy<2>, boundaries::ZouHePolicy<2>,
                                               boundaries::ZouHePolicy<2>, initializers::VelocityInitializer<2>,
                                               equilibrium::DefaultEquilibrium<2>>;
    std::ofstream log("/dev/null");
    const auto t0 = std::chrono::steady_clock::now();
    Lattice<LLB_POLICY<2, Configuration>> lattice(argv[1], 9, log);
    const auto t1 = std::chrono::steady_clock::now();
    std::ofstream out(argv[2]);
    lattice.print_lattice_structure(out, true);
    std::fprintf(stderr, "read seconds %.6f\n", std::chrono::duration<double>(t1 - t0).count());
    return 0;
}
