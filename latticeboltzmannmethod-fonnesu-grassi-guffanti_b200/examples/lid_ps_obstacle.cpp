// Lid-driven cavity with a partially saturated obstacle (PSBounceBackPolicy on
// the obstacle, plain bounce-back on the walls) and TRT collision (magic
// parameter 1/4), set up as LLALBM's own test/unit/LidWithPSObstacle.cpp does
// -- through LLALBM's Lattice API; LLB_POLICY switches between SerialPolicy
// and CUDAPolicy.
//
//   lid_ps_obstacle <lattice-file> <steps> <tau-even> <ps-tau> <out-dir>
//
// Writes populations.f64, u.f64 and rho.f64 to out-dir.
#include <llalbm.hpp>
#include <llalbm_cuda/CUDAPolicy.hpp>

#include <cmath>
#include <cstdio>
#include <string>

#ifndef LLB_POLICY
#define LLB_POLICY CUDAPolicy
#endif

template <typename T>
static void dump_raw(const std::string& path, const T* data, size_t n) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return;
    std::fwrite(data, sizeof(T), n, f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    using namespace llalbm::core;
    if (argc < 6) {
        std::fprintf(stderr, "usage: %s lattice-file steps tau-even ps-tau out-dir\n", argv[0]);
        return 2;
    }
    using Configuration =
        LatticeConfiguration<2, collisions::TRTCollisionPolicy<2>, boundaries::BounceBackPolicy<2>,
                             boundaries::PSBounceBackPolicy<2>, boundaries::ZouHePolicy<2>,
                             boundaries::ZouHePolicy<2>, initializers::VelocityInitializer<2>,
                             equilibrium::DefaultEquilibrium<2>>;
    using Parallelization = LLB_POLICY<2, Configuration>;  // SerialPolicy<2, Configuration> on the CPU

    Lattice<Parallelization> lattice(argv[1], 9, std::cout);
    collisions::TRTCollisionPolicy<2>::initialize(std::stod(argv[3]), 1.0, 1.0 / std::sqrt(3.0));
    collisions::TRTCollisionPolicy<2>::enforce_magic_parameter(0.25);
    boundaries::PSBounceBackPolicy<2>::initialize(std::stod(argv[4]), 0.01);
    lattice.compute_obstacle_weight();
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> lid = {
        [](double t, BoundaryPoint<2>) { return 0.1 * (1.0 - std::exp(-0.002 * t)); },
        [](double, BoundaryPoint<2>) { return 0.0; }};
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> none = {
        [](double, BoundaryPoint<2>) { return 0.0; }, [](double, BoundaryPoint<2>) { return 0.0; }};
    initializers::VelocityInitializer<2>::attach_update_functions(lid, none);

    lattice.perform_lbm(static_cast<double>(std::stol(argv[2])), 1, 1, false);

    const std::string out = argv[5];
    const auto& pop = lattice.get_populations();
    dump_raw(out + "/populations.f64", pop.data(), static_cast<size_t>(pop.size()));
    const auto& u = lattice.get_global_u();
    dump_raw(out + "/u.f64", u.data(), static_cast<size_t>(u.size()));
    const auto& rho = lattice.get_global_rho();
    dump_raw(out + "/rho.f64", rho.data(), static_cast<size_t>(rho.size()));
    return 0;
}
