// Lid-driven cavity (config 1: 129 x 129, BGK tau 0.884, lid u = (0.1, 0)) through
// LLALBM's own Lattice API.  The parallelization policy is the one template
// argument that changes between the CPU run and the GPU run (LLB_POLICY:
// SerialPolicy or CUDAPolicy); everything else is the reference's usage.
//
//   lid_driven_cavity <lattice-file> <steps> <save-step> <out-dir> [ramp]
//
// With `ramp` the lid accelerates as in examples/1_LidDrivenCavity.cpp:
// u_x = 0.15 (1 - exp(-0.001 t)).
// Writes populations.f64, u.f64 and rho.f64 (raw Eigen tensor data) to out-dir.
#include <llalbm.hpp>
#include <llalbm_cuda/CUDAPolicy.hpp>

#include <cstdio>
#include <string>

#ifndef LLB_POLICY
#define LLB_POLICY CUDAPolicy
#endif

template <typename T>
static void dump(const std::string& path, const T& tensor) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return;
    std::fwrite(tensor.data(), sizeof(double), static_cast<size_t>(tensor.size()), f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    using namespace llalbm::core;
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s lattice-file steps save-step out-dir\n", argv[0]);
        return 2;
    }
    using Configuration = LatticeConfiguration<2, collisions::BGKCollisionPolicy<2>, boundaries::BounceBackPolicy<2>,
                                               boundaries::BounceBackPolicy<2>, boundaries::ZouHePolicy<2>,
                                               boundaries::ZouHePolicy<2>, initializers::VelocityInitializer<2>,
                                               equilibrium::DefaultEquilibrium<2>>;
    using Parallelization = LLB_POLICY<2, Configuration>;  // SerialPolicy<2, Configuration> on the CPU

    Lattice<Parallelization> lattice(argv[1], 9, std::cout);
    collisions::BGKCollisionPolicy<2>::initialize(0.884);
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> lid = {
        [](double, BoundaryPoint<2>) { return 0.1; }, [](double, BoundaryPoint<2>) { return 0.0; }};
    if (argc > 5 && std::string(argv[5]) == "ramp")
        lid[0] = [](double t, BoundaryPoint<2>) { return 0.15 * (1.0 - std::exp(-t * (0.001))); };
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> none = {
        [](double, BoundaryPoint<2>) { return 0.0; }, [](double, BoundaryPoint<2>) { return 0.0; }};
    initializers::VelocityInitializer<2>::attach_update_functions(lid, none);

    const long steps = std::stol(argv[2]);
    const long save = std::stol(argv[3]);
    lattice.perform_lbm(static_cast<double>(steps), 1, save > 0 ? static_cast<std::size_t>(save) : 1, save > 0);

    const std::string out = argv[4];
    dump(out + "/populations.f64", lattice.get_populations());
    dump(out + "/u.f64", lattice.get_global_u());
    dump(out + "/rho.f64", lattice.get_global_rho());
    return 0;
}
