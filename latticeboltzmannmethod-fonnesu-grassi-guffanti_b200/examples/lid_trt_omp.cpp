// Lid-driven cavity with the reference's OpenMP policy family (OMPTRT collision,
// OMPBounceBack walls and obstacles, OMPZouHe lid, OMPVelocityInitializer,
// OMPDefaultEquilibrium), as test/unit/OMPTRTLidDrivenTest.cpp configures them,
// on a lattice read from a file.  The parallelization policy is the one template
// argument that changes between the CPU run and the GPU run (LLB_POLICY:
// OMPPolicy or CUDAPolicy; CUDAPolicy accepts the OpenMP policy family).
//
//   lid_trt_omp <lattice-file> <steps> <save-step> <out-dir>
//
// TRT with tau_even 0.6, magic parameter 1/4 (TRTCollision.hpp:387-440); the
// lid accelerates as in examples/1_LidDrivenCavity.cpp: u_x = 0.15 (1 -
// exp(-0.001 t)).  Writes populations.f64, u.f64 and rho.f64 (raw Eigen tensor
// data) to out-dir.
#include <llalbm.hpp>
#include <llalbm_cuda/CUDAPolicy.hpp>

#include <cmath>
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
    using Configuration =
        LatticeConfiguration<2, collisions::OMPTRTCollisionPolicy<2>, boundaries::OMPBounceBackPolicy<2>,
                             boundaries::OMPBounceBackPolicy<2>, boundaries::OMPZouHePolicy<2>,
                             boundaries::OMPZouHePolicy<2>, initializers::OMPVelocityInitializer<2>,
                             equilibrium::OMPDefaultEquilibrium<2>>;
    using Parallelization = LLB_POLICY<2, Configuration>;  // OMPPolicy<2, Configuration> on the CPU

    Lattice<Parallelization> lattice(argv[1], 9, std::cout);
    collisions::OMPTRTCollisionPolicy<2>::initialize(0.6, 0.6, 1. / std::sqrt(3.0));
    collisions::OMPTRTCollisionPolicy<2>::enforce_magic_parameter(1.0 / 4.0);
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> lid = {
        [](double t, BoundaryPoint<2>) { return 0.15 * (1.0 - std::exp(-t * (0.001))); },
        [](double, BoundaryPoint<2>) { return 0.0; }};
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> none = {
        [](double, BoundaryPoint<2>) { return 0.0; }, [](double, BoundaryPoint<2>) { return 0.0; }};
    initializers::OMPVelocityInitializer<2>::attach_update_functions(lid, none);

    const long steps = std::stol(argv[2]);
    const long save = std::stol(argv[3]);
    lattice.perform_lbm(static_cast<double>(steps), 1, save > 0 ? static_cast<std::size_t>(save) : 1, save > 0);

    const std::string out = argv[4];
    dump(out + "/populations.f64", lattice.get_populations());
    dump(out + "/u.f64", lattice.get_global_u());
    dump(out + "/rho.f64", lattice.get_global_rho());
    return 0;
}
