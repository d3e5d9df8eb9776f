// Flow past a cylinder in a channel with TRT collision (magic parameter 1/4),
// a parabolic Zou-He velocity inlet, a Zou-He pressure outlet (rho = 1) and a
// FlowAnalyzer computing lift and drag every 10 steps -- through LLALBM's own
// Lattice API; LLB_POLICY switches between SerialPolicy and CUDAPolicy.
//
//   cylinder_flow <lattice-file> <steps> <tau-even> <u-max> <out-dir>
//
// Writes populations.f64, u.f64, rho.f64 and lift_drag.f64 to out-dir (run it
// from out-dir: the FlowAnalyzer writes ./flow_analysis).
#include <llalbm.hpp>
#include <llalbm_cuda/CUDAPolicy.hpp>

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
    using namespace llalbm::analysis;
    if (argc < 6) {
        std::fprintf(stderr, "usage: %s lattice-file steps tau-even u-max out-dir\n", argv[0]);
        return 2;
    }
    using Configuration =
        LatticeConfiguration<2, collisions::TRTCollisionPolicy<2>, boundaries::BounceBackPolicy<2>,
                             boundaries::BounceBackPolicy<2>, boundaries::ZouHePolicy<2>,
                             boundaries::ZouHePressurePolicy<2>, initializers::VelocityInitializer<2>,
                             equilibrium::DefaultEquilibrium<2>>;
    using Parallelization = LLB_POLICY<2, Configuration>;  // SerialPolicy<2, Configuration> on the CPU

    Lattice<Parallelization> lattice(argv[1], 9, std::cout);
    const long rows = lattice.get_lattice_dimensions()[0];
    const double umax = std::stod(argv[4]);
    collisions::TRTCollisionPolicy<2>::initialize(std::stod(argv[3]), 1.0, 1.0 / std::sqrt(3.0));
    collisions::TRTCollisionPolicy<2>::enforce_magic_parameter(0.25);
    boundaries::ZouHePressurePolicy<2>::initialize(1.0);
    boundaries::ZouHePressurePolicy<2>::reset();
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> inlet = {
        [umax, rows](double, BoundaryPoint<2> p) {
            const double H = static_cast<double>(rows - 2);
            const double yy = static_cast<double>(p.coords[0] - 1) + 0.5;
            return 4.0 * umax * yy * (H - yy) / (H * H);
        },
        [](double, BoundaryPoint<2>) { return 0.0; }};
    std::array<std::function<double(double, BoundaryPoint<2>)>, 2> outlet = {
        boundaries::ZouHePressurePolicy<2>::velocity_function(0),
        boundaries::ZouHePressurePolicy<2>::velocity_function(1)};
    initializers::VelocityInitializer<2>::attach_update_functions(inlet, outlet);

    auto analyzer = std::make_shared<FlowAnalyzer<2>>(lattice.get_obstacle_nodes(), 10, false);
    lattice.attach_flow_analyzer(analyzer);
    lattice.perform_lbm(static_cast<double>(std::stol(argv[2])), 1, 1, false);

    const std::string out = argv[5];
    auto& pop = lattice.get_populations();
    dump_raw(out + "/populations.f64", pop.data(), static_cast<size_t>(pop.size()));
    dump_raw(out + "/u.f64", lattice.get_global_u().data(), static_cast<size_t>(lattice.get_global_u().size()));
    dump_raw(out + "/rho.f64", lattice.get_global_rho().data(), static_cast<size_t>(lattice.get_global_rho().size()));
    std::vector<double> ld;
    for (const auto& p : analyzer->get_all_results()) { ld.push_back(p.first); ld.push_back(p.second); }
    dump_raw(out + "/lift_drag.f64", ld.data(), ld.size());
    return 0;
}
