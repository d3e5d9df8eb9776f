// ref_runner -- ORACLE TEST INFRASTRUCTURE (never shipped, never timed as the product).
//
// Drives the UNMODIFIED LLALBM headers (compiled from the reference tree against
// the container shim in oracle/eigen_shim) through their own public API:
// Lattice<P> construction (lattice file, ConstructionInfo + build_lattice, or
// Lattice::reinit with node vectors), static policy parameters, update functions,
// perform_lbm, getters and FlowAnalyzer.  It dumps the results as raw binary
// arrays so the tests can pin the C restatement (oracle/lbm_oracle.c) and the
// CUDA path against the reference itself, and it times perform_lbm for the CPU
// baseline.
//
// Build: oracle/Makefile (outputs only into oracle/_ref/).
#include "llalbm.hpp"
#include "llalbm_cuda/ZouHePressurePolicy.hpp"

#include <omp.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>

using namespace llalbm::core;
namespace gen = llalbm::util::generation;

namespace {

struct Options {
    std::string geometry = "file";  // file | raw | construct
    std::string path;
    long rows = 0, cols = 0;
    std::string policy = "serial";  // serial | omp
    std::string collision = "bgk";  // bgk | trt
    double tau = 0.6, tau_even = 0.6, tau_odd = -1.0, magic = -1.0;
    std::string inlet_bc = "zh";    // zh | open
    std::string outlet_bc = "zh";   // zh | open | zhp
    std::string inlet_u = "const:0:0";
    std::string outlet_u = "const:0:0";
    double rho_out = 1.0, tangential_u = 0.0;
    std::string obstacle = "bb";    // bb | ps (PSBounceBackPolicy, serial policies)
    double ps_tau = 0.6;
    std::string ps_b = "default";   // default | pattern (b of obstacle q = ((37 q + 11) mod 101) / 100)
    long steps = 10;
    long warmup = 0;
    long analyzer_every = 0;
    int threads = 0;
    bool timing = false;
    bool dump_nodes = false;
    bool dump_fields = true;
    std::string out = ".";
};

[[noreturn]] void die(const std::string& m) {
    std::fprintf(stderr, "ref_runner: %s\n", m.c_str());
    std::exit(2);
}

std::vector<std::string> split(const std::string& s, char sep) {
    std::vector<std::string> out;
    std::string cur;
    for (char c : s) {
        if (c == sep) { out.push_back(cur); cur.clear(); }
        else cur.push_back(c);
    }
    out.push_back(cur);
    return out;
}

// Update-function specifications shared with the C oracle and the Python tests:
//   const:ux:uy                constant velocity
//   parabolic:umax:i0:i1       u_x = 4 umax yy (H - yy) / H^2, yy = (i - i0) + 0.5, H = i1 - i0 + 1
//   lidramp:a:b                u_x = a (1 - exp(-t b))   (examples/1_LidDrivenCavity.cpp:80)
//   pressure                   velocity cached by the Zou-He pressure policy
using UpdateFn = std::function<double(double, BoundaryPoint<2>)>;

std::array<UpdateFn, 2> make_functions(const std::string& spec) {
    const auto f = split(spec, ':');
    std::array<UpdateFn, 2> fn;
    if (f[0] == "const" && f.size() == 3) {
        const double ux = std::stod(f[1]), uy = std::stod(f[2]);
        fn[0] = [ux](double, BoundaryPoint<2>) { return ux; };
        fn[1] = [uy](double, BoundaryPoint<2>) { return uy; };
    } else if (f[0] == "parabolic" && f.size() == 4) {
        const double umax = std::stod(f[1]);
        const long i0 = std::stol(f[2]), i1 = std::stol(f[3]);
        fn[0] = [umax, i0, i1](double, BoundaryPoint<2> p) {
            const double H = static_cast<double>(i1 - i0 + 1);
            const double yy = static_cast<double>(p.coords[0] - i0) + 0.5;
            return 4.0 * umax * yy * (H - yy) / (H * H);
        };
        fn[1] = [](double, BoundaryPoint<2>) { return 0.0; };
    } else if (f[0] == "lidramp" && f.size() == 3) {
        const double a = std::stod(f[1]), b = std::stod(f[2]);
        fn[0] = [a, b](double t, BoundaryPoint<2>) { return a * (1.0 - std::exp(-t * b)); };
        fn[1] = [](double, BoundaryPoint<2>) { return 0.0; };
    } else if (f[0] == "pressure") {
        fn[0] = boundaries::ZouHePressurePolicy<2>::velocity_function(0);
        fn[1] = boundaries::ZouHePressurePolicy<2>::velocity_function(1);
    } else {
        die("bad update-function spec '" + spec + "'");
    }
    return fn;
}

template <typename T>
void write_raw(const std::string& path, const T* data, std::size_t n) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) die("cannot write " + path);
    if (n && std::fwrite(data, sizeof(T), n, f) != n) die("short write " + path);
    std::fclose(f);
}

// O(N) construction of the reference's node vectors from a grid of
// InputNodeType codes, for lattices too large for the reference's own O(N^2)
// classification (ConstructionTools.hpp:142-179, NodeIdentification.hpp:137-211).
// Vector order, side identification and wet filtering are the reference's:
// row-major (i, j) order as in TensorLoopAccessor (LatticeReader.hpp:108-204),
// identify_node_type and eliminate_non_wet_nodes are called directly, and the
// obstacle direction bits use the reference's rule (bit k set iff the node at
// coords + c_k is fluid, inlet or outlet), looked up in the grid instead of
// by std::find over the vectors.
template <typename LatticeT>
void build_from_raw(LatticeT& lattice, const Options& o) {
    const long R = o.rows, C = o.cols;
    std::vector<unsigned char> types(static_cast<std::size_t>(R * C));
    {
        std::FILE* f = std::fopen(o.path.c_str(), "rb");
        if (!f) die("cannot open " + o.path);
        if (std::fread(types.data(), 1, types.size(), f) != types.size()) die("short raw grid");
        std::fclose(f);
    }
    auto at = [&](long i, long j) { return types[static_cast<std::size_t>(i + R * j)]; };  // column-major
    std::vector<Point<2>> fluid;
    std::vector<BoundaryPoint<2>> boundary, inlet, outlet;
    std::vector<ObstaclePoint<2>> obstacle;
    for (long i = 0; i < R; ++i) {
        for (long j = 0; j < C; ++j) {
            const unsigned t = at(i, j);
            BoundaryPoint<2> bp({i, j});
            switch (t) {
            case InputNodeType::FLUID: fluid.push_back(Point<2>({i, j})); break;
            case InputNodeType::BOUNDARY: boundary.push_back(bp); break;
            case InputNodeType::INLET: inlet.push_back(bp); break;
            case InputNodeType::OUTLET: outlet.push_back(bp); break;
            case InputNodeType::OBSTACLE: obstacle.push_back(ObstaclePoint<2>({i, j})); break;
            default: break;
            }
        }
    }
    const std::array<Eigen::Index, 2> dims = {R, C};
    llalbm::util::identify_node_type(dims, inlet);
    llalbm::util::identify_node_type(dims, outlet);
    static const int di[9] = {0, 0, -1, 0, 1, -1, -1, 1, 1};
    static const int dj[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    for (auto& node : obstacle) {
        node.directions.reset();
        for (int k = 1; k < 9; ++k) {
            const long ni = node.coords[0] + di[k], nj = node.coords[1] + dj[k];
            if (ni < 0 || nj < 0 || ni >= R || nj >= C) continue;
            const unsigned t = at(ni, nj);
            if (t == InputNodeType::FLUID || t == InputNodeType::INLET || t == InputNodeType::OUTLET)
                node.directions.set(static_cast<std::size_t>(k), true);
        }
    }
    llalbm::util::eliminate_non_wet_nodes(obstacle);
    lattice.reinit(9, dims, fluid, boundary, inlet, outlet, obstacle);
}

// ConstructionInfo script: one call per line.
//   dims R C | perimeter TYPE | interval i0 j0 i1 j1 TYPE | rect i j ei ej |
//   square i j e | sphere i j r | random n maxr minr seed
// The adders are the reference's own (ConstructionInfo.hpp:147-486).
// build_lattice (ConstructionTools.hpp:54-201) cannot be called here: its node
// count at :123 is std::accumulate over begin() and end() of two different
// temporaries returned by get_domain_dimensions(), undefined behaviour that
// never terminates in this build.  Its remaining steps are repeated with the
// reference's own functions: set -> vector copies in set order (:94-118), the
// fluid list = all grid points minus every listed node, in sorted (i, j) order
// (:120-179), identify_node_type, identify_obstacle_propagation,
// eliminate_non_wet_nodes (:182-187) and Lattice::reinit (:192-200).
// The script's node sets are also dumped as an InputNodeType grid (types.u8).
template <typename LatticeT>
void build_from_script(LatticeT& lattice, const Options& o) {
    gen::ConstructionInfo<2> info;
    std::ifstream in(o.path);
    if (!in) die("cannot open " + o.path);
    auto type_of = [](const std::string& s) {
        if (s == "BOUNDARY") return gen::NonFluidNodeType::BOUNDARY;
        if (s == "INLET") return gen::NonFluidNodeType::INLET;
        if (s == "OUTLET") return gen::NonFluidNodeType::OUTLET;
        die("bad node type " + s);
    };
    std::string cmd;
    while (in >> cmd) {
        if (cmd == "dims") {
            long r, c; in >> r >> c;
            info.attach_domain_dimensions({r, c});
        } else if (cmd == "perimeter") {
            std::string t; in >> t;
            info.add_perimeter_nodes(type_of(t));
        } else if (cmd == "interval") {
            long a, b, c, d; std::string t; in >> a >> b >> c >> d >> t;
            info.add_nodes_interval(Point<2>({a, b}), Point<2>({c, d}), type_of(t));
        } else if (cmd == "rect") {
            long a, b, c, d; in >> a >> b >> c >> d;
            info.add_obstacle_hyper_rectangle(Point<2>({a, b}), {c, d});
        } else if (cmd == "square") {
            long a, b, e; in >> a >> b >> e;
            info.add_obstacle_hyper_square(Point<2>({a, b}), e);
        } else if (cmd == "sphere") {
            long a, b, r; in >> a >> b >> r;
            info.add_obstacle_hyper_sphere(Point<2>({a, b}), r);
        } else if (cmd == "random") {
            long n, mx, mn, seed; in >> n >> mx >> mn >> seed;
            info.add_obstacle_random_spheres(n, mx, mn, seed);
        } else {
            die("bad construct command " + cmd);
        }
    }
    const auto dims = info.get_domain_dimensions();
    const long R = dims[0], C = dims[1];
    const auto bset = info.get_boundary_nodes();
    const auto iset = info.get_inlet_nodes();
    const auto oset = info.get_outlet_nodes();
    const auto obset = info.get_obstacle_nodes();
    std::vector<BoundaryPoint<2>> boundary(bset.begin(), bset.end()), inlet(iset.begin(), iset.end()),
        outlet(oset.begin(), oset.end());
    std::vector<ObstaclePoint<2>> obstacle(obset.begin(), obset.end());
    std::vector<unsigned char> types(static_cast<std::size_t>(R * C), InputNodeType::FLUID);
    std::vector<unsigned char> listed(static_cast<std::size_t>(R * C), 0);
    auto mark = [&](long i, long j, unsigned char t) {
        const std::size_t x = static_cast<std::size_t>(i + R * j);
        if (listed[x]) die("node in more than one construction set");
        listed[x] = 1;
        types[x] = t;
    };
    for (const auto& p : boundary) mark(p.coords[0], p.coords[1], InputNodeType::BOUNDARY);
    for (const auto& p : inlet) mark(p.coords[0], p.coords[1], InputNodeType::INLET);
    for (const auto& p : outlet) mark(p.coords[0], p.coords[1], InputNodeType::OUTLET);
    for (const auto& p : obstacle) mark(p.coords[0], p.coords[1], InputNodeType::OBSTACLE);
    std::vector<Point<2>> fluid;
    for (long i = 0; i < R; ++i)
        for (long j = 0; j < C; ++j)
            if (!listed[static_cast<std::size_t>(i + R * j)]) fluid.push_back(Point<2>({i, j}));
    llalbm::util::identify_node_type<2>(dims, inlet);
    llalbm::util::identify_node_type<2>(dims, outlet);
    llalbm::util::identify_obstacle_propagation<2>(dims, obstacle, fluid, inlet, outlet);
    llalbm::util::eliminate_non_wet_nodes<2>(obstacle);
    lattice.reinit(9, dims, fluid, boundary, inlet, outlet, obstacle);
    write_raw(o.out + "/types.u8", types.data(), types.size());
}

template <typename LatticeT>
void dump_nodes(LatticeT& lat, const std::string& out) {
    std::vector<long long> v;
    for (const auto& p : lat.get_fluid_nodes()) { v.push_back(p.coords[0]); v.push_back(p.coords[1]); }
    write_raw(out + "/fluid.i64", v.data(), v.size());
    auto dump_b = [&](const std::vector<BoundaryPoint<2>>& nodes, const std::string& name) {
        std::vector<long long> w;
        for (const auto& p : nodes) { w.push_back(p.coords[0]); w.push_back(p.coords[1]); w.push_back(p.type); }
        write_raw(out + "/" + name, w.data(), w.size());
    };
    dump_b(lat.get_boundary_nodes(), "boundary.i64");
    dump_b(lat.get_inlet_nodes(), "inlet.i64");
    dump_b(lat.get_outlet_nodes(), "outlet.i64");
    std::vector<long long> o;
    for (const auto& p : lat.get_obstacle_nodes()) {
        o.push_back(p.coords[0]); o.push_back(p.coords[1]);
        o.push_back(static_cast<long long>(p.directions.to_ulong()));
    }
    write_raw(out + "/obstacle.i64", o.data(), o.size());
    const auto d = lat.get_lattice_dimensions();
    long long dims[2] = {d[0], d[1]};
    write_raw(out + "/dims.i64", dims, 2);
}

template <typename Coll>
void set_collision(const Options& o) {
    if constexpr (requires { Coll::tau; }) {
        Coll::initialize(o.tau);
    } else {
        Coll::initialize(o.tau_even, o.tau_odd > 0 ? o.tau_odd : 1.0, 1.0 / std::sqrt(3.0));
        if (o.magic > 0) Coll::enforce_magic_parameter(o.magic);
    }
}

// Lazy choice: naming SerialPolicy<2, C> checks its IsGloballySerial constraint,
// so the unused branch must never be formed.
template <bool OMP, typename C> struct ParOf { using type = SerialPolicy<2, C>; };
template <typename C> struct ParOf<true, C> { using type = OMPPolicy<2, C>; };

template <bool OMP, bool TRT, int IN, int OUT, bool PS = false>
struct Select {
    template <typename S, typename M> using pick = std::conditional_t<OMP, M, S>;
    using Coll = std::conditional_t<TRT, pick<collisions::TRTCollisionPolicy<2>, collisions::OMPTRTCollisionPolicy<2>>,
                                    pick<collisions::BGKCollisionPolicy<2>, collisions::OMPBGKCollisionPolicy<2>>>;
    using BB = pick<boundaries::BounceBackPolicy<2>, boundaries::OMPBounceBackPolicy<2>>;
    using ZH = pick<boundaries::ZouHePolicy<2>, boundaries::OMPZouHePolicy<2>>;
    using Open = pick<boundaries::OpenBoundaryPolicy<2>, boundaries::OMPOpenBoundaryPolicy<2>>;
    using ZHP = pick<boundaries::ZouHePressurePolicy<2>, boundaries::OMPZouHePressurePolicy<2>>;
    using In = std::conditional_t<IN == 0, ZH, Open>;
    using Out = std::conditional_t<OUT == 0, ZH, std::conditional_t<OUT == 1, Open, ZHP>>;
    using Init = pick<initializers::VelocityInitializer<2>, initializers::OMPVelocityInitializer<2>>;
    using Eq = pick<equilibrium::DefaultEquilibrium<2>, equilibrium::OMPDefaultEquilibrium<2>>;
    using Obst = std::conditional_t<PS, pick<boundaries::PSBounceBackPolicy<2>, boundaries::OMPPSBounceBackPolicy<2>>, BB>;
    using Config = LatticeConfiguration<2, Coll, BB, Obst, In, Out, Init, Eq>;
    using Par = typename ParOf<OMP, Config>::type;
};

template <bool OMP, bool TRT, int IN, int OUT, bool PS = false>
int run_case(const Options& o) {
    using S = Select<OMP, TRT, IN, OUT, PS>;
    using Par = typename S::Par;
    std::ofstream log(o.out + "/ref_runner.log");
    std::unique_ptr<Lattice<Par>> lat;
    if (o.geometry == "file") {
        lat = std::make_unique<Lattice<Par>>(o.path, 9, log);
    } else {
        lat = std::make_unique<Lattice<Par>>();
        if (o.geometry == "raw") build_from_raw(*lat, o);
        else if (o.geometry == "construct") build_from_script(*lat, o);
        else die("bad geometry " + o.geometry);
    }
    if (o.dump_nodes) dump_nodes(*lat, o.out);

    set_collision<typename S::Coll>(o);
    if constexpr (PS) {
        // the reference's own set-up sequence (test/unit/LidWithPSObstacle.cpp:74-76);
        // compute_obstacle_weight fills copies of the nodes, so every b stays 1
        S::Obst::initialize(o.ps_tau);
        lat->compute_obstacle_weight();
        if (o.ps_b == "pattern") {
            // per-obstacle weights set on the lattice's own nodes (ObstaclePoint::set_b),
            // which the policy reads (PSBounceBackPolicy.hpp:193)
            auto& obs = lat->get_obstacle_nodes();
            for (std::size_t q = 0; q < obs.size(); ++q)
                obs[q].set_b(static_cast<double>((37 * q + 11) % 101) / 100.0);
        } else if (o.ps_b != "default") {
            die("bad --ps-b");
        }
    }
    boundaries::ZouHePressurePolicy<2>::initialize(o.rho_out, o.tangential_u);
    boundaries::ZouHePressurePolicy<2>::reset();
    auto inlets = make_functions(o.inlet_u);
    auto outlets = make_functions(o.outlet_u);
    S::Init::attach_update_functions(inlets, outlets);

    std::shared_ptr<llalbm::analysis::FlowAnalyzer<2>> analyzer;
    if (o.analyzer_every > 0) {
        analyzer = std::make_shared<llalbm::analysis::FlowAnalyzer<2>>(
            lat->get_obstacle_nodes(), static_cast<std::size_t>(o.analyzer_every), false);
        lat->attach_flow_analyzer(analyzer);
    }

    if (o.timing) {
        if (o.warmup > 0) lat->perform_lbm(static_cast<double>(o.warmup), 1, 1, false);
        const auto t0 = std::chrono::steady_clock::now();
        lat->perform_lbm(static_cast<double>(o.steps), 1, 1, false);
        const auto t1 = std::chrono::steady_clock::now();
        const double s = std::chrono::duration<double>(t1 - t0).count();
        std::printf("\n{\"seconds\": %.6f, \"steps\": %ld, \"threads\": %d, \"rows\": %ld, \"cols\": %ld}\n", s, o.steps,
                    OMP ? omp_get_max_threads() : 1, static_cast<long>(lat->get_lattice_dimensions()[0]),
                    static_cast<long>(lat->get_lattice_dimensions()[1]));
        return 0;
    }

    lat->perform_lbm(static_cast<double>(o.steps), 1, 1, false);
    std::fflush(stdout);
    if (o.dump_fields) {
        const auto& pop = lat->get_populations();
        write_raw(o.out + "/populations.f64", pop.data(), static_cast<std::size_t>(pop.size()));
        const auto& u = lat->get_global_u();
        write_raw(o.out + "/u.f64", u.data(), static_cast<std::size_t>(u.size()));
        const auto& rho = lat->get_global_rho();
        write_raw(o.out + "/rho.f64", rho.data(), static_cast<std::size_t>(rho.size()));
    }
    if (analyzer) {
        std::vector<double> ld;
        for (const auto& p : analyzer->get_all_results()) { ld.push_back(p.first); ld.push_back(p.second); }
        write_raw(o.out + "/lift_drag.f64", ld.data(), ld.size());
    }
    return 0;
}

template <bool OMP, bool TRT>
int dispatch_bc(const Options& o) {
    const int in = o.inlet_bc == "zh" ? 0 : o.inlet_bc == "open" ? 1 : -1;
    const int out = o.outlet_bc == "zh" ? 0 : o.outlet_bc == "open" ? 1 : o.outlet_bc == "zhp" ? 2 : -1;
    if (in < 0 || out < 0) die("bad boundary policy");
    if (o.obstacle == "ps") {
        // partially saturated obstacles: Zou-He velocity inlets only
        if (in != 0) die("ps obstacles run with zh inlets");
        if (out == 0) return run_case<OMP, TRT, 0, 0, true>(o);
        if (out == 1) return run_case<OMP, TRT, 0, 1, true>(o);
        return run_case<OMP, TRT, 0, 2, true>(o);
    }
    if (o.obstacle != "bb") die("bad obstacle policy");
    if (in == 0 && out == 0) return run_case<OMP, TRT, 0, 0>(o);
    if (in == 0 && out == 1) return run_case<OMP, TRT, 0, 1>(o);
    if (in == 0 && out == 2) return run_case<OMP, TRT, 0, 2>(o);
    if (in == 1 && out == 0) return run_case<OMP, TRT, 1, 0>(o);
    if (in == 1 && out == 1) return run_case<OMP, TRT, 1, 1>(o);
    return run_case<OMP, TRT, 1, 2>(o);
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    for (int a = 1; a < argc; ++a) {
        const std::string k = argv[a];
        auto val = [&]() -> std::string {
            if (a + 1 >= argc) die("missing value for " + k);
            return argv[++a];
        };
        if (k == "--lattice-file") { o.geometry = "file"; o.path = val(); }
        else if (k == "--types-raw") { o.geometry = "raw"; o.path = val(); o.rows = std::stol(val()); o.cols = std::stol(val()); }
        else if (k == "--construct") { o.geometry = "construct"; o.path = val(); }
        else if (k == "--policy") o.policy = val();
        else if (k == "--collision") o.collision = val();
        else if (k == "--tau") o.tau = std::stod(val());
        else if (k == "--tau-even") o.tau_even = std::stod(val());
        else if (k == "--tau-odd") o.tau_odd = std::stod(val());
        else if (k == "--magic") o.magic = std::stod(val());
        else if (k == "--inlet") o.inlet_bc = val();
        else if (k == "--outlet") o.outlet_bc = val();
        else if (k == "--inlet-u") o.inlet_u = val();
        else if (k == "--outlet-u") o.outlet_u = val();
        else if (k == "--rho-out") o.rho_out = std::stod(val());
        else if (k == "--tangential-u") o.tangential_u = std::stod(val());
        else if (k == "--obstacle") o.obstacle = val();
        else if (k == "--ps-tau") o.ps_tau = std::stod(val());
        else if (k == "--ps-b") o.ps_b = val();
        else if (k == "--steps") o.steps = std::stol(val());
        else if (k == "--warmup") o.warmup = std::stol(val());
        else if (k == "--analyzer") o.analyzer_every = std::stol(val());
        else if (k == "--threads") o.threads = std::stoi(val());
        else if (k == "--timing") o.timing = true;
        else if (k == "--dump-nodes") o.dump_nodes = true;
        else if (k == "--no-fields") o.dump_fields = false;
        else if (k == "--out") o.out = val();
        else die("unknown option " + k);
    }
    if (o.threads > 0) omp_set_num_threads(o.threads);
    const bool omp = o.policy == "omp";
    const bool trt = o.collision == "trt";
    if (o.policy != "omp" && o.policy != "serial") die("bad policy");
    if (o.collision != "trt" && o.collision != "bgk") die("bad collision");
    if (omp && o.obstacle == "ps") die("ps obstacles run with the serial policies");
    if (omp && trt) return dispatch_bc<true, true>(o);
    if (omp) return dispatch_bc<true, false>(o);
    if (trt) return dispatch_bc<false, true>(o);
    return dispatch_bc<false, false>(o);
}
