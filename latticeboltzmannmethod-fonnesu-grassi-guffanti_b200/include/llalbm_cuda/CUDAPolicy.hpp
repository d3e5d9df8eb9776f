/**
 * @file CUDAPolicy.hpp
 * @brief CUDA parallelization policy for LLALBM: a drop-in beside OMPPolicy,
 *        SerialPolicy, STDExecPolicy and OpenACCPolicy that runs the D2Q9 time
 *        step on an NVIDIA B200 (sm_100a) through libllalbm_cuda.so.
 *
 * Include after <llalbm.hpp>; add `<repo>/include` to the include path and link
 * libllalbm_cuda.so.  A program switches by changing one template argument:
 *
 *     using Parallelization = llalbm::core::CUDAPolicy<2, Configuration>;  // was OMPPolicy
 *     llalbm::core::Lattice<Parallelization> lattice(...);
 *
 * The Configuration keeps the reference's policy types (any of the Serial,
 * OpenMP, std::execution and OpenACC families): BGK or TRT collision,
 * BounceBack walls and obstacles (obstacles also PSBounceBack, partially
 * saturated), ZouHe / OpenBoundary / ZouHePressure
 * inlets and outlets, VelocityInitializer, DefaultEquilibrium.  Their static
 * parameters (tau, tau_even / tau_odd, the update functions, the pressure
 * policy's rho_out) are read when perform_lbm starts, as the reference's
 * policies read them while it runs.  Anything else fails a static_assert.
 *
 * Lattice<CUDAPolicy<2, C>> is a partial specialization with the reference
 * Lattice's public surface (llalbm/src/core/lattices/Lattice.hpp:46-643):
 * the three constructors, reinit (used by build_lattice), perform_lbm,
 * the getters, print_lattice_structure and attach_flow_analyzer.  The
 * populations stay on the GPU between calls; the getters copy them back.
 * Engine errors throw std::runtime_error with the engine's message.
 */
#ifndef LLALBM_CUDA_POLICY_HPP
#define LLALBM_CUDA_POLICY_HPP

#include <llalbm_cuda.h>

#include <algorithm>
#include <bitset>
#include <chrono>
#include <fstream>
#include <cstdlib>
#include <iostream>
#include <map>
#include <sstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "ZouHePressurePolicy.hpp"

namespace llalbm::core
{
    /// Tag of the CUDA parallelization family.
    class CUDATag {};

    namespace cuda_detail
    {
        template <class T, template <std::size_t> class... Family>
        inline constexpr bool is_any = (std::is_same_v<T, Family<2>> || ...);

        template <class C>
        inline constexpr bool is_bgk = is_any<C, collisions::BGKCollisionPolicy, collisions::OMPBGKCollisionPolicy,
                                              collisions::STDExecBGKCollisionPolicy, collisions::OpenACCBGKCollisionPolicy>;
        template <class C>
        inline constexpr bool is_trt = is_any<C, collisions::TRTCollisionPolicy, collisions::OMPTRTCollisionPolicy,
                                              collisions::STDExecTRTCollisionPolicy, collisions::OpenACCTRTCollisionPolicy>;
        template <class B>
        inline constexpr bool is_bounce_back = is_any<B, boundaries::BounceBackPolicy, boundaries::OMPBounceBackPolicy,
                                                      boundaries::STDExecBounceBackPolicy, boundaries::OpenACCBounceBackPolicy>;
        // partially saturated bounce-back (PSBounceBackPolicy.hpp): plain
        // bounce-back on walls, the partially saturated rule on obstacles
        template <class B>
        inline constexpr bool is_ps_bounce_back =
            is_any<B, boundaries::PSBounceBackPolicy, boundaries::OMPPSBounceBackPolicy,
                   boundaries::STDExecPSBounceBackPolicy, boundaries::OpenACCPSBounceBackPolicy>;
        template <class B>
        inline constexpr bool is_zou_he = is_any<B, boundaries::ZouHePolicy, boundaries::OMPZouHePolicy,
                                                 boundaries::STDExecZouHePolicy, boundaries::OpenACCZouHePolicy>;
        template <class B>
        inline constexpr bool is_open = is_any<B, boundaries::OpenBoundaryPolicy, boundaries::OMPOpenBoundaryPolicy,
                                               boundaries::STDExecOpenBoundaryPolicy, boundaries::OpenACCOpenBoundaryPolicy>;
        template <class B>
        inline constexpr bool is_pressure = is_any<B, boundaries::ZouHePressurePolicy, boundaries::OMPZouHePressurePolicy>;
        template <class I>
        inline constexpr bool is_velocity_init =
            is_any<I, initializers::VelocityInitializer, initializers::OMPVelocityInitializer,
                   initializers::STDExecVelocityInitializer, initializers::OpenACCVelocityInitializer>;
        template <class E>
        inline constexpr bool is_default_eq =
            is_any<E, equilibrium::DefaultEquilibrium, equilibrium::OMPDefaultEquilibrium,
                   equilibrium::STDExecDefaultEquilibrium, equilibrium::OpenACCDefaultEquilibrium>;

        template <class B>
        constexpr int open_bc()
        {
            if constexpr (is_zou_he<B>) return LLB_BC_ZH_VELOCITY;
            else if constexpr (is_open<B>) return LLB_BC_OPEN;
            else if constexpr (is_pressure<B>) return LLB_BC_ZH_PRESSURE;
            else return -1;
        }

        inline void check(int rc, llb_handle h, const char* what)
        {
            if (rc != LLB_OK)
                throw std::runtime_error(std::string("CUDAPolicy: ") + what + ": " + llb_last_error(h));
        }

        struct HandleDeleter
        {
            void operator()(llb_lattice* h) const
            {
                if (h) llb_destroy(h);
            }
        };
        using Handle = std::unique_ptr<llb_lattice, HandleDeleter>;

        struct WriterDeleter
        {
            void operator()(llb_writer* w) const
            {
                if (w) llb_writer_destroy(w);
            }
        };
        using Writer = std::unique_ptr<llb_writer, WriterDeleter>;

        inline void check_writer(int rc, llb_writer_handle w, const char* what)
        {
            if (rc != LLB_OK)
                throw std::runtime_error(std::string("CUDAPolicy: ") + what + ": " + llb_writer_last_error(w));
        }

        /**
         * The reference's lattice-file reader, read_lattice_file<2>
         * (utils/readers/LatticeReader.hpp:367-522), with its classification --
         * the per-node std::find scans of identify_obstacle_propagation
         * (utils/analysis/NodeIdentification.hpp:137-211), O(N^2) -- replaced by
         * the library's O(R*C) one (llb_classify_*, the same rules).  Same file
         * format and header checks (dimensions 2, positive extents, per-type
         * counts summing to R*C, one `i j type` line per non-fluid node), and the
         * same node vectors in the same order: fluid, boundary (type NONE),
         * inlet and outlet (their side), wet obstacles (their direction bits).
         * Where the reference asserts, this throws std::runtime_error; a header
         * count that differs from the nodes listed also throws (the reference's
         * vectors would keep default entries or overflow their .at()).
         */
        inline void read_lattice_file_fast(const std::string& path, std::vector<Point<2>>& fluid,
                                           std::vector<BoundaryPoint<2>>& boundary,
                                           std::vector<BoundaryPoint<2>>& inlet, std::vector<BoundaryPoint<2>>& outlet,
                                           std::vector<ObstaclePoint<2>>& obstacle,
                                           std::array<Eigen::Index, 2>& dims)
        {
            std::ifstream in(path);
            if (!in.is_open()) throw std::runtime_error("lattice file could not be opened: " + path);
            auto bad = [&](const std::string& why) { return std::runtime_error("lattice file " + path + ": " + why); };
            auto numbers = [&](std::vector<long long>& v) {
                std::string line;
                if (!std::getline(in, line)) throw bad("header ends early");
                std::istringstream ss(line);
                long long x;
                v.clear();
                while (ss >> x) v.push_back(x);
            };
            std::vector<long long> h;
            numbers(h);
            if (h.size() != 1 || h[0] != 2) throw bad("file and template dimensions do not match");
            numbers(h);
            if (h.size() != 2 || h[0] <= 0 || h[1] <= 0) throw bad("extensions must be two positive numbers");
            const long long R = h[0], C = h[1];
            std::vector<long long> counts;
            numbers(counts);
            long long total = 0;
            for (long long c : counts) {
                if (c < 0) throw bad("negative node count");
                total += c;
            }
            if (counts.size() < 6 || total != R * C) throw bad("node counts do not add up to the lattice size");
            // InputNodeType codes (utils/aliases.hpp): FLUID 0, SOLID 1, BOUNDARY 2, INLET 3, OUTLET 4, OBSTACLE 5
            std::vector<uint8_t> types(static_cast<std::size_t>(R * C), LLB_NODE_FLUID);
            // the file lists the non-fluid nodes; every other node is fluid
            const long long listed = total - counts[0];
            long long tally[6] = {R * C - listed, 0, 0, 0, 0, 0};
            for (long long q = 0; q < listed; ++q) {
                long long i, j, t;
                if (!(in >> i >> j >> t)) throw bad("fewer node lines than the header announces");
                if (i < 0 || j < 0 || i >= R || j >= C || t < 0 || t > 5) throw bad("node line out of range");
                uint8_t& cell = types[static_cast<std::size_t>(i + R * j)];
                if (cell != LLB_NODE_FLUID) throw bad("node listed twice");
                cell = static_cast<uint8_t>(t);
                ++tally[t];
            }
            for (int t = 0; t < 6; ++t)
                if (tally[t] != counts[static_cast<std::size_t>(t)]) throw bad("header counts differ from the nodes listed");
            int64_t n[5];
            if (llb_classify_count(R, C, types.data(), n) != LLB_OK)
                throw bad("an inlet or outlet node lies off the lattice perimeter");
            std::vector<int64_t> fij(2 * n[0]), wij(2 * n[1]), iij(2 * n[2]), oij(2 * n[3]), bij(2 * n[4]);
            std::vector<int32_t> iside(n[2]), oside(n[3]);
            std::vector<uint16_t> dirs(n[4]);
            llb_node_lists L{n[0], n[1], n[2], n[3], n[4], fij.data(), wij.data(), iij.data(), iside.data(),
                             oij.data(), oside.data(), bij.data(), dirs.data()};
            if (llb_classify_fill(R, C, types.data(), &L) != LLB_OK) throw bad("classification failed");
            dims = {static_cast<Eigen::Index>(R), static_cast<Eigen::Index>(C)};
            fluid.resize(static_cast<std::size_t>(n[0]));
            for (int64_t q = 0; q < n[0]; ++q) {
                fluid[q].coords[0] = fij[2 * q];
                fluid[q].coords[1] = fij[2 * q + 1];
            }
            auto fill_boundary = [](std::vector<BoundaryPoint<2>>& v, const std::vector<int64_t>& ij,
                                    const int32_t* side, int64_t m) {
                v.resize(static_cast<std::size_t>(m));
                for (int64_t q = 0; q < m; ++q) {
                    v[q].coords[0] = ij[2 * q];
                    v[q].coords[1] = ij[2 * q + 1];
                    v[q].type = side ? static_cast<btypes>(side[q]) : btypes::NONE;
                }
            };
            fill_boundary(boundary, wij, nullptr, n[1]);
            fill_boundary(inlet, iij, iside.data(), n[2]);
            fill_boundary(outlet, oij, oside.data(), n[3]);
            obstacle.resize(static_cast<std::size_t>(n[4]));
            for (int64_t q = 0; q < n[4]; ++q) {
                obstacle[q].coords[0] = bij[2 * q];
                obstacle[q].coords[1] = bij[2 * q + 1];
                obstacle[q].directions = std::bitset<9>(dirs[q]);
            }
        }
    }  // namespace cuda_detail

    template <std::size_t dim, typename Configuration>
    class CUDAPolicy : public CUDATag
    {
        static_assert(dim == 2, "CUDAPolicy implements the D2Q9 lattice only");
    };

    /// 2D specialization: maps the Configuration's policies onto the engine.
    template <typename Configuration>
    class CUDAPolicy<2, Configuration> : public CUDATag
    {
      public:
        static constexpr std::size_t dims = Configuration::dimensions;
        using CollisionPolicy = typename Configuration::collision_policy_t;
        using WallPolicy = typename Configuration::wall_policy_t;
        using ObstaclePolicy = typename Configuration::obstacle_policy_t;
        using InletPolicy = typename Configuration::inlet_policy_t;
        using OutletPolicy = typename Configuration::outlet_policy_t;
        using InitializationPolicy = typename Configuration::initialization_policy_t;
        using EquilibriumPolicy = typename Configuration::equilibrium_policy_t;

        static_assert(dims == 2, "CUDAPolicy implements the D2Q9 lattice only");
        static_assert(cuda_detail::is_bgk<CollisionPolicy> || cuda_detail::is_trt<CollisionPolicy>,
                      "CUDAPolicy: the collision policy must be a BGK or TRT policy");
        static_assert((cuda_detail::is_bounce_back<WallPolicy> || cuda_detail::is_ps_bounce_back<WallPolicy>) &&
                          (cuda_detail::is_bounce_back<ObstaclePolicy> ||
                           cuda_detail::is_ps_bounce_back<ObstaclePolicy>),
                      "CUDAPolicy: walls and obstacles must use a BounceBack or PSBounceBack policy");
        static_assert(cuda_detail::open_bc<InletPolicy>() >= 0 && cuda_detail::open_bc<OutletPolicy>() >= 0,
                      "CUDAPolicy: inlets/outlets must use ZouHe, OpenBoundary or ZouHePressure");
        static_assert(cuda_detail::is_velocity_init<InitializationPolicy>,
                      "CUDAPolicy: the initialization policy must be a VelocityInitializer");
        static_assert(cuda_detail::is_default_eq<EquilibriumPolicy>,
                      "CUDAPolicy: the equilibrium policy must be DefaultEquilibrium");

        static constexpr int collision = cuda_detail::is_bgk<CollisionPolicy> ? LLB_BGK : LLB_TRT;
        static constexpr int inlet_bc = cuda_detail::open_bc<InletPolicy>();
        static constexpr int outlet_bc = cuda_detail::open_bc<OutletPolicy>();

        /// As every reference policy: hands the open nodes to the initializer.
        static void attach_nodes(std::vector<BoundaryPoint<2>>& inlet_nodes, std::vector<BoundaryPoint<2>>& outlet_nodes)
        {
            InitializationPolicy::attach_nodes(inlet_nodes, outlet_nodes);
        }

        static void fill_collision(llb_desc& d)
        {
            d.collision = collision;
            if constexpr (cuda_detail::is_bgk<CollisionPolicy>)
            {
                d.tau = CollisionPolicy::tau;
            }
            else
            {
                d.tau_even = CollisionPolicy::tau_even;
                d.tau_odd = CollisionPolicy::tau_odd;
            }
        }

        /// Boundary values of step t for the open nodes, inlets then outlets:
        /// the update functions' (u_x, u_y), or (rho0, tangential u) for the
        /// Zou-He pressure policy.
        static void open_values(double t, const std::vector<BoundaryPoint<2>>& inlets,
                                const std::vector<BoundaryPoint<2>>& outlets, double* out)
        {
            std::size_t q = 0;
            auto fill = [&](const std::vector<BoundaryPoint<2>>& nodes, auto fn, int bc, double rho0, double ut) {
                for (const auto& node : nodes)
                {
                    if (bc == LLB_BC_ZH_PRESSURE)
                    {
                        out[2 * q] = rho0;
                        out[2 * q + 1] = ut;
                    }
                    else
                    {
                        out[2 * q] = fn[0](t, node);
                        out[2 * q + 1] = fn[1](t, node);
                    }
                    ++q;
                }
            };
            double ri = 1.0, ui = 0.0, ro = 1.0, uo = 0.0;
            if constexpr (inlet_bc == LLB_BC_ZH_PRESSURE)
            {
                ri = InletPolicy::rho_out();
                ui = InletPolicy::tangential_u();
            }
            if constexpr (outlet_bc == LLB_BC_ZH_PRESSURE)
            {
                ro = OutletPolicy::rho_out();
                uo = OutletPolicy::tangential_u();
            }
            fill(inlets, InitializationPolicy::inlet_update_function, inlet_bc, ri, ui);
            fill(outlets, InitializationPolicy::outlet_update_function, outlet_bc, ro, uo);
        }
    };

    /**
     * Lattice running on the GPU.  Same public API as the reference Lattice.
     */
    template <typename Configuration>
    class Lattice<CUDAPolicy<2, Configuration>>
    {
      public:
        using Policy = CUDAPolicy<2, Configuration>;
        static constexpr std::size_t dim = 2;

      private:
        static constexpr std::size_t CHUNK = 256;  // steps per engine call between host events

        Tensor<double, 3> populations;
        Tensor<double, 3> after_collision_populations;
        Tensor<double, 2> global_rho;
        Tensor<double, 3> global_u;
        std::array<Eigen::Index, 2> lattice_dimensions{};
        std::vector<Point<2>> fluid_nodes;
        std::vector<BoundaryPoint<2>> boundary_coord;
        std::vector<BoundaryPoint<2>> inlet_nodes_coord;
        std::vector<BoundaryPoint<2>> outlet_nodes_coord;
        std::vector<ObstaclePoint<2>> obstacle_nodes;
        std::size_t q = 0;
        std::shared_ptr<llalbm::analysis::FlowAnalyzer<2>> flow_analyzer = nullptr;
        llalbm::util::logger::Logger logger;
        cuda_detail::Handle engine;
        int device = 0;

        void build_tensors()
        {
            const Eigen::Index R = lattice_dimensions[0], C = lattice_dimensions[1];
            populations = Tensor<double, 3>(std::array<Eigen::Index, 3>{R, C, static_cast<Eigen::Index>(q)});
            after_collision_populations = Tensor<double, 3>(std::array<Eigen::Index, 3>{R, C, static_cast<Eigen::Index>(q)});
            global_rho = Tensor<double, 2>(std::array<Eigen::Index, 2>{R, C});
            global_u = Tensor<double, 3>(std::array<Eigen::Index, 3>{R, C, 2});
            engine.reset();
        }

        template <class P>
        static std::vector<int64_t> coords(const std::vector<P>& v)
        {
            std::vector<int64_t> out(2 * v.size());
            for (std::size_t n = 0; n < v.size(); ++n)
            {
                out[2 * n] = v[n].coords[0];
                out[2 * n + 1] = v[n].coords[1];
            }
            return out;
        }

        static std::vector<int32_t> sides(const std::vector<BoundaryPoint<2>>& v)
        {
            std::vector<int32_t> out(v.size());
            for (std::size_t n = 0; n < v.size(); ++n) out[n] = static_cast<int32_t>(v[n].type);
            return out;
        }

        void create_engine()
        {
            if (q != 9) throw std::runtime_error("CUDAPolicy: D2Q9 needs q = 9");
            const auto f = coords(fluid_nodes), w = coords(boundary_coord), in = coords(inlet_nodes_coord),
                       out = coords(outlet_nodes_coord), ob = coords(obstacle_nodes);
            const auto is = sides(inlet_nodes_coord), os = sides(outlet_nodes_coord);
            std::vector<uint16_t> dirs(obstacle_nodes.size());
            for (std::size_t n = 0; n < obstacle_nodes.size(); ++n)
                dirs[n] = static_cast<uint16_t>(obstacle_nodes[n].directions.to_ulong());
            llb_desc d{};
            d.rows = lattice_dimensions[0];
            d.cols = lattice_dimensions[1];
            d.n_fluid = static_cast<int64_t>(fluid_nodes.size());
            d.fluid_ij = f.data();
            d.n_wall = static_cast<int64_t>(boundary_coord.size());
            d.wall_ij = w.data();
            d.n_inlet = static_cast<int64_t>(inlet_nodes_coord.size());
            d.inlet_ij = in.data();
            d.inlet_side = is.data();
            d.n_outlet = static_cast<int64_t>(outlet_nodes_coord.size());
            d.outlet_ij = out.data();
            d.outlet_side = os.data();
            d.n_obstacle = static_cast<int64_t>(obstacle_nodes.size());
            d.obstacle_ij = ob.data();
            d.obstacle_dirs = dirs.data();
            d.inlet_bc = Policy::inlet_bc;
            d.outlet_bc = Policy::outlet_bc;
            Policy::fill_collision(d);
            std::vector<double> obstacle_b;
            if constexpr (cuda_detail::is_ps_bounce_back<typename Policy::ObstaclePolicy>)
            {
                // the policy's tau and each obstacle's b, read when the run starts
                d.obstacle_bc = LLB_OBSTACLE_PARTIAL;
                d.ps_tau = Policy::ObstaclePolicy::tau;
                obstacle_b.resize(obstacle_nodes.size());
                for (std::size_t n = 0; n < obstacle_nodes.size(); ++n) obstacle_b[n] = obstacle_nodes[n].get_b();
                d.obstacle_b = obstacle_b.data();
            }
            d.storage = LLB_STORE_F64;
            d.pattern = LLB_PATTERN_AB;
            d.device = device;
            d.open_table_rows = static_cast<int32_t>(CHUNK + 1);
            llb_handle h = nullptr;
            cuda_detail::check(llb_create(&d, &h), nullptr, "llb_create");
            engine.reset(h);
        }

        std::size_t n_open() const { return inlet_nodes_coord.size() + outlet_nodes_coord.size(); }

        // uploads boundary values of steps [t0, t0 + count)
        void upload_values(std::size_t t0, std::size_t count, std::vector<double>& buf)
        {
            if (n_open() == 0) return;
            buf.resize(count * n_open() * 2);
            for (std::size_t r = 0; r < count; ++r)
                Policy::open_values(static_cast<double>(t0 + r), inlet_nodes_coord, outlet_nodes_coord,
                                    buf.data() + r * n_open() * 2);
            cuda_detail::check(llb_set_open_values(engine.get(), static_cast<int64_t>(t0), static_cast<int32_t>(count),
                                                   buf.data()),
                               engine.get(), "llb_set_open_values");
        }

        void pull_macro()
        {
            cuda_detail::check(llb_get_macro(engine.get(), global_rho.data(), global_u.data()), engine.get(),
                               "llb_get_macro");
        }

        // FlowAnalyzer on the post-collision state: the values the analyzer reads
        // are gathered on the GPU and placed into the host tensor it is given.
        void analyze(const std::vector<ObstaclePoint<2>>& pts)
        {
            std::vector<double> vals(pts.size() * 8);
            cuda_detail::check(llb_gather_force_inputs(engine.get(), vals.data()), engine.get(),
                               "llb_gather_force_inputs");
            static const int di[9] = {0, 0, -1, 0, 1, -1, -1, 1, 1};
            static const int dj[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
            static const int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
            const Eigen::Index R = lattice_dimensions[0], C = lattice_dimensions[1];
            for (std::size_t n = 0; n < pts.size(); ++n)
                for (int k = 1; k < 9; ++k)
                {
                    if (!pts[n].directions.test(static_cast<std::size_t>(k))) continue;
                    const Eigen::Index i = pts[n].coords[0] + di[k], j = pts[n].coords[1] + dj[k];
                    if (i < 0 || j < 0 || i >= R || j >= C) continue;
                    after_collision_populations(i, j, opp[k]) = vals[n * 8 + (k - 1)];
                }
            flow_analyzer->compute_flow_properties(after_collision_populations);
        }

      public:
        Lattice() : logger("LATTICE", std::cout) {}

        Lattice(const std::array<Eigen::Index, 2>& lattice_dimensions_, const std::size_t& q_,
                std::ostream& out_stream = std::cout)
            : lattice_dimensions(lattice_dimensions_), q(q_), logger("LATTICE", out_stream)
        {
            logger.info("Constructing CUDA Lattice Object...");
            build_tensors();
            Policy::attach_nodes(inlet_nodes_coord, outlet_nodes_coord);
        }

        Lattice(const std::string& path_, const std::size_t& q_, std::ostream& out_stream = std::cout)
            : q(q_), logger("LATTICE", out_stream)
        {
            cuda_detail::read_lattice_file_fast(path_, fluid_nodes, boundary_coord, inlet_nodes_coord,
                                                outlet_nodes_coord, obstacle_nodes, lattice_dimensions);
            logger.info("Constructing CUDA Lattice Object...");
            build_tensors();
            Policy::attach_nodes(inlet_nodes_coord, outlet_nodes_coord);
        }

        /// Selects the CUDA device (default 0); call before perform_lbm.
        void set_device(int device_) { device = device_; engine.reset(); }

        void reinit(const std::size_t q_, const std::array<Eigen::Index, 2>& lattice_dimensions_,
                    const std::vector<Point<2>>& fluid_nodes_, const std::vector<BoundaryPoint<2>>& boundary_coord_,
                    const std::vector<BoundaryPoint<2>>& inlet_nodes_coord_,
                    const std::vector<BoundaryPoint<2>>& outlet_nodes_coord_,
                    const std::vector<ObstaclePoint<2>>& obstacle_nodes_)
        {
            logger.info("Reinitializing CUDA lattice");
            q = q_;
            lattice_dimensions = lattice_dimensions_;
            build_tensors();
            boundary_coord = boundary_coord_;
            inlet_nodes_coord = inlet_nodes_coord_;
            outlet_nodes_coord = outlet_nodes_coord_;
            obstacle_nodes = obstacle_nodes_;
            fluid_nodes = fluid_nodes_;
            Policy::attach_nodes(inlet_nodes_coord, outlet_nodes_coord);
        }

        /**
         * Runs the simulation like the reference perform_lbm (Lattice.hpp:288-438):
         * fresh equilibrium start, `time / time_step` steps, u written to
         * results/ every save_step steps, FlowAnalyzer hook, NaN check under
         * LLALBM_DEBUG.  The update functions receive the step index as time.
         * The output files are the reference writer's, byte for byte
         * (LatticeWriter.hpp:60-92); a save only enqueues the copy of u on the
         * engine's stream, and a native writer thread formats and writes the
         * files while the next steps run.  All files are written when
         * perform_lbm returns.
         */
        void perform_lbm(const double time, const double time_step = 1, const std::size_t save_step = 1,
                         const bool should_save = true)
        {
            if (!(time_step > 0) || !(time > 0) || !(time > time_step))
                throw std::invalid_argument("perform_lbm: need time > time_step > 0");
            if (should_save) llalbm::util::writer::create_output_directory();
            else logger.info("Results will not be saved");
            if (flow_analyzer) flow_analyzer->initialize();
            else logger.info("Flow analyzer not attached");

            const std::size_t n_steps = static_cast<std::size_t>(time / time_step);
            create_engine();
            llb_handle h = engine.get();
            cuda_detail::Writer writer;
            if (should_save)
            {
                llb_writer_handle w = nullptr;
                const int rc = llb_writer_create(llalbm::util::writer::output_dir_path.c_str(), 3, 0, &w);
                if (rc != LLB_OK) throw std::runtime_error("CUDAPolicy: llb_writer_create failed");
                writer.reset(w);
            }
            auto save = [&](std::size_t n) {
                cuda_detail::check_writer(llb_writer_save_u(writer.get(), h, static_cast<int64_t>(n)), writer.get(),
                                          "llb_writer_save_u");
            };
            std::vector<ObstaclePoint<2>> analyzer_points;
            if (flow_analyzer)
            {
                analyzer_points = flow_analyzer->get_points();
                const auto ij = coords(analyzer_points);
                std::vector<uint16_t> dirs(analyzer_points.size());
                for (std::size_t n = 0; n < dirs.size(); ++n)
                    dirs[n] = static_cast<uint16_t>(analyzer_points[n].directions.to_ulong());
                cuda_detail::check(llb_set_force_points(h, ij.data(), dirs.data(), static_cast<int64_t>(ij.size() / 2)),
                                   h, "llb_set_force_points");
                after_collision_populations.setConstant(0.0);
            }
            const std::size_t every = flow_analyzer ? flow_analyzer->get_iterations_between_save() : 0;
            auto is_save = [&](std::size_t i) { return should_save && i % save_step == 0; };
            auto is_analysis = [&](std::size_t i) { return every > 0 && i > 0 && i % every == 0; };
            std::size_t saved_file = 0;
            std::vector<double> buf;

            logger.info("Will do " + std::to_string(n_steps) + " steps");
#ifdef TIMER
            const auto start = std::chrono::high_resolution_clock::now();
#endif
            // step 0: initial equilibrium + first collision
            upload_values(0, std::min<std::size_t>(CHUNK, std::max<std::size_t>(n_steps, 1)), buf);
            const bool macro0 = is_save(0) || n_steps == 1;
            cuda_detail::check(llb_init(h, macro0 ? LLB_STEP_MACRO : 0u), h, "llb_init");
            if (is_save(0)) save(saved_file++);
            std::size_t uploaded_to = std::min<std::size_t>(CHUNK, n_steps);  // rows [0, uploaded_to) are set
            std::size_t i = 1;
            while (i < n_steps)
            {
                // run up to (and including) the next step that needs the host
                std::size_t last = std::min<std::size_t>(n_steps - 1, i + CHUNK - 1);
                for (std::size_t s = i; s <= last; ++s)
                    if (is_save(s) || is_analysis(s)) { last = s; break; }
                // The engine keeps CHUNK + 1 rows of boundary values and step t reads
                // rows t and t - 1: refill only once every uploaded row is consumed.
                if (i == uploaded_to)
                {
                    const std::size_t count = std::min<std::size_t>(CHUNK, n_steps - uploaded_to);
                    upload_values(uploaded_to, count, buf);
                    uploaded_to += count;
                }
                last = std::min(last, uploaded_to - 1);
                const bool macro = is_save(last) || last == n_steps - 1;
                cuda_detail::check(llb_step(h, static_cast<int32_t>(last - i + 1), macro ? LLB_STEP_MACRO : 0u), h,
                                   "llb_step");
#ifndef LLALBM_VERBOSE
                std::cout << "\rStep " + std::to_string(last) + " / " + std::to_string(n_steps) << std::flush;
#endif
                if (is_save(last)) save(saved_file++);
                if (is_analysis(last)) analyze(analyzer_points);
#ifdef LLALBM_DEBUG
                if (llb_check_numerics(h) == LLB_E_NUMERIC)
                {
                    logger.error("Numerical instability detected in the velocity tensor");
                    exit(1);
                }
#endif
                i = last + 1;
            }
            cuda_detail::check(llb_synchronize(h), h, "llb_synchronize");
            if (writer)
                cuda_detail::check_writer(llb_writer_flush(writer.get()), writer.get(), "llb_writer_flush");
            pull_macro();  // global_rho / global_u of the last step, as the reference leaves them
#ifdef TIMER
            const auto end = std::chrono::high_resolution_clock::now();
            std::chrono::duration<double> duration = end - start;
            std::cout << std::endl << "Time: " << duration.count() << std::endl;
#endif
            if (flow_analyzer) flow_analyzer->save_global_results();
            logger.info("\n");
            logger.info("Done!");
        }

        /// Streams the resident state to the reference's `populations` (fluid,
        /// inlet and outlet nodes; 0 elsewhere) and returns it.
        Eigen::Tensor<double, 3>& get_populations()
        {
            if (engine) cuda_detail::check(llb_get_populations(engine.get(), populations.data()), engine.get(),
                                           "llb_get_populations");
            return populations;
        }
        Eigen::Tensor<double, 3>& get_global_u() { return global_u; }
        Eigen::Tensor<double, 2>& get_global_rho() { return global_rho; }
        std::array<Eigen::Index, 2>& get_lattice_dimensions() { return lattice_dimensions; }
        std::vector<Point<2>>& get_fluid_nodes() { return fluid_nodes; }
        std::vector<BoundaryPoint<2>>& get_boundary_nodes() { return boundary_coord; }
        std::vector<BoundaryPoint<2>>& get_inlet_nodes() { return inlet_nodes_coord; }
        std::vector<BoundaryPoint<2>>& get_outlet_nodes() { return outlet_nodes_coord; }
        std::vector<ObstaclePoint<2>>& get_obstacle_nodes() { return obstacle_nodes; }
        /// The engine handle (valid after perform_lbm), for direct C-ABI calls.
        llb_handle engine_handle() { return engine.get(); }

        /// Same listing as the reference's print_lattice_structure.
        void print_lattice_structure(std::ostream& out, const bool print_fluid = false) const
        {
            unsigned int count = 0;
            out << "Lattice Information" << std::endl << "-> List of obstacle nodes: " << std::endl;
            for (const auto& p : obstacle_nodes)
            {
                out << p.coords[0] << " " << p.coords[1] << " propagation direction " << p.directions.to_string()
                    << std::endl;
                ++count;
            }
            auto typed = [&](const char* title, const std::vector<BoundaryPoint<2>>& v) {
                out << title << std::endl;
                for (const auto& p : v)
                {
                    out << p.coords[0] << " " << p.coords[1] << " type " << p.type << std::endl;
                    ++count;
                }
            };
            typed("-> List of inlet nodes: ", inlet_nodes_coord);
            typed("-> List of outlet nodes: ", outlet_nodes_coord);
            typed("-> List of boundary nodes: ", boundary_coord);
            out << "===================================" << std::endl
                << "Cumulative number of non fluid: " << count << std::endl
                << "===================================" << std::endl;
            if (print_fluid)
            {
                out << "List of fluid nodes: " << std::endl;
                for (const auto& p : fluid_nodes) out << p.coords[0] << " " << p.coords[1] << " " << std::endl;
            }
        }

        void attach_flow_analyzer(std::shared_ptr<llalbm::analysis::FlowAnalyzer<2>> flow_analyzer_)
        {
            flow_analyzer = flow_analyzer_->shared_from_this();
        }

        /**
         * The reference's weight pass for partially saturated obstacles
         * (Lattice.hpp:245-278): b of every obstacle in a 5 x 5 block = the
         * block's obstacle count / 25.  The reference stores those weights
         * into copies of the nodes it groups by block, so the lattice's own
         * obstacle nodes keep their b (1 unless set before reinit); the same
         * happens here, which keeps the runs identical to the reference's.
         */
        void compute_obstacle_weight()
        {
            std::map<std::pair<int, int>, std::vector<ObstaclePoint<2>>> blocks;
            for (const auto& p : obstacle_nodes)
                blocks[{static_cast<int>(p.coords[0] / 5), static_cast<int>(p.coords[1] / 5)}].push_back(p);
            for (auto& block : blocks)
                for (auto& p : block.second) p.set_b(static_cast<double>(block.second.size()) / 25.0);
        }
    };
}  // namespace llalbm::core

#endif  // LLALBM_CUDA_POLICY_HPP
