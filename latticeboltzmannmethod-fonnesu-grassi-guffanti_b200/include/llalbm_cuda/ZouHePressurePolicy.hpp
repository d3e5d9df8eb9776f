/**
 * @file ZouHePressurePolicy.hpp
 * @brief Zou-He *pressure* (prescribed density) boundary policy for LLALBM's D2Q9
 *        lattice, in the style of the library's own boundary policies.
 *
 * LLALBM ships only the Zou-He *velocity* closure
 * (llalbm/src/core/boundaries/ZouHePolicy.hpp:58-123).  This header adds the
 * density-prescribed variant of Zou & He (1997) for straight walls, as Serial
 * and OpenMP policies usable as the `OutletPolicy` (or `InletPolicy`) of a
 * `LatticeConfiguration`, and recognised by `CUDAPolicy`.
 *
 * Semantics (identical in this CPU policy, the C oracle and the CUDA kernel):
 *   - the closure runs after streaming and bounce-back, like every LLALBM
 *     boundary policy (Lattice.hpp:402-410);
 *   - with rho0 prescribed, the wall-normal velocity follows from the known
 *     populations, e.g. on a RIGHT wall
 *       s  = ((p0 + p2) + p4) + 2.0 * ((p1 + p5) + p8)
 *       ux = s / rho0 - 1.0,   uy = tangential_u
 *     and the unknown populations are completed with exactly the expressions of
 *     the velocity closure (ZouHePolicy.hpp:70-118) using ru = rho0*ux,
 *     rv = rho0*uy;
 *   - corner nodes (btypes *_C) are left untouched, like ZouHePolicy;
 *   - the node then collides with feq(rho0, u) where u is the velocity the
 *     closure computed from the populations *after* the streaming that precedes
 *     that collision.
 *
 * LLALBM passes global_rho/global_u to boundary policies by value
 * (OMPPolicy.hpp:50-72), so a boundary policy cannot hand its velocity to the
 * collision directly.  The policy therefore keeps the computed velocity in a
 * static per-node cache, and `velocity_function(c)` returns update functions
 * (for VelocityInitializer::attach_update_functions) that read it back at the
 * next `update_nodes` call -- which is exactly "the velocity computed after the
 * preceding streaming".  Open nodes always collide with rho = global_rho = 1 in
 * LLALBM (the tensor is never written for them), so through LLALBM's own
 * Lattice this policy is faithful for rho0 == 1 only; CUDAPolicy uses rho0.
 */
#ifndef LLALBM_CUDA_ZOUHE_PRESSURE_POLICY_HPP
#define LLALBM_CUDA_ZOUHE_PRESSURE_POLICY_HPP

#include <functional>
#include <vector>

namespace llalbm::core::boundaries
{
    namespace zh_pressure_detail
    {
        /// Completes one straight-wall node; returns false for corners / NONE.
        /// `p` holds the 9 populations of the node (read and written in place).
        inline bool close_node(double p[9], const int side, const double rho0, const double ut,
                               double& ux_out, double& uy_out)
        {
            constexpr double two_thirds = 2.0 / 3.0;
            constexpr double one_sixth = 1.0 / 6.0;
            constexpr double one_half = 0.5;
            double ux, uy, ru, rv, s;
            switch (side)
            {
            case TOP_WALL:
                s = ((p[0] + p[1]) + p[3]) + 2.0 * ((p[2] + p[5]) + p[6]);
                ux = ut;
                uy = s / rho0 - 1.0;
                ru = rho0 * ux;
                rv = rho0 * uy;
                p[4] = p[2] - two_thirds * rv;
                p[7] = p[5] - one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
                p[8] = p[6] - one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
                break;
            case BOTTOM_WALL:
                s = ((p[0] + p[1]) + p[3]) + 2.0 * ((p[4] + p[7]) + p[8]);
                ux = ut;
                uy = 1.0 - s / rho0;
                ru = rho0 * ux;
                rv = rho0 * uy;
                p[2] = p[4] + two_thirds * rv;
                p[5] = p[7] + one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
                p[6] = p[8] + one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
                break;
            case LEFT_WALL:
                s = ((p[0] + p[2]) + p[4]) + 2.0 * ((p[3] + p[7]) + p[6]);
                ux = 1.0 - s / rho0;
                uy = ut;
                ru = rho0 * ux;
                rv = rho0 * uy;
                p[1] = p[3] + two_thirds * ru;
                p[5] = p[7] + one_sixth * ru + one_half * rv - one_half * (p[2] - p[4]);
                p[8] = p[6] + one_sixth * ru - one_half * rv + one_half * (p[2] - p[4]);
                break;
            case RIGHT_WALL:
                s = ((p[0] + p[2]) + p[4]) + 2.0 * ((p[1] + p[5]) + p[8]);
                ux = s / rho0 - 1.0;
                uy = ut;
                ru = rho0 * ux;
                rv = rho0 * uy;
                p[3] = p[1] - two_thirds * ru;
                p[7] = p[5] - one_sixth * ru - one_half * rv + one_half * (p[2] - p[4]);
                p[6] = p[8] - one_sixth * ru + one_half * rv - one_half * (p[2] - p[4]);
                break;
            default:
                return false;
            }
            ux_out = ux;
            uy_out = uy;
            return true;
        }

        /// Shared static state of the pressure policies (one set per process,
        /// like every LLALBM policy parameter).
        struct State
        {
            double rho_out = 1.0;
            double tangential_u = 0.0;
            Eigen::Index rows = 0, cols = 0;
            std::vector<double> velocity;  // (rows*cols*2), column-major like Tensor(R,C,2)

            void ensure(const Eigen::Index r, const Eigen::Index c)
            {
                if (rows != r || cols != c)
                {
                    rows = r;
                    cols = c;
                    velocity.assign(static_cast<std::size_t>(r * c * 2), 0.0);
                }
            }
            double get(const Eigen::Index i, const Eigen::Index j, const int comp) const
            {
                if (velocity.empty() || i < 0 || j < 0 || i >= rows || j >= cols) return 0.0;
                return velocity[static_cast<std::size_t>(i + rows * (j + cols * comp))];
            }
            void set(const Eigen::Index i, const Eigen::Index j, const double ux, const double uy)
            {
                velocity[static_cast<std::size_t>(i + rows * j)] = ux;
                velocity[static_cast<std::size_t>(i + rows * (j + cols))] = uy;
            }
        };

        inline State& state()
        {
            static State s;
            return s;
        }

        inline void update(Tensor<double, 3>& populations, const std::vector<BoundaryPoint<2>>& nodes,
                           const std::size_t begin, const std::size_t end)
        {
            State& st = state();
            for (std::size_t n = begin; n < end; ++n)
            {
                const Eigen::Index i = nodes[n].coords[0];
                const Eigen::Index j = nodes[n].coords[1];
                double p[9];
                for (int k = 0; k < 9; ++k) p[k] = populations(i, j, k);
                double ux, uy;
                if (!close_node(p, nodes[n].type, st.rho_out, st.tangential_u, ux, uy)) continue;
                for (int k = 0; k < 9; ++k) populations(i, j, k) = p[k];
                st.set(i, j, ux, uy);
            }
        }
    }  // namespace zh_pressure_detail

    template <std::size_t dim>
    class ZouHePressurePolicy;

    /// Serial Zou-He pressure policy (2D).
    template <>
    class ZouHePressurePolicy<2> : public BoundaryPolicyTag, public SequentialTag
    {
      public:
        /// Sets the prescribed density and tangential velocity of the boundary.
        static void initialize(const double rho_out, const double tangential_u = 0.0)
        {
            zh_pressure_detail::state().rho_out = rho_out;
            zh_pressure_detail::state().tangential_u = tangential_u;
        }
        static double rho_out() { return zh_pressure_detail::state().rho_out; }
        static double tangential_u() { return zh_pressure_detail::state().tangential_u; }

        static void update_boundaries(Tensor<double, 3>& populations, std::vector<BoundaryPoint<2>>& boundary_coord,
                                      Tensor<double, 2> global_rho, Tensor<double, 3> global_u)
        {
            zh_pressure_detail::state().ensure(populations.dimensions()[0], populations.dimensions()[1]);
            zh_pressure_detail::update(populations, boundary_coord, 0, boundary_coord.size());
        }

        /// Update function (component 0 = u_x, 1 = u_y) returning the velocity
        /// the closure computed for the node; attach it as the outlet (or inlet)
        /// update function of the VelocityInitializer.
        static std::function<double(double, BoundaryPoint<2>)> velocity_function(const int component)
        {
            return [component](double, BoundaryPoint<2> p) {
                return zh_pressure_detail::state().get(p.coords[0], p.coords[1], component);
            };
        }

        /// Clears the cached velocities (call before a new perform_lbm run).
        static void reset() { zh_pressure_detail::state().velocity.assign(zh_pressure_detail::state().velocity.size(), 0.0); }
    };

    /// OpenMP Zou-He pressure policy (2D): same arithmetic, nodes split across threads.
    template <std::size_t dim>
    class OMPZouHePressurePolicy;

    template <>
    class OMPZouHePressurePolicy<2> : public BoundaryPolicyTag, public OMPTag
    {
      public:
        static void initialize(const double rho_out, const double tangential_u = 0.0)
        {
            ZouHePressurePolicy<2>::initialize(rho_out, tangential_u);
        }
        static double rho_out() { return zh_pressure_detail::state().rho_out; }
        static double tangential_u() { return zh_pressure_detail::state().tangential_u; }

        static void update_boundaries(Tensor<double, 3>& populations, std::vector<BoundaryPoint<2>>& boundary_coord,
                                      Tensor<double, 2> global_rho, Tensor<double, 3> global_u)
        {
            zh_pressure_detail::state().ensure(populations.dimensions()[0], populations.dimensions()[1]);
            const std::size_t n = boundary_coord.size();
#pragma omp parallel for
            for (std::size_t b = 0; b < n; ++b)
                zh_pressure_detail::update(populations, boundary_coord, b, b + 1);
        }
        static std::function<double(double, BoundaryPoint<2>)> velocity_function(const int component)
        {
            return ZouHePressurePolicy<2>::velocity_function(component);
        }
        static void reset() { ZouHePressurePolicy<2>::reset(); }
    };
}  // namespace llalbm::core::boundaries

#endif  // LLALBM_CUDA_ZOUHE_PRESSURE_POLICY_HPP
