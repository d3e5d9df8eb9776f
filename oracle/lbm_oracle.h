/*
 * lbm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of LLALBM's D2Q9 time step (Lattice<P>::perform_lbm,
 * llalbm/src/core/lattices/Lattice.hpp:288-438) in the reference's own push
 * formulation, over the reference's node lists.  It is the checker for the
 * CUDA library: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it.  Its results are pinned bit-for-bit against the
 * reference headers themselves (oracle/ref_runner.cpp) by tests/test_oracle.py.
 *
 * Layouts follow the reference's Eigen tensors (column-major, row index i
 * fastest):  populations (R, C, 9) -> i + R*(j + C*k);  u (R, C, 2);  rho (R, C).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LBO_BGK = 0, LBO_TRT = 1 };
/* open-boundary policies: Zou-He velocity (ZouHePolicy), open no-op
   (OpenBoundaryPolicy), Zou-He pressure (the extension in ZouHePressurePolicy.hpp) */
enum { LBO_BC_ZH_VELOCITY = 0, LBO_BC_OPEN = 1, LBO_BC_ZH_PRESSURE = 2 };
/* obstacle policies: BounceBackPolicy, PSBounceBackPolicy (partially saturated) */
enum { LBO_OBST_BOUNCE_BACK = 0, LBO_OBST_PARTIAL = 1 };

typedef struct {
    int64_t rows, cols;
    int64_t n_fluid;   const int64_t* fluid;                          /* [n][2] (i, j) */
    int64_t n_wall;    const int64_t* wall;                           /* [n][2] */
    int64_t n_inlet;   const int64_t* inlet;  const int32_t* inlet_side;   /* btypes */
    int64_t n_outlet;  const int64_t* outlet; const int32_t* outlet_side;
    int64_t n_obst;    const int64_t* obst;   const uint16_t* obst_dirs;   /* bit k: direction k */
    int32_t collision;                 /* LBO_BGK / LBO_TRT */
    double tau, tau_even, tau_odd;
    int32_t inlet_bc, outlet_bc;       /* LBO_BC_* */
    double rho_out, tangential_u;      /* Zou-He pressure parameters */
    int32_t obstacle_bc;               /* LBO_OBST_* */
    double ps_tau;                     /* PSBounceBackPolicy<2>::tau */
    const double* obst_b;              /* per obstacle b (ObstaclePoint::get_b), NULL: 1.0 */
} lbo_problem;

/*
 * Runs perform_lbm(steps) from a fresh start.
 *   open_u       [table_rows][n_inlet + n_outlet][2]: update-function values
 *                (inlets first, then outlets) at step t = min(t, table_rows-1).
 *                Pressure-policy nodes ignore it and read the policy's cache.
 *   analyzer_every, analyzer_pts/dirs/n: FlowAnalyzer hook (Lattice.hpp:384-387):
 *                lift/drag pairs appended to lift_drag (capacity steps pairs);
 *                *n_lift_drag receives the count.  analyzer_every == 0 disables.
 * Outputs (any may be NULL): populations (R*C*9), u (R*C*2), rho (R*C),
 *   fstar = after-collision populations of the last step (R*C*9).
 * Returns 0 on success, negative on bad input.
 */
int lbo_run(const lbo_problem* p, int64_t steps, const double* open_u, int64_t table_rows,
            int64_t analyzer_every, const int64_t* analyzer_pts, const uint16_t* analyzer_dirs,
            int64_t analyzer_n, double* lift_drag, int64_t* n_lift_drag,
            double* populations, double* u, double* rho, double* fstar);

/*
 * FlowAnalyzer<2>::compute_flow_properties (FlowAnalyzer.hpp:348-451) on a
 * populations tensor: sequential sums in point order.  out[0] = lift, out[1] = drag.
 */
void lbo_flow_properties(int64_t rows, int64_t cols, const double* densities, const int64_t* pts,
                         const uint16_t* dirs, int64_t n, double out[2]);

#ifdef __cplusplus
}
#endif
#endif
