/*
 * lbm_oracle.c -- TEST INFRASTRUCTURE ONLY (see lbm_oracle.h).
 *
 * A restatement of LLALBM's D2Q9 step in plain C.  Every function mirrors one
 * reference policy call, in the order perform_lbm issues them, with the same
 * floating-point expressions (C and C++ share operator precedence and
 * left-to-right association; the file is built with -ffp-contract=off so no
 * multiply-add is fused, like the reference's default x86-64 build).
 * Reference paths are relative to the LLALBM project root.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* btypes (llalbm/src/utils/aliases.hpp:28-38) */
enum { BT_NONE = 0, BT_TOP = 1, BT_RIGHT = 2, BT_BOTTOM = 3, BT_LEFT = 4 };

typedef struct {
    int64_t R, C;
    double* pop;   /* populations */
    double* eq;    /* equilibrium_populations */
    double* post;  /* after_collision_populations */
    double* rho;   /* global_rho */
    double* u;     /* global_u */
} lattice_t;

#define P(T, i, j, k) (T)[(i) + L->R * ((j) + L->C * (int64_t)(k))]
#define RHO(i, j) L->rho[(i) + L->R * (j)]
#define U(i, j, c) L->u[(i) + L->R * ((j) + L->C * (int64_t)(c))]

/* DefaultEquilibrium<2>::calc_equilibrium (DefaultEquilibrium.hpp:54-78 and the
   BoundaryPoint overload :88-112 -- identical bodies). */
static void calc_equilibrium(lattice_t* L, const int64_t* nodes, int64_t n, double* out)
{
    const double two9 = (2.0 / 9.0);
    const double one18 = (1.0 / 18.0);
    const double one36 = (1.0 / 36.0);
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        const double rho = RHO(i, j);
        const double ux = U(i, j, 0);
        const double uy = U(i, j, 1);
        const double u2 = ux * ux + uy * uy;
        P(out, i, j, 0) = two9 * rho * (2 - 3 * u2);
        P(out, i, j, 1) = one18 * rho * (2 + 6 * ux + 9 * ux * ux - 3 * u2);
        P(out, i, j, 2) = one18 * rho * (2 + 6 * uy + 9 * uy * uy - 3 * u2);
        P(out, i, j, 3) = one18 * rho * (2 - 6 * ux + 9 * ux * ux - 3 * u2);
        P(out, i, j, 4) = one18 * rho * (2 - 6 * uy + 9 * uy * uy - 3 * u2);
        P(out, i, j, 5) = one36 * rho * (1 + 3 * (ux + uy) + 9 * ux * uy + 3 * u2);
        P(out, i, j, 6) = one36 * rho * (1 - 3 * (ux - uy) - 9 * ux * uy + 3 * u2);
        P(out, i, j, 7) = one36 * rho * (1 - 3 * (ux + uy) + 9 * ux * uy + 3 * u2);
        P(out, i, j, 8) = one36 * rho * (1 + 3 * (ux - uy) - 9 * ux * uy + 3 * u2);
    }
}

/* DefaultEquilibrium<2>::update_macro (DefaultEquilibrium.hpp:123-155): fluid nodes only. */
static void update_macro(lattice_t* L, const int64_t* nodes, int64_t n)
{
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        const double p0 = P(L->pop, i, j, 0), p1 = P(L->pop, i, j, 1), p2 = P(L->pop, i, j, 2);
        const double p3 = P(L->pop, i, j, 3), p4 = P(L->pop, i, j, 4), p5 = P(L->pop, i, j, 5);
        const double p6 = P(L->pop, i, j, 6), p7 = P(L->pop, i, j, 7), p8 = P(L->pop, i, j, 8);
        const double rho = p0 + p1 + p2 + p3 + p4 + p5 + p6 + p7 + p8;
        const double rhoinv = 1.0 / rho;
        const double ux = rhoinv * (p1 + p5 + p8 - (p3 + p6 + p7));
        const double uy = rhoinv * (p2 + p5 + p6 - (p4 + p7 + p8));
        RHO(i, j) = rho;
        U(i, j, 0) = ux;
        U(i, j, 1) = uy;
    }
}

/* BGKCollisionPolicy<2>::collide / collide_open_boundary (BGKCollision.hpp:119-155, 201-237). */
static void collide_bgk(lattice_t* L, const int64_t* nodes, int64_t n, double tau)
{
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        const double t = 1.0 / tau;
        const double o_m_t = 1.0 - t;
        for (int k = 0; k < 9; ++k) P(L->post, i, j, k) = o_m_t * P(L->pop, i, j, k) + t * P(L->eq, i, j, k);
    }
}

/* TRTCollisionPolicy<2>::collide / collide_open_boundary (TRTCollision.hpp:146-191, 233-278). */
static void collide_trt(lattice_t* L, const int64_t* nodes, int64_t n, double tau_even, double tau_odd)
{
    static const int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        P(L->post, i, j, 0) = P(L->pop, i, j, 0) - (1.0 / tau_even) * (P(L->pop, i, j, 0) - P(L->eq, i, j, 0));
        for (int k = 1; k < 9; ++k) {
            const int b = opp[k];
            P(L->post, i, j, k) = P(L->pop, i, j, k) -
                0.5 * (1.0 / tau_even) * (P(L->pop, i, j, k) + P(L->pop, i, j, b) - P(L->eq, i, j, k) - P(L->eq, i, j, b)) -
                0.5 * (1.0 / tau_odd) * (P(L->pop, i, j, k) - P(L->pop, i, j, b) - P(L->eq, i, j, k) + P(L->eq, i, j, b));
        }
    }
}

/* Direction vectors as (di, dj) of the reference's push (BGKCollision.hpp:179-187). */
static const int DI[9] = {0, 0, -1, 0, 1, -1, -1, 1, 1};
static const int DJ[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};

/* stream (BGKCollision.hpp:164-189, TRTCollision.hpp:200-221): unconditional push. */
static void stream_fluid(lattice_t* L, const int64_t* nodes, int64_t n)
{
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        for (int k = 0; k < 9; ++k) P(L->pop, i + DI[k], j + DJ[k], k) = P(L->post, i, j, k);
    }
}

/* stream_open_boundary (BGKCollision.hpp:246-304, TRTCollision.hpp:287-343): push
   only to neighbours inside the lattice. */
static void stream_open(lattice_t* L, const int64_t* nodes, int64_t n)
{
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        for (int k = 0; k < 9; ++k) {
            const int64_t ni = i + DI[k], nj = j + DJ[k];
            if (ni < 0 || nj < 0 || ni >= L->R || nj >= L->C) continue;
            P(L->pop, ni, nj, k) = P(L->post, i, j, k);
        }
    }
}

/* BounceBackPolicy<2>::update_boundaries on wall nodes (BounceBackPolicy.hpp:68-133):
   the wall node sends every in-lattice direction back, reversed. */
static void bounce_walls(lattice_t* L, const int64_t* nodes, int64_t n)
{
    static const int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        double p[9];
        for (int k = 0; k < 9; ++k) p[k] = P(L->pop, i, j, k);
        /* same statement order as the reference: 3,4,1,2,7,8,5,6 receive p1..p8 */
        for (int s = 1; s < 9; ++s) {
            const int k = opp[s];
            const int64_t ni = i + DI[k], nj = j + DJ[k];
            if (ni < 0 || nj < 0 || ni >= L->R || nj >= L->C) continue;
            P(L->pop, ni, nj, k) = p[s];
        }
    }
}

/* BounceBackPolicy<2>::update_boundaries on obstacle nodes (BounceBackPolicy.hpp:143-187):
   for each set bit k, pop(x + c_k, k) = pop(x, opp(k)). */
static void bounce_obstacles(lattice_t* L, const int64_t* nodes, const uint16_t* dirs, int64_t n)
{
    static const int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        for (int k = 1; k < 9; ++k)
            if (dirs[q] & (1u << k)) P(L->pop, i + DI[k], j + DJ[k], k) = P(L->pop, i, j, opp[k]);
    }
}

/* PSBounceBackPolicy<2>::update_boundaries on obstacle nodes
   (PSBounceBackPolicy.hpp:177-293): for each set bit k the fluid neighbour
   x + c_k receives a mix of the relaxed reflection and its own previous value,
   with e from the neighbour's global_rho/global_u and the obstacle's global_rho
   (1, never updated for obstacles). */
static void ps_obstacles(lattice_t* L, const int64_t* nodes, const uint16_t* dirs, const double* bvals, int64_t n,
                         double tau)
{
    const double two9 = (2.0 / 9.0);
    const double one18 = (1.0 / 18.0);
    const double one36 = (1.0 / 36.0);
    (void)two9;
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        const double b = bvals ? bvals[q] : 1.0;
        const double p1 = P(L->pop, i, j, 1), p2 = P(L->pop, i, j, 2), p3 = P(L->pop, i, j, 3);
        const double p4 = P(L->pop, i, j, 4), p5 = P(L->pop, i, j, 5), p6 = P(L->pop, i, j, 6);
        const double p7 = P(L->pop, i, j, 7), p8 = P(L->pop, i, j, 8);
        const double t = 1.0 / tau;
        const double rx = RHO(i, j);
        double rho, ux, uy, u2, ea, eb;
#define MAC(ii, jj) rho = RHO(ii, jj); ux = U(ii, jj, 0); uy = U(ii, jj, 1); u2 = ux * ux + uy * uy
        if (dirs[q] & (1u << 1)) {
            MAC(i, j + 1);
            ea = one18 * rho * (2 + 6 * ux + 9 * ux * ux - 3 * u2);  /* e1 */
            eb = one18 * rho * (2 - 6 * ux + 9 * ux * ux - 3 * u2);  /* e3 */
            P(L->pop, i, j + 1, 1) = p3 - (1.0 - b) * (p3 - eb) * t + b * ((P(L->pop, i, j + 1, 1) - ea) - (p3 - 2 * one18 * rx));
        }
        if (dirs[q] & (1u << 2)) {
            MAC(i - 1, j);
            ea = one18 * rho * (2 + 6 * uy + 9 * uy * uy - 3 * u2);  /* e2 */
            eb = one18 * rho * (2 - 6 * uy + 9 * uy * uy - 3 * u2);  /* e4 */
            P(L->pop, i - 1, j, 2) = p4 - (1.0 - b) * (p4 - eb) * t + b * ((P(L->pop, i - 1, j, 2) - ea) - (p4 - 2 * one18 * rx));
        }
        if (dirs[q] & (1u << 3)) {
            MAC(i, j - 1);
            ea = one18 * rho * (2 + 6 * ux + 9 * ux * ux - 3 * u2);  /* e1 */
            eb = one18 * rho * (2 - 6 * ux + 9 * ux * ux - 3 * u2);  /* e3 */
            P(L->pop, i, j - 1, 3) = p1 - (1.0 - b) * (p1 - ea) * t + b * ((P(L->pop, i, j - 1, 3) - eb) - (p1 - 2 * one18 * rx));
        }
        if (dirs[q] & (1u << 4)) {
            MAC(i + 1, j);
            ea = one18 * rho * (2 + 6 * uy + 9 * uy * uy - 3 * u2);  /* e2 */
            eb = one18 * rho * (2 - 6 * uy + 9 * uy * uy - 3 * u2);  /* e4 */
            P(L->pop, i + 1, j, 4) = p2 - (1.0 - b) * (p2 - ea) * t + b * ((P(L->pop, i + 1, j, 4) - eb) - (p2 - 2 * one18 * rx));
        }
        if (dirs[q] & (1u << 5)) {
            MAC(i - 1, j + 1);
            ea = one36 * rho * (1 + 3 * (ux + uy) + 9 * ux * uy + 3 * u2);  /* e5 */
            eb = one36 * rho * (1 - 3 * (ux + uy) + 9 * ux * uy + 3 * u2);  /* e7 */
            P(L->pop, i - 1, j + 1, 5) = p7 - (1.0 - b) * (p7 - eb) * t + b * ((P(L->pop, i - 1, j + 1, 5) - ea) - (p7 - one36 * rx));
        }
        if (dirs[q] & (1u << 6)) {
            MAC(i - 1, j - 1);
            ea = one36 * rho * (1 - 3 * (ux - uy) - 9 * ux * uy + 3 * u2);  /* e6 */
            eb = one36 * rho * (1 + 3 * (ux - uy) - 9 * ux * uy + 3 * u2);  /* e8 */
            P(L->pop, i - 1, j - 1, 6) = p8 - (1.0 - b) * (p8 - eb) * t + b * ((P(L->pop, i - 1, j - 1, 6) - ea) - (p8 - one36 * rx));
        }
        if (dirs[q] & (1u << 7)) {
            MAC(i + 1, j - 1);
            ea = one36 * rho * (1 + 3 * (ux + uy) + 9 * ux * uy + 3 * u2);  /* e5 */
            eb = one36 * rho * (1 - 3 * (ux + uy) + 9 * ux * uy + 3 * u2);  /* e7 */
            P(L->pop, i + 1, j - 1, 7) = p5 - (1.0 - b) * (p5 - ea) * t + b * ((P(L->pop, i + 1, j - 1, 7) - eb) - (p5 - one36 * rx));
        }
        if (dirs[q] & (1u << 8)) {
            MAC(i + 1, j + 1);
            ea = one36 * rho * (1 - 3 * (ux - uy) - 9 * ux * uy + 3 * u2);  /* e6 */
            eb = one36 * rho * (1 + 3 * (ux - uy) - 9 * ux * uy + 3 * u2);  /* e8 */
            P(L->pop, i + 1, j + 1, 8) = p6 - (1.0 - b) * (p6 - ea) * t + b * ((P(L->pop, i + 1, j + 1, 8) - eb) - (p6 - one36 * rx));
        }
#undef MAC
    }
}

/* ZouHePolicy<2>::update_boundaries (ZouHePolicy.hpp:58-123).  global_u is the
   by-value copy the policy receives; the density it computes is stored into a
   copy and lost, so it is not kept here. */
static void zou_he_velocity(lattice_t* L, const int64_t* nodes, const int32_t* side, int64_t n)
{
    const double two_thirds = 2.0 / 3.0;
    const double one_sixth = 1.0 / 6.0;
    const double one_half = 0.5;
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        double* pp = L->pop;
        double rho, ru, rv;
#define p(k) P(pp, i, j, k)
        switch (side[q]) {
        case BT_TOP:
            rho = (p(0) + p(1) + p(3) + 2.0 * (p(2) + p(5) + p(6))) / (1.0 + U(i, j, 1));
            ru = rho * U(i, j, 0);
            rv = rho * U(i, j, 1);
            p(4) = p(2) - two_thirds * rv;
            p(7) = p(5) - one_sixth * rv - one_half * ru + one_half * (p(1) - p(3));
            p(8) = p(6) - one_sixth * rv + one_half * ru - one_half * (p(1) - p(3));
            break;
        case BT_BOTTOM:
            rho = (p(0) + p(1) + p(3) + 2.0 * (p(4) + p(7) + p(8))) / (1.0 - U(i, j, 1));
            ru = rho * U(i, j, 0);
            rv = rho * U(i, j, 1);
            p(2) = p(4) + two_thirds * rv;
            p(5) = p(7) + one_sixth * rv + one_half * ru - one_half * (p(1) - p(3));
            p(6) = p(8) + one_sixth * rv - one_half * ru + one_half * (p(1) - p(3));
            break;
        case BT_LEFT:
            rho = (p(0) + p(2) + p(4) + 2.0 * (p(3) + p(7) + p(6))) / (1.0 - U(i, j, 0));
            ru = rho * U(i, j, 0);
            rv = rho * U(i, j, 1);
            p(1) = p(3) + two_thirds * ru;
            p(5) = p(7) + one_sixth * ru + one_half * rv - one_half * (p(2) - p(4));
            p(8) = p(6) + one_sixth * ru - one_half * rv + one_half * (p(2) - p(4));
            break;
        case BT_RIGHT:
            rho = (p(0) + p(2) + p(4) + 2.0 * (p(1) + p(5) + p(8))) / (1.0 + U(i, j, 0));
            ru = rho * U(i, j, 0);
            rv = rho * U(i, j, 1);
            p(3) = p(1) - two_thirds * ru;
            p(7) = p(5) - one_sixth * ru - one_half * rv + one_half * (p(2) - p(4));
            p(6) = p(8) - one_sixth * ru + one_half * rv - one_half * (p(2) - p(4));
            break;
        default:
            break; /* corners and NONE: untouched */
        }
#undef p
    }
}

/* Zou-He pressure closure (extension; ZouHePressurePolicy.hpp close_node): the
   computed velocity goes to `cache` (R*C*2), read back at the next update_nodes. */
static void zou_he_pressure(lattice_t* L, const int64_t* nodes, const int32_t* side, int64_t n, double rho0,
                            double ut, double* cache)
{
    const double two_thirds = 2.0 / 3.0;
    const double one_sixth = 1.0 / 6.0;
    const double one_half = 0.5;
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        double p[9];
        for (int k = 0; k < 9; ++k) p[k] = P(L->pop, i, j, k);
        double ux, uy, ru, rv, s;
        switch (side[q]) {
        case BT_TOP:
            s = ((p[0] + p[1]) + p[3]) + 2.0 * ((p[2] + p[5]) + p[6]);
            ux = ut;
            uy = s / rho0 - 1.0;
            ru = rho0 * ux;
            rv = rho0 * uy;
            p[4] = p[2] - two_thirds * rv;
            p[7] = p[5] - one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
            p[8] = p[6] - one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
            break;
        case BT_BOTTOM:
            s = ((p[0] + p[1]) + p[3]) + 2.0 * ((p[4] + p[7]) + p[8]);
            ux = ut;
            uy = 1.0 - s / rho0;
            ru = rho0 * ux;
            rv = rho0 * uy;
            p[2] = p[4] + two_thirds * rv;
            p[5] = p[7] + one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
            p[6] = p[8] + one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
            break;
        case BT_LEFT:
            s = ((p[0] + p[2]) + p[4]) + 2.0 * ((p[3] + p[7]) + p[6]);
            ux = 1.0 - s / rho0;
            uy = ut;
            ru = rho0 * ux;
            rv = rho0 * uy;
            p[1] = p[3] + two_thirds * ru;
            p[5] = p[7] + one_sixth * ru + one_half * rv - one_half * (p[2] - p[4]);
            p[8] = p[6] + one_sixth * ru - one_half * rv + one_half * (p[2] - p[4]);
            break;
        case BT_RIGHT:
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
            continue;
        }
        for (int k = 0; k < 9; ++k) P(L->pop, i, j, k) = p[k];
        cache[i + L->R * j] = ux;
        cache[i + L->R * (j + L->C)] = uy;
    }
}

/* VelocityInitializer<2>::update_nodes (InletOutletInitializer.hpp:90-129).
   Pressure-policy nodes (extension) take the velocity their closure computed
   and collide with the prescribed density rho_out; through the reference's own
   Lattice the density of an open node stays 1 (global_rho is never written for
   it), which is the same thing for rho_out == 1. */
static void update_nodes(lattice_t* L, const int64_t* nodes, int64_t n, const double* vals, int bc,
                         const double* cache, double rho_out)
{
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = nodes[2 * q], j = nodes[2 * q + 1];
        if (bc == LBO_BC_ZH_PRESSURE) {
            RHO(i, j) = rho_out;
            U(i, j, 0) = cache[i + L->R * j];
            U(i, j, 1) = cache[i + L->R * (j + L->C)];
        } else {
            U(i, j, 0) = vals[2 * q];
            U(i, j, 1) = vals[2 * q + 1];
        }
    }
}

void lbo_flow_properties(int64_t rows, int64_t cols, const double* densities, const int64_t* pts,
                         const uint16_t* dirs, int64_t n, double out[2])
{
    /* FlowAnalyzer<2>::compute_flow_properties (FlowAnalyzer.hpp:348-451) */
    const int64_t R = rows, C = cols;
#define D(i, j, k) densities[(i) + R * ((j) + C * (int64_t)(k))]
    double total_lift = 0., total_drag = 0.;
    for (int64_t q = 0; q < n; ++q) {
        const int64_t i = pts[2 * q], j = pts[2 * q + 1];
        const unsigned b = dirs[q];
        double local_lift = 0., local_drag = 0.;
        if (b & (1u << 1)) local_drag -= D(i, j + 1, 3);
        if (b & (1u << 2)) local_lift -= D(i - 1, j, 4);
        if (b & (1u << 3)) local_drag += D(i, j - 1, 1);
        if (b & (1u << 4)) local_lift += D(i + 1, j, 2);
        if (b & (1u << 5)) {
            local_drag -= (D(i - 1, j + 1, 7)) * sqrt(2) / 2.0;
            local_lift -= (D(i - 1, j + 1, 7)) * sqrt(2) / 2.0;
        }
        if (b & (1u << 6)) {
            local_drag += (D(i - 1, j - 1, 8)) * sqrt(2) / 2.0;
            local_lift -= (D(i - 1, j - 1, 8)) * sqrt(2) / 2.0;
        }
        if (b & (1u << 7)) {
            local_drag += (D(i + 1, j - 1, 5)) * sqrt(2) / 2.0;
            local_lift += (D(i + 1, j - 1, 5)) * sqrt(2) / 2.0;
        }
        if (b & (1u << 8)) {
            local_drag -= (D(i + 1, j + 1, 6)) * sqrt(2) / 2.0;
            local_lift += (D(i + 1, j + 1, 6)) * sqrt(2) / 2.0;
        }
        total_drag += local_drag;
        total_lift += local_lift;
    }
#undef D
    (void)C;
    out[0] = total_lift;
    out[1] = total_drag;
}

static int check_nodes(const int64_t* nodes, int64_t n, int64_t R, int64_t C)
{
    for (int64_t q = 0; q < n; ++q)
        if (nodes[2 * q] < 0 || nodes[2 * q] >= R || nodes[2 * q + 1] < 0 || nodes[2 * q + 1] >= C) return -1;
    return 0;
}

int lbo_run(const lbo_problem* pr, int64_t steps, const double* open_u, int64_t table_rows,
            int64_t analyzer_every, const int64_t* analyzer_pts, const uint16_t* analyzer_dirs,
            int64_t analyzer_n, double* lift_drag, int64_t* n_lift_drag,
            double* populations, double* u, double* rho, double* fstar)
{
    if (!pr || pr->rows <= 0 || pr->cols <= 0 || steps < 0) return -1;
    const int64_t R = pr->rows, C = pr->cols, N = R * C;
    if (check_nodes(pr->fluid, pr->n_fluid, R, C) || check_nodes(pr->wall, pr->n_wall, R, C) ||
        check_nodes(pr->inlet, pr->n_inlet, R, C) || check_nodes(pr->outlet, pr->n_outlet, R, C) ||
        check_nodes(pr->obst, pr->n_obst, R, C))
        return -2;
    /* The reference streams fluid nodes unconditionally (no bounds check); a fluid
       node on the lattice edge would write outside the tensor there.  Refuse it. */
    for (int64_t q = 0; q < pr->n_fluid; ++q) {
        const int64_t i = pr->fluid[2 * q], j = pr->fluid[2 * q + 1];
        if (i == 0 || j == 0 || i == R - 1 || j == C - 1) return -3;
    }
    if ((pr->n_inlet + pr->n_outlet) > 0 && (!open_u || table_rows <= 0)) return -4;

    lattice_t Ls = {R, C, 0, 0, 0, 0, 0};
    lattice_t* L = &Ls;
    L->pop = (double*)calloc((size_t)(N * 9), sizeof(double));
    L->eq = (double*)calloc((size_t)(N * 9), sizeof(double));
    L->post = (double*)calloc((size_t)(N * 9), sizeof(double));
    L->rho = (double*)calloc((size_t)N, sizeof(double));
    L->u = (double*)calloc((size_t)(N * 2), sizeof(double));
    double* cache = (double*)calloc((size_t)(N * 2), sizeof(double));
    if (!L->pop || !L->eq || !L->post || !L->rho || !L->u || !cache) {
        free(L->pop); free(L->eq); free(L->post); free(L->rho); free(L->u); free(cache);
        return -5;
    }
    const int64_t n_open = pr->n_inlet + pr->n_outlet;
    int64_t n_ld = 0;

    /* perform_lbm (Lattice.hpp:288-438) */
    for (int64_t x = 0; x < N; ++x) L->rho[x] = 1.0;                 /* :295 */
    /* global_u already 0 (:296) */
    calc_equilibrium(L, pr->fluid, pr->n_fluid, L->pop);              /* :326-328 */
    calc_equilibrium(L, pr->inlet, pr->n_inlet, L->pop);
    calc_equilibrium(L, pr->outlet, pr->n_outlet, L->pop);
    for (int64_t s = 0; s < steps; ++s) {
        const int64_t row = s < table_rows ? s : table_rows - 1;
        const double* vals = n_open ? open_u + (size_t)(row * n_open * 2) : 0;
        update_nodes(L, pr->inlet, pr->n_inlet, vals, pr->inlet_bc, cache, pr->rho_out);                        /* :351 */
        update_nodes(L, pr->outlet, pr->n_outlet, vals ? vals + 2 * pr->n_inlet : 0, pr->outlet_bc, cache, pr->rho_out);
        update_macro(L, pr->fluid, pr->n_fluid);                                                   /* :357 */
        calc_equilibrium(L, pr->fluid, pr->n_fluid, L->eq);                                        /* :363-365 */
        calc_equilibrium(L, pr->inlet, pr->n_inlet, L->eq);
        calc_equilibrium(L, pr->outlet, pr->n_outlet, L->eq);
        if (pr->collision == LBO_TRT) {                                                            /* :380-382 */
            collide_trt(L, pr->fluid, pr->n_fluid, pr->tau_even, pr->tau_odd);
            collide_trt(L, pr->inlet, pr->n_inlet, pr->tau_even, pr->tau_odd);
            collide_trt(L, pr->outlet, pr->n_outlet, pr->tau_even, pr->tau_odd);
        } else {
            collide_bgk(L, pr->fluid, pr->n_fluid, pr->tau);
            collide_bgk(L, pr->inlet, pr->n_inlet, pr->tau);
            collide_bgk(L, pr->outlet, pr->n_outlet, pr->tau);
        }
        if (analyzer_every > 0 && s > 0 && s % analyzer_every == 0 && lift_drag) {                /* :384-387 */
            lbo_flow_properties(R, C, L->post, analyzer_pts, analyzer_dirs, analyzer_n, lift_drag + 2 * n_ld);
            ++n_ld;
        }
        stream_fluid(L, pr->fluid, pr->n_fluid);                                                   /* :393-395 */
        stream_open(L, pr->inlet, pr->n_inlet);
        stream_open(L, pr->outlet, pr->n_outlet);
        bounce_walls(L, pr->wall, pr->n_wall);                                                     /* :402 */
        if (pr->obstacle_bc == LBO_OBST_PARTIAL)                                                   /* :403 */
            ps_obstacles(L, pr->obst, pr->obst_dirs, pr->obst_b, pr->n_obst, pr->ps_tau);
        else
            bounce_obstacles(L, pr->obst, pr->obst_dirs, pr->n_obst);
        if (pr->inlet_bc == LBO_BC_ZH_VELOCITY)                                                    /* :409 */
            zou_he_velocity(L, pr->inlet, pr->inlet_side, pr->n_inlet);
        else if (pr->inlet_bc == LBO_BC_ZH_PRESSURE)
            zou_he_pressure(L, pr->inlet, pr->inlet_side, pr->n_inlet, pr->rho_out, pr->tangential_u, cache);
        if (pr->outlet_bc == LBO_BC_ZH_VELOCITY)                                                   /* :410 */
            zou_he_velocity(L, pr->outlet, pr->outlet_side, pr->n_outlet);
        else if (pr->outlet_bc == LBO_BC_ZH_PRESSURE)
            zou_he_pressure(L, pr->outlet, pr->outlet_side, pr->n_outlet, pr->rho_out, pr->tangential_u, cache);
    }
    if (n_lift_drag) *n_lift_drag = n_ld;
    if (populations) memcpy(populations, L->pop, sizeof(double) * (size_t)(N * 9));
    if (fstar) memcpy(fstar, L->post, sizeof(double) * (size_t)(N * 9));
    if (u) memcpy(u, L->u, sizeof(double) * (size_t)(N * 2));
    if (rho) memcpy(rho, L->rho, sizeof(double) * (size_t)N);
    free(L->pop); free(L->eq); free(L->post); free(L->rho); free(L->u); free(cache);
    return 0;
}
