// Per-storage arithmetic of one lattice node, and the kernel skeletons shared by
// all storage forms.
//
//   ModelF64   FP64 populations; every expression is the reference's own, in the
//              reference's association order (its translation unit is compiled
//              with --fmad=false, so no multiply-add is contracted).
//   ModelShift<T>  populations stored as f_k - w_k in T (float or __half);
//              moments, closures and collision in FP32 on the shifted values,
//              multiply-adds written out as __fmaf_rn (its translation unit is
//              also compiled with --fmad=false).
#pragma once

#include "llb_internal.cuh"

namespace llb {

// ============================================================================
// FP64: the reference's expressions
// ============================================================================
struct ModelF64 {
    using T = double;
    using R = double;

    static __device__ __forceinline__ R keep(int k) { return w_init(k); }
    static __device__ __forceinline__ R load(const T* p) { return *p; }
    static __device__ __forceinline__ void store(T* p, R v) { *p = v; }
    static __device__ __forceinline__ double to_f64(R v, int) { return v; }

    // DefaultEquilibrium<2>::update_macro (DefaultEquilibrium.hpp:135-153)
    static __device__ __forceinline__ void moments(const R* p, R& rho, R& ux, R& uy) {
        rho = p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7] + p[8];
        const double rhoinv = 1.0 / rho;
        ux = rhoinv * (p[1] + p[5] + p[8] - (p[3] + p[6] + p[7]));
        uy = rhoinv * (p[2] + p[5] + p[6] - (p[4] + p[7] + p[8]));
    }

    // ZouHePolicy<2>::update_boundaries (ZouHePolicy.hpp:70-118); ux, uy are the
    // node's global_u at the time of the call.
    static __device__ __forceinline__ void closure_velocity(R* p, int side, double ux, double uy) {
        constexpr double two_thirds = 2.0 / 3.0;
        constexpr double one_sixth = 1.0 / 6.0;
        constexpr double one_half = 0.5;
        double rho, ru, rv;
        switch (side) {
        case SIDE_TOP:
            rho = (p[0] + p[1] + p[3] + 2.0 * (p[2] + p[5] + p[6])) / (1.0 + uy);
            ru = rho * ux;
            rv = rho * uy;
            p[4] = p[2] - two_thirds * rv;
            p[7] = p[5] - one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
            p[8] = p[6] - one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
            break;
        case SIDE_BOTTOM:
            rho = (p[0] + p[1] + p[3] + 2.0 * (p[4] + p[7] + p[8])) / (1.0 - uy);
            ru = rho * ux;
            rv = rho * uy;
            p[2] = p[4] + two_thirds * rv;
            p[5] = p[7] + one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
            p[6] = p[8] + one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
            break;
        case SIDE_LEFT:
            rho = (p[0] + p[2] + p[4] + 2.0 * (p[3] + p[7] + p[6])) / (1.0 - ux);
            ru = rho * ux;
            rv = rho * uy;
            p[1] = p[3] + two_thirds * ru;
            p[5] = p[7] + one_sixth * ru + one_half * rv - one_half * (p[2] - p[4]);
            p[8] = p[6] + one_sixth * ru - one_half * rv + one_half * (p[2] - p[4]);
            break;
        case SIDE_RIGHT:
            rho = (p[0] + p[2] + p[4] + 2.0 * (p[1] + p[5] + p[8])) / (1.0 + ux);
            ru = rho * ux;
            rv = rho * uy;
            p[3] = p[1] - two_thirds * ru;
            p[7] = p[5] - one_sixth * ru - one_half * rv + one_half * (p[2] - p[4]);
            p[6] = p[8] - one_sixth * ru + one_half * rv - one_half * (p[2] - p[4]);
            break;
        default:
            break;  // corners: no closure
        }
    }

    // Zou-He pressure closure (ZouHePressurePolicy.hpp close_node); returns the
    // velocity it implies.  Corners: untouched, velocity (0, 0).
    static __device__ __forceinline__ void closure_pressure(R* p, int side, double rho0, double ut, double& ux,
                                                            double& uy) {
        constexpr double two_thirds = 2.0 / 3.0;
        constexpr double one_sixth = 1.0 / 6.0;
        constexpr double one_half = 0.5;
        double ru, rv, s;
        switch (side) {
        case SIDE_TOP:
            s = ((p[0] + p[1]) + p[3]) + 2.0 * ((p[2] + p[5]) + p[6]);
            ux = ut;
            uy = s / rho0 - 1.0;
            ru = rho0 * ux;
            rv = rho0 * uy;
            p[4] = p[2] - two_thirds * rv;
            p[7] = p[5] - one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
            p[8] = p[6] - one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
            break;
        case SIDE_BOTTOM:
            s = ((p[0] + p[1]) + p[3]) + 2.0 * ((p[4] + p[7]) + p[8]);
            ux = ut;
            uy = 1.0 - s / rho0;
            ru = rho0 * ux;
            rv = rho0 * uy;
            p[2] = p[4] + two_thirds * rv;
            p[5] = p[7] + one_sixth * rv + one_half * ru - one_half * (p[1] - p[3]);
            p[6] = p[8] + one_sixth * rv - one_half * ru + one_half * (p[1] - p[3]);
            break;
        case SIDE_LEFT:
            s = ((p[0] + p[2]) + p[4]) + 2.0 * ((p[3] + p[7]) + p[6]);
            ux = 1.0 - s / rho0;
            uy = ut;
            ru = rho0 * ux;
            rv = rho0 * uy;
            p[1] = p[3] + two_thirds * ru;
            p[5] = p[7] + one_sixth * ru + one_half * rv - one_half * (p[2] - p[4]);
            p[8] = p[6] + one_sixth * ru - one_half * rv + one_half * (p[2] - p[4]);
            break;
        case SIDE_RIGHT:
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
            ux = 0.0;
            uy = 0.0;
            break;
        }
    }

    // calc_equilibrium (DefaultEquilibrium.hpp:64-76) followed by the collision,
    // BGK (BGKCollision.hpp:142-153) or TRT (TRTCollision.hpp:155-188), in place.
    template <int COLL>
    static __device__ __forceinline__ void collide(R* p, double rho, double ux, double uy, const Collision& c) {
        constexpr double two9 = (2.0 / 9.0);
        constexpr double one18 = (1.0 / 18.0);
        constexpr double one36 = (1.0 / 36.0);
        const double u2 = ux * ux + uy * uy;
        double e[9];
        e[0] = two9 * rho * (2 - 3 * u2);
        e[1] = one18 * rho * (2 + 6 * ux + 9 * ux * ux - 3 * u2);
        e[2] = one18 * rho * (2 + 6 * uy + 9 * uy * uy - 3 * u2);
        e[3] = one18 * rho * (2 - 6 * ux + 9 * ux * ux - 3 * u2);
        e[4] = one18 * rho * (2 - 6 * uy + 9 * uy * uy - 3 * u2);
        e[5] = one36 * rho * (1 + 3 * (ux + uy) + 9 * ux * uy + 3 * u2);
        e[6] = one36 * rho * (1 - 3 * (ux - uy) - 9 * ux * uy + 3 * u2);
        e[7] = one36 * rho * (1 - 3 * (ux + uy) + 9 * ux * uy + 3 * u2);
        e[8] = one36 * rho * (1 + 3 * (ux - uy) - 9 * ux * uy + 3 * u2);
        if (COLL == 0) {
#pragma unroll
            for (int k = 0; k < 9; ++k) p[k] = c.omt * p[k] + c.t * e[k];
        } else {
            double q[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) q[k] = p[k];
            p[0] = q[0] - c.ie * (q[0] - e[0]);
#pragma unroll
            for (int k = 1; k < 9; ++k) {
                const int b = opp(k);
                p[k] = q[k] - c.he * (q[k] + q[b] - e[k] - e[b]) - c.ho * (q[k] - q[b] - e[k] + e[b]);
            }
        }
    }

    static __device__ __forceinline__ double rho_f64(R rho) { return rho; }
    static __device__ __forceinline__ bool finite(R rho) { return isfinite(rho); }
    static __device__ __forceinline__ R from_f64(double v) { return v; }
};

// ============================================================================
// Shifted low-precision storage: g_k = f_k - w_k, arithmetic in FP32.
// The closures are unchanged in g because opposite directions share weights;
// only the density sums carry the constant (sum of the weights involved = 1).
// ============================================================================
template <typename TS>
struct ModelShift {
    using T = TS;
    using R = float;

    static __device__ __forceinline__ R keep(int) { return 0.0f; }
    static __device__ __forceinline__ R load(const T* p) {
        if constexpr (sizeof(T) == 2) return __half2float(*reinterpret_cast<const __half*>(p));
        else return *p;
    }
    static __device__ __forceinline__ void store(T* p, R v) {
        if constexpr (sizeof(T) == 2) *reinterpret_cast<__half*>(p) = __float2half_rn(v);
        else *p = v;
    }
    static __device__ __forceinline__ double to_f64(R v, int k) { return static_cast<double>(v) + w_init(k); }

    // returns rho - 1 in rho (kept small for precision)
    static __device__ __forceinline__ void moments(const R* g, R& drho, R& ux, R& uy) {
        drho = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7])) + g[8];
        const R inv = 1.0f / (1.0f + drho);
        ux = inv * ((g[1] + g[5] + g[8]) - (g[3] + g[6] + g[7]));
        uy = inv * ((g[2] + g[5] + g[6]) - (g[4] + g[7] + g[8]));
    }

    static __device__ __forceinline__ void close(R* g, int side, R ru, R rv) {
        constexpr R two_thirds = 2.0f / 3.0f, one_sixth = 1.0f / 6.0f, one_half = 0.5f;
        // multiply-adds written out (__fmaf_rn): the translation unit is built
        // without automatic contraction, so every kernel rounds alike
        switch (side) {
        case SIDE_TOP:
            g[4] = __fmaf_rn(-two_thirds, rv, g[2]);
            g[7] = __fmaf_rn(one_half, g[1] - g[3], __fmaf_rn(-one_half, ru, __fmaf_rn(-one_sixth, rv, g[5])));
            g[8] = __fmaf_rn(-one_half, g[1] - g[3], __fmaf_rn(one_half, ru, __fmaf_rn(-one_sixth, rv, g[6])));
            break;
        case SIDE_BOTTOM:
            g[2] = __fmaf_rn(two_thirds, rv, g[4]);
            g[5] = __fmaf_rn(-one_half, g[1] - g[3], __fmaf_rn(one_half, ru, __fmaf_rn(one_sixth, rv, g[7])));
            g[6] = __fmaf_rn(one_half, g[1] - g[3], __fmaf_rn(-one_half, ru, __fmaf_rn(one_sixth, rv, g[8])));
            break;
        case SIDE_LEFT:
            g[1] = __fmaf_rn(two_thirds, ru, g[3]);
            g[5] = __fmaf_rn(-one_half, g[2] - g[4], __fmaf_rn(one_half, rv, __fmaf_rn(one_sixth, ru, g[7])));
            g[8] = __fmaf_rn(one_half, g[2] - g[4], __fmaf_rn(-one_half, rv, __fmaf_rn(one_sixth, ru, g[6])));
            break;
        case SIDE_RIGHT:
            g[3] = __fmaf_rn(-two_thirds, ru, g[1]);
            g[7] = __fmaf_rn(one_half, g[2] - g[4], __fmaf_rn(-one_half, rv, __fmaf_rn(-one_sixth, ru, g[5])));
            g[6] = __fmaf_rn(-one_half, g[2] - g[4], __fmaf_rn(one_half, rv, __fmaf_rn(-one_sixth, ru, g[8])));
            break;
        default:
            break;
        }
    }

    // sum of the known populations' shifted values as the Zou-He density uses them
    static __device__ __forceinline__ R known_sum(const R* g, int side) {
        switch (side) {
        case SIDE_TOP: return __fmaf_rn(2.0f, g[2] + g[5] + g[6], g[0] + g[1] + g[3]);
        case SIDE_BOTTOM: return __fmaf_rn(2.0f, g[4] + g[7] + g[8], g[0] + g[1] + g[3]);
        case SIDE_LEFT: return __fmaf_rn(2.0f, g[3] + g[7] + g[6], g[0] + g[2] + g[4]);
        case SIDE_RIGHT: return __fmaf_rn(2.0f, g[1] + g[5] + g[8], g[0] + g[2] + g[4]);
        default: return 0.0f;
        }
    }

    static __device__ __forceinline__ void closure_velocity(R* g, int side, double ux_d, double uy_d) {
        if (side < SIDE_TOP || side > SIDE_LEFT) return;
        const R ux = static_cast<R>(ux_d), uy = static_cast<R>(uy_d);
        const R s = 1.0f + known_sum(g, side);
        const R un = side == SIDE_TOP ? uy : side == SIDE_BOTTOM ? -uy : side == SIDE_LEFT ? -ux : ux;
        const R rho = s / (1.0f + un);
        close(g, side, rho * ux, rho * uy);
    }

    static __device__ __forceinline__ void closure_pressure(R* g, int side, double rho0_d, double ut_d, double& ux,
                                                            double& uy) {
        if (side < SIDE_TOP || side > SIDE_LEFT) { ux = 0.0; uy = 0.0; return; }
        const R rho0 = static_cast<R>(rho0_d), ut = static_cast<R>(ut_d);
        // s / rho0 - 1 written as (sum_known_shifted - (rho0 - 1)) / rho0
        const R un = (known_sum(g, side) - (rho0 - 1.0f)) / rho0;
        R vx, vy;
        if (side == SIDE_TOP) { vx = ut; vy = un; }
        else if (side == SIDE_BOTTOM) { vx = ut; vy = -un; }
        else if (side == SIDE_LEFT) { vx = -un; vy = ut; }
        else { vx = un; vy = ut; }
        close(g, side, rho0 * vx, rho0 * vy);
        ux = vx;
        uy = vy;
    }

    // shifted equilibrium g_eq = w_k * (drho + rho*(3cu + 4.5cu^2 - 1.5u^2)), then
    // BGK or TRT on the shifted values (the shifts cancel in both operators).
    // Opposite directions k, opp(k) share w_k and cu^2 and differ in the sign
    // of cu, so each pair is computed once: g_eq = w (even +- odd).
    template <int COLL>
    static __device__ __forceinline__ void collide(R* g, R drho, R ux, R uy, const Collision& c) {
        // multiply-adds written out (__fmaf_rn): the translation unit is built
        // without automatic contraction, so every kernel rounds alike
        const R rho = 1.0f + drho;
        const R u2 = 1.5f * __fmaf_rn(ux, ux, uy * uy);
        const R e0 = w_f32(0) * __fmaf_rn(-rho, u2, drho);
        // pairs (1,3), (2,4), (5,7), (6,8): cu of the first direction of each pair
        // (DJ, DI are 0 or +-1, so cu is a sum or difference of ux and uy)
        constexpr int first[4] = {1, 2, 5, 6};
        R ev[4], od[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int k = first[p];
            const R cu = static_cast<R>(DJ(k)) * ux - static_cast<R>(DI(k)) * uy;
            ev[p] = w_f32(k) * __fmaf_rn(rho, __fmaf_rn(4.5f * cu, cu, -u2), drho);
            od[p] = w_f32(k) * (rho * (3.0f * cu));
        }
        if (COLL == 0) {
            const R t = c.tf, omt = c.omtf;
            g[0] = __fmaf_rn(omt, g[0], t * e0);
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const int k = first[p], b = opp(k);
                g[k] = __fmaf_rn(omt, g[k], t * (ev[p] + od[p]));
                g[b] = __fmaf_rn(omt, g[b], t * (ev[p] - od[p]));
            }
        } else {
            const R ie = c.ief, he = c.hef, ho = c.hof;
            g[0] = __fmaf_rn(-ie, g[0] - e0, g[0]);
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const int k = first[p], b = opp(k);
                // symmetric and antisymmetric non-equilibrium parts of the pair
                const R sym = __fmaf_rn(-2.0f, ev[p], g[k] + g[b]);
                const R asym = __fmaf_rn(-2.0f, od[p], g[k] - g[b]);
                const R qk = g[k], qb = g[b];
                g[k] = __fmaf_rn(-ho, asym, __fmaf_rn(-he, sym, qk));
                g[b] = __fmaf_rn(ho, asym, __fmaf_rn(-he, sym, qb));
            }
        }
    }

    static __device__ __forceinline__ double rho_f64(R drho) { return 1.0 + static_cast<double>(drho); }
    static __device__ __forceinline__ bool finite(R drho) { return isfinite(drho); }
    static __device__ __forceinline__ R from_f64(double v) { return static_cast<R>(v - 1.0); }
};

}  // namespace llb
