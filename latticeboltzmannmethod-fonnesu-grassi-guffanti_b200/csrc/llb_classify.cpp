// Host-side lattice classification: the reference's node vectors from a grid of
// InputNodeType codes, in O(R*C).
//
// Reference behaviour restated (paths relative to the LLALBM project root):
//   * vector order: row index outer, column inner, as TensorLoopAccessor visits
//     the type tensor (utils/readers/LatticeReader.hpp:108-204);
//   * inlets and outlets must lie on the lattice perimeter
//     (verify_lattice_bounds, LatticeReader.hpp:282-297);
//   * their side: identify_node_type (utils/analysis/NodeIdentification.hpp:45-110);
//   * obstacle direction bit k is set iff the node at coords + c_k is fluid, inlet
//     or outlet (identify_obstacle_propagation, :137-211, with its offset ->
//     direction table :145-155), looked up in the grid instead of std::find;
//   * obstacles with no bit set are dropped (eliminate_non_wet_nodes, :229-242).
#include <cstring>

#include "../../include/llalbm_cuda.h"

namespace {

constexpr int DI_[9] = {0, 0, -1, 0, 1, -1, -1, 1, 1};
constexpr int DJ_[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};

// btypes (utils/aliases.hpp:28-38)
enum { NONE = 0, TOP_WALL, RIGHT_WALL, BOTTOM_WALL, LEFT_WALL, RIGHT_TOP_C, RIGHT_BOTTOM_C, LEFT_BOTTOM_C, LEFT_TOP_C };

int side_of(int64_t i, int64_t j, int64_t R, int64_t C) {
    if (i == 0) return j == 0 ? LEFT_TOP_C : (j == C - 1 ? RIGHT_TOP_C : TOP_WALL);
    if (i == R - 1) return j == 0 ? LEFT_BOTTOM_C : (j == C - 1 ? RIGHT_BOTTOM_C : BOTTOM_WALL);
    if (j == 0) return LEFT_WALL;
    if (j == C - 1) return RIGHT_WALL;
    return NONE;
}

bool on_perimeter(int64_t i, int64_t j, int64_t R, int64_t C) { return i == 0 || j == 0 || i == R - 1 || j == C - 1; }

bool is_active_type(uint8_t t) { return t == LLB_NODE_FLUID || t == LLB_NODE_INLET || t == LLB_NODE_OUTLET; }

uint16_t obstacle_bits(const uint8_t* types, int64_t R, int64_t C, int64_t i, int64_t j) {
    uint16_t b = 0;
    for (int k = 1; k < 9; ++k) {
        const int64_t ni = i + DI_[k], nj = j + DJ_[k];
        if (ni < 0 || nj < 0 || ni >= R || nj >= C) continue;
        if (is_active_type(types[ni + R * nj])) b |= static_cast<uint16_t>(1u << k);
    }
    return b;
}

int scan(int64_t R, int64_t C, const uint8_t* types, int64_t counts[5], llb_node_lists* out) {
    if (R <= 0 || C <= 0 || !types) return LLB_E_INVALID;
    int64_t n[5] = {0, 0, 0, 0, 0};
    for (int64_t i = 0; i < R; ++i) {
        for (int64_t j = 0; j < C; ++j) {
            const uint8_t t = types[i + R * j];
            if (t > LLB_NODE_OBSTACLE) return LLB_E_INVALID;
            switch (t) {
            case LLB_NODE_FLUID:
                if (out) { out->fluid_ij[2 * n[0]] = i; out->fluid_ij[2 * n[0] + 1] = j; }
                ++n[0];
                break;
            case LLB_NODE_BOUNDARY:
                if (out) { out->wall_ij[2 * n[1]] = i; out->wall_ij[2 * n[1] + 1] = j; }
                ++n[1];
                break;
            case LLB_NODE_INLET:
            case LLB_NODE_OUTLET: {
                if (!on_perimeter(i, j, R, C)) return LLB_E_GEOMETRY;
                const int slot = t == LLB_NODE_INLET ? 2 : 3;
                if (out) {
                    int64_t* ij = slot == 2 ? out->inlet_ij : out->outlet_ij;
                    int32_t* sd = slot == 2 ? out->inlet_side : out->outlet_side;
                    ij[2 * n[slot]] = i;
                    ij[2 * n[slot] + 1] = j;
                    sd[n[slot]] = side_of(i, j, R, C);
                }
                ++n[slot];
                break;
            }
            case LLB_NODE_OBSTACLE: {
                const uint16_t b = obstacle_bits(types, R, C, i, j);
                if (b == 0) break;  // not wet
                if (out) {
                    out->obstacle_ij[2 * n[4]] = i;
                    out->obstacle_ij[2 * n[4] + 1] = j;
                    out->obstacle_dirs[n[4]] = b;
                }
                ++n[4];
                break;
            }
            default:  // SOLID: in no vector
                break;
            }
        }
    }
    if (counts) std::memcpy(counts, n, sizeof(n));
    return LLB_OK;
}

}  // namespace

extern "C" int llb_classify_count(int64_t rows, int64_t cols, const uint8_t* types, int64_t counts[5]) {
    if (!counts) return LLB_E_INVALID;
    return scan(rows, cols, types, counts, nullptr);
}

extern "C" int llb_classify_fill(int64_t rows, int64_t cols, const uint8_t* types, llb_node_lists* out) {
    if (!out) return LLB_E_INVALID;
    int64_t counts[5];
    int rc = scan(rows, cols, types, counts, nullptr);
    if (rc != LLB_OK) return rc;
    if (counts[0] != out->n_fluid || counts[1] != out->n_wall || counts[2] != out->n_inlet ||
        counts[3] != out->n_outlet || counts[4] != out->n_obstacle)
        return LLB_E_INVALID;
    if ((counts[0] && !out->fluid_ij) || (counts[1] && !out->wall_ij) ||
        (counts[2] && (!out->inlet_ij || !out->inlet_side)) || (counts[3] && (!out->outlet_ij || !out->outlet_side)) ||
        (counts[4] && (!out->obstacle_ij || !out->obstacle_dirs)))
        return LLB_E_INVALID;
    return scan(rows, cols, types, nullptr, out);
}
