// Internal definitions shared by the engine's translation units.
//
// Data layout in HBM (one lattice):
//   populations : 9 planes, plane k at base + k*plane, node (i, j) at j*ld + i
//                 (column-major like the reference's Eigen tensors, row index
//                 fastest; ld = rows rounded up so every column starts on a
//                 256-byte boundary).  Two such buffers (AB) or one (AA).
//   mask        : one byte per node, same (j*ld + i) indexing.
//   open_idx    : int32 per node, index of an inlet/outlet node in the open
//                 value table (read only for open nodes).
//   open_vals   : ring of [cap][n_open] double2 per-step boundary values.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>

namespace llb {

// ---- node mask byte ----------------------------------------------------------
// bits 0-1  class: DEAD (never updated), FLUID, BB (wall or wet obstacle: as a
//           streaming source it bounces the population back), OPEN (inlet/outlet)
// bit  2    PLAIN: all 8 streaming sources of an active node are FLUID or OPEN
// bits 3-5  side of an OPEN node: 0 none/corner, 1 top, 2 right, 3 bottom, 4 left
//           (the reference's btypes TOP_WALL..LEFT_WALL)
// bits 6-7  closure of an OPEN node: 0 Zou-He velocity, 1 none, 2 Zou-He pressure
// Population slots of DEAD nodes always hold the initial value of their
// direction (filled at creation, rewritten only with that value), so a pull
// from a dead source reads the reference's never-written slot as is.
constexpr uint8_t CLS_DEAD = 0, CLS_FLUID = 1, CLS_BB = 2, CLS_OPEN = 3;
constexpr uint8_t MASK_PLAIN = 4;
// Bounce bits, one byte per node beside the mask (active nodes that are not
// PLAIN): bit k - 1 set when the source of direction k (1..8), x - c_k, is a
// wall or obstacle.  Sources outside the lattice (open nodes on the lattice
// edge only; fluid nodes never lie on it) set no bit.
constexpr int SIDE_SHIFT = 3, BC_SHIFT = 6;
constexpr int SIDE_NONE = 0, SIDE_TOP = 1, SIDE_RIGHT = 2, SIDE_BOTTOM = 3, SIDE_LEFT = 4;
constexpr int BC_ZH_VEL = 0, BC_OPEN = 1, BC_ZH_PRES = 2;

__host__ __device__ constexpr uint8_t mask_class(uint8_t m) { return m & 3u; }
__host__ __device__ constexpr int mask_side(uint8_t m) { return (m >> SIDE_SHIFT) & 7; }
__host__ __device__ constexpr int mask_bc(uint8_t m) { return (m >> BC_SHIFT) & 3; }
__host__ __device__ constexpr bool class_active(uint8_t c) { return c == CLS_FLUID || c == CLS_OPEN; }

// The node mask and bounce bytes of a dense lattice (2 bytes per node against
// the 18 populations a node moves) are read again by every step; the
// one-thread-per-node step loads them with an L2 evict_last policy, so the
// population stream does not push them out of L2 between steps and a node's
// first load is an L2 hit.  Measured on B200 (cavity 2048^2, one thread per
// node): FP32 70.1k-71.5k -> 77.0k-77.3k MLUPS, FP64 41.5k-43.0k -> 43.5k-43.8k;
// the same policy on the compacted planes' slot tables (6 bytes per node)
// made no difference on porous lattices and cost the batch's slot kernel 2 %.
__device__ __forceinline__ unsigned long long l2_keep_policy() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint8_t ld_keep(const uint8_t* a, unsigned long long pol) {
    unsigned v;
    asm("ld.global.nc.L2::cache_hint.u8 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return static_cast<uint8_t>(v);
}

// D2Q9 directions as (di, dj) of the reference's push (BGKCollision.hpp:179-187):
// 1 (0,+1) 2 (-1,0) 3 (0,-1) 4 (+1,0) 5 (-1,+1) 6 (-1,-1) 7 (+1,-1) 8 (+1,+1).
// A pull reads direction k from the node at (i - di, j - dj).
__host__ __device__ constexpr int DI(int k) {
    return k == 2 || k == 5 || k == 6 ? -1 : (k == 4 || k == 7 || k == 8 ? 1 : 0);
}
__host__ __device__ constexpr int DJ(int k) {
    return k == 1 || k == 5 || k == 8 ? 1 : (k == 3 || k == 6 || k == 7 ? -1 : 0);
}
// opposite directions 1<->3, 2<->4, 5<->7, 6<->8
__host__ __device__ constexpr int opp(int k) {
    return k == 1 ? 3 : k == 2 ? 4 : k == 3 ? 1 : k == 4 ? 2 : k == 5 ? 7 : k == 6 ? 8 : k == 7 ? 5 : k == 8 ? 6 : 0;
}

// Initial populations of every active node: the reference's equilibrium at
// rho = 1, u = 0 (Lattice.hpp:326-328 with DefaultEquilibrium.hpp:64-76),
// evaluated with the same expressions.  A population slot nobody streams into
// keeps this value for the whole run (DEAD sources, and sources outside the
// lattice of open nodes on its edge).
__host__ __device__ constexpr double w_init(int k) {
    return k == 0 ? (2.0 / 9.0) * 1.0 * (2 - 3 * 0.0)
         : k <= 4 ? (1.0 / 18.0) * 1.0 * (2 + 6 * 0.0 + 9 * 0.0 * 0.0 - 3 * 0.0)
                  : (1.0 / 36.0) * 1.0 * (1 + 3 * (0.0 + 0.0) + 9 * 0.0 * 0.0 + 3 * 0.0);
}
// Lattice weights used by the shifted (f - w) storage forms.
__host__ __device__ constexpr float w_f32(int k) { return k == 0 ? 4.0f / 9.0f : (k <= 4 ? 1.0f / 9.0f : 1.0f / 36.0f); }

// ---- kernel parameters ------------------------------------------------------
constexpr int MAX_BLOCK_Y = 8;  // columns per block of the step kernel, at most

// Bytes of a population plane per entry of the active-sector list.
constexpr int LIST_BYTES = 32;

struct Geometry {
    int rows, cols;     // R, C
    int ld;             // column stride (elements) of populations / mask / open_idx
    long long plane;    // ld * cols
    const uint8_t* __restrict__ mask;
    const uint8_t* __restrict__ bb;       // bounce bits
    // partially saturated obstacles (NULL otherwise): bit k - 1 set when the
    // source of direction k is such an obstacle; its b per node
    const uint8_t* __restrict__ ps;
    const double* __restrict__ psb;
    const int32_t* __restrict__ open_idx;
    // active-sector list of the plain steps (NULL: the one-thread-per-node
    // grid): ids of the 32-byte sectors of a population plane that hold an
    // active node
    const int32_t* __restrict__ sectors;
    const uint8_t* __restrict__ smask;  // mask byte of each listed node (sector order)
    const uint8_t* __restrict__ sbb;    // bounce byte of each listed node
    int n_sectors;
};

// Column-compacted storage of the active nodes (pipeline PIPE_COMPACT).
// Each population plane holds only the fluid and open nodes, column by
// column, rows in order; a column's run starts on a 32-byte boundary (the
// gap before the next column is padding).  Obstacle interiors and dead
// regions take no slot, so a step reads and writes only the bytes of active
// nodes.  Per slot t:
//   info[t]  node mask byte | bounce byte << 8 (padding: 0, dead);
//   nb[t]    fluid nodes: (t - cL) | (cR - t) << 16, where cL / cR is the slot
//            of row i in the left / right column, or of the next active row
//            below it when row i is not active there; then (i - 1, j -+ 1)
//            sits at cL - 1 / cR - 1 and (i + 1, j -+ 1) right after row i's
//            position; (i -+ 1, j) sit at t -+ 1.
//            Open nodes and fluid nodes with a dead source: the dense index
//            j * ld + i (their pull tests every source through seg).
//   seg[j * nseg + s]  (.x) bit r set when row 32 s + r of column j is
//            active, (.y) slot of the first active row at or after row 32 s;
//            the slot of active row i is seg.y + popc(seg.x & (2^(i%32) - 1)).
//   chunk[w] (.x) column, (.y) first active row of 32 consecutive slots of
//            that column; col[j] first slot of column j (col[C] = slots used):
//            the copies between the dense and the compacted planes.
// A FLUID node whose sources include a dead node carries COMPACT_DEAD_SRC in
// its mask byte (bit 3, the side field, unused by fluid nodes).
constexpr uint8_t COMPACT_DEAD_SRC = 8;
struct CompactGeo {
    const uint16_t* __restrict__ info;
    const uint32_t* __restrict__ nb;
    const int2* __restrict__ seg;
    const int2* __restrict__ chunk;
    const int32_t* __restrict__ col;
    int nseg;           // 32-row segments per column
    int n_chunks;
    long long n_slots;  // col[C]
    long long cplane;   // slots per plane (multiple of 256 bytes)
};

struct OpenTable {
    const double2* __restrict__ vals;  // [cap][n_open]
    int n_open;
    int cap;
};

struct Collision {
    int model;          // 0 BGK, 1 TRT
    // BGK: t = 1/tau, omt = 1 - t   (BGKCollision.hpp:142-143)
    double t, omt;
    // TRT: ie = 1/tau_even, he = 0.5*(1/tau_even), ho = 0.5*(1/tau_odd)   (TRTCollision.hpp:155-188)
    double ie, he, ho;
    // the same rates rounded to FP32 for the shifted storage forms
    float tf, omtf, ief, hef, hof;
    // partially saturated obstacles: 1/tau of PSBounceBackPolicy (PSBounceBackPolicy.hpp:200)
    double ps_t;
};

struct MacroOut {
    double* rho;        // (R, C) dense, column-major
    double* u;          // (R, C, 2) dense
};

// Step index of a launch: t = (tbase ? *tbase : 0) + t_off.  Direct launches
// pass the absolute step in t_off; graph replays pass the step's offset inside
// the graph and the host sets *tbase before each replay.
struct StepSync {
    const long long* tbase;
    long long t_off;
    unsigned* flags;    // bit 0: non-finite density seen
    // polls of a pipelined kernel's mbarrier waits for its stages before it
    // gives up (the drain of its own copies in flight always waits the full
    // DEFAULT_WAIT_LIMIT)
    long long wait_limit;
};
constexpr long long DEFAULT_WAIT_LIMIT = 1LL << 24;

}  // namespace llb
