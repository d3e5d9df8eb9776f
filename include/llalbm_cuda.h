/*
 * llalbm_cuda.h -- C ABI of libllalbm_cuda.so, the sm_100a (B200) engine behind
 * LLALBM's CUDA parallelization policy.
 *
 * The reference library's plugin boundary is the static interface of a
 * ParallelizationPolicy (llalbm/src/core/parallelization/OMPPolicy.hpp:35-164),
 * called by Lattice<P>::perform_lbm (llalbm/src/core/lattices/Lattice.hpp:288-438)
 * once per policy function per step.  This engine fuses one whole step into one
 * kernel, so its entry points replace groups of those policy calls; each
 * declaration below names the calls it replaces.  Paths are relative to the
 * LLALBM project root.
 *
 * Conventions: plain C types only; every function returns LLB_OK (0) or a
 * negative LLB_E_* status and never throws; a handle is owned by one host
 * thread at a time; distinct handles are independent (own CUDA stream and
 * device buffers) and may be driven from distinct threads; the library owns
 * every device buffer and the caller owns every host buffer.  Arrays follow
 * the reference's Eigen tensor layouts (column-major, row index i fastest):
 *   populations (R, C, 9) -> [i + R*(j + C*k)],  u (R, C, 2),  rho (R, C),
 * and node coordinates are (i, j) pairs of int64, as Eigen::Index in
 * Point / BoundaryPoint / ObstaclePoint (llalbm/src/utils/aliases.hpp:55-357).
 */
#ifndef LLALBM_CUDA_H
#define LLALBM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LLB_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define LLB_OK 0
#define LLB_E_INVALID (-1)     /* bad argument (null pointer, bad enum, bad size) */
#define LLB_E_GEOMETRY (-2)    /* node lists inconsistent (overlap, out of range, fluid on edge) */
#define LLB_E_NOMEM (-3)       /* device or host allocation failed */
#define LLB_E_CUDA (-4)        /* CUDA runtime error (message in llb_last_error) */
#define LLB_E_NODEVICE (-5)    /* no usable CUDA device */
#define LLB_E_STATE (-6)       /* call out of order (e.g. llb_step before llb_init) */
#define LLB_E_NUMERIC (-7)     /* non-finite density detected on the device */
#define LLB_E_UNSUPPORTED (-8) /* valid input outside what the engine implements */
#define LLB_E_TIMEOUT (-9)     /* a bounded wait gave up */

/* ---- enums ------------------------------------------------------------- */
/* collision operators: BGKCollisionPolicy (collisions/BGKCollision.hpp:62-306),
   TRTCollisionPolicy (collisions/TRTCollision.hpp:65-345) */
#define LLB_BGK 0
#define LLB_TRT 1
/* population storage: FP64; FP32 or FP16 storing f_k - w_k (collision in FP32) */
#define LLB_STORE_F64 0
#define LLB_STORE_F32S 1
#define LLB_STORE_F16S 2
/* memory pattern: two buffers (ping-pong) or one buffer updated in place (A-A) */
#define LLB_PATTERN_AB 0
#define LLB_PATTERN_AA 1
/* open-boundary policies: ZouHePolicy (boundaries/ZouHePolicy.hpp:58-123),
   OpenBoundaryPolicy (boundaries/OpenBoundaryPolicy.hpp:58-61), and the Zou-He
   pressure policy this project adds (llalbm_cuda/ZouHePressurePolicy.hpp) */
#define LLB_BC_ZH_VELOCITY 0
#define LLB_BC_OPEN 1
#define LLB_BC_ZH_PRESSURE 2
/* obstacle policies: BounceBackPolicy (boundaries/BounceBackPolicy.hpp:143-187)
   and PSBounceBackPolicy, partially saturated bounce-back
   (boundaries/PSBounceBackPolicy.hpp:177-293; FP64 storage, single lattices) */
#define LLB_OBSTACLE_BOUNCE_BACK 0
#define LLB_OBSTACLE_PARTIAL 1
/* InputNodeType codes of the lattice file format (aliases.hpp:41-48) */
#define LLB_NODE_FLUID 0
#define LLB_NODE_SOLID 1
#define LLB_NODE_BOUNDARY 2
#define LLB_NODE_INLET 3
#define LLB_NODE_OUTLET 4
#define LLB_NODE_OBSTACLE 5
/* llb_step flags */
#define LLB_STEP_MACRO 1u /* write rho/u of the last step (Lattice.hpp:370-374 save) */

/* ---- lattice description ----------------------------------------------- */
typedef struct llb_lattice* llb_handle;

/* Everything Lattice::reinit receives (Lattice.hpp:453-481) plus the policy
   parameters the reference keeps in static members.  Side codes are the
   reference's btypes (aliases.hpp:28-38); corner types mean "no closure". */
typedef struct {
    int64_t rows, cols;                                   /* lattice_dimensions */
    int64_t n_fluid;    const int64_t* fluid_ij;          /* fluid_nodes */
    int64_t n_wall;     const int64_t* wall_ij;           /* boundary_coord */
    int64_t n_inlet;    const int64_t* inlet_ij;   const int32_t* inlet_side;   /* inlet_nodes_coord */
    int64_t n_outlet;   const int64_t* outlet_ij;  const int32_t* outlet_side;  /* outlet_nodes_coord */
    int64_t n_obstacle; const int64_t* obstacle_ij; const uint16_t* obstacle_dirs; /* may be NULL */
    int32_t inlet_bc, outlet_bc;                          /* LLB_BC_* */
    int32_t collision;                                    /* LLB_BGK / LLB_TRT */
    double tau;                                           /* BGK: BGKCollisionPolicy<2>::tau */
    double tau_even, tau_odd;                             /* TRT: TRTCollisionPolicy<2>::tau_even/odd */
    int32_t storage;                                      /* LLB_STORE_* */
    int32_t pattern;                                      /* LLB_PATTERN_* */
    int32_t device;                                       /* CUDA ordinal */
    int32_t open_table_rows;  /* per-step open-value ring capacity; 1 = values constant in time */
    int32_t obstacle_bc;                                  /* LLB_OBSTACLE_* (0: bounce-back) */
    double ps_tau;                                        /* PSBounceBackPolicy<2>::tau */
    const double* obstacle_b;  /* per wet obstacle, ObstaclePoint::get_b(); NULL: 1.0 (its default) */
} llb_desc;

/* Node vectors as the reference builds them from a grid of InputNodeType codes. */
typedef struct {
    int64_t n_fluid, n_wall, n_inlet, n_outlet, n_obstacle;
    int64_t* fluid_ij;
    int64_t* wall_ij;
    int64_t* inlet_ij;   int32_t* inlet_side;
    int64_t* outlet_ij;  int32_t* outlet_side;
    int64_t* obstacle_ij; uint16_t* obstacle_dirs;
} llb_node_lists;

/* ---- host-side lattice construction (no GPU needed) --------------------- */

/* Replaces the classification of read_lattice_file (utils/readers/LatticeReader.hpp:488-519):
   TensorLoopAccessor's row-major vector fill, verify_lattice_bounds,
   identify_node_type (utils/analysis/NodeIdentification.hpp:45-110),
   identify_obstacle_propagation (:137-211) and eliminate_non_wet_nodes (:229-242),
   in O(R*C) instead of the reference's O(N^2) std::find scans.
   `types` is (R, C) column-major InputNodeType codes.  counts[5] receives
   fluid, wall, inlet, outlet and wet-obstacle counts. */
int llb_classify_count(int64_t rows, int64_t cols, const uint8_t* types, int64_t counts[5]);
/* Fills caller-allocated arrays sized by llb_classify_count (n_* fields are
   checked against the counts). */
int llb_classify_fill(int64_t rows, int64_t cols, const uint8_t* types, llb_node_lists* out);

/* ---- lattice lifetime --------------------------------------------------- */

/* Replaces Lattice::reinit / the Lattice constructors' tensor allocation
   (Lattice.hpp:115-147, 173-239, 453-481) and the policy attach_nodes call
   (OMPPolicy.hpp:127-131): validates the node lists, builds the 1-byte node
   mask and uploads it, allocates the resident population buffers. */
int llb_create(const llb_desc* desc, llb_handle* out);
int llb_destroy(llb_handle h);

/* Replaces InitializationPolicy::update_nodes (OMPPolicy.hpp:139-143,
   initializers/InletOutletInitializer.hpp:90-129): values of the update
   functions for steps t_first .. t_first+count-1, laid out
   [count][n_inlet + n_outlet][2], inlets first.  Velocity and open nodes take
   (u_x, u_y); Zou-He pressure nodes take (rho0, tangential u). */
int llb_set_open_values(llb_handle h, int64_t t_first, int32_t count, const double* values);

/* Replaces the initial equilibrium (Lattice.hpp:295-296, 326-328) and the
   collision of step 0: afterwards the resident state is the post-collision
   populations of step 0. */
int llb_init(llb_handle h, uint32_t flags);

/* Replaces `nsteps` iterations of the perform_lbm loop body (Lattice.hpp:338-410):
   update_nodes, update_macro, calc_equilibrium, collide (+ open collide), stream
   (+ open stream), wall and obstacle bounce-back, inlet and outlet closures --
   one fused kernel per step.  LLB_STEP_MACRO keeps rho/u of the last step. */
int llb_step(llb_handle h, int32_t nsteps, uint32_t flags);

/* Index of the next step (number of collisions done). */
int llb_get_step(llb_handle h, int64_t* step);

/* ---- results (device -> host) ------------------------------------------ */

/* global_rho / global_u of the last LLB_STEP_MACRO step (Lattice.hpp:58-70 getters
   :499-506); either pointer may be NULL. */
int llb_get_macro(llb_handle h, double* rho, double* u);
/* rho and u of the current populations S_t (t = llb_get_step): what the next
   step's macro output would write, without stepping (fluid moments; the
   prescribed or Zou-He values of open nodes; rho 1 and u 0 elsewhere). */
int llb_compute_macro(llb_handle h, double* rho, double* u);
/* `populations` (Lattice.hpp:492): streams the resident post-collision state
   and applies bounce-back and the closures into an (R, C, 9) tensor.  Values
   are defined for fluid, inlet and outlet nodes; other nodes read 0. */
int llb_get_populations(llb_handle h, double* populations);
/* `after_collision_populations` of the last step, (R, C, 9); 0 off active nodes. */
int llb_get_post_collision(llb_handle h, double* populations);

/* FlowAnalyzer<2>::compute_flow_properties (utils/analysis/FlowAnalyzer.hpp:348-451)
   over the resident post-collision state: per-point terms exactly as the
   reference, totals summed on the device with compensated FP64.
   llb_set_force_points uploads the considered points once (ij: 2 n
   coordinates, dirs: n direction words). */
int llb_set_force_points(llb_handle h, const int64_t* ij, const uint16_t* dirs, int64_t n);
int llb_flow_forces(llb_handle h, double lift_drag[2]);
/* Gathers, for each considered point and each set direction bit, the
   post-collision value the reference reads (FlowAnalyzer.hpp:394-427) into
   values[n][8] (0 where the bit is clear), for feeding the reference analyzer. */
int llb_gather_force_inputs(llb_handle h, double* values);

/* Allocation-free variant of llb_set_force_points + llb_flow_forces; it has no
   counterpart in the reference.  For callers that cannot let the library call
   cudaMalloc once their loop runs -- a server whose device memory is committed
   up front under a fixed budget, or a host that must not trigger the
   device-wide synchronisation cudaMalloc/cudaFree can cause: the points and
   the per-block partial sums go to one static device array of
   LLB_NOALLOC_MAX_FORCE_POINTS points (about 1.2 MB per device, held until
   the process exits) instead of buffers allocated per call.  Same per-point
   terms and summation order as llb_flow_forces.  More than the maximum points
   fails with LLB_E_INVALID.  The first call on a device looks the array up
   (cudaGetSymbolAddress); CUDA loads device code lazily, so that lookup is
   where the array's memory is taken: make the first call before the loop that
   must not allocate and before any stream capture on that device.  All calls
   share the array: calls that overlap on the GPU race and must be serialised
   by the caller.  ij holds 2 n coordinates and dirs n direction words. */
#define LLB_NOALLOC_MAX_FORCE_POINTS 65536
int llb_flow_forces_noalloc(llb_handle h, const int64_t* ij, const uint16_t* dirs, int64_t n,
                            double lift_drag[2]);

/* Mass and momentum of the resident post-collision state (sum over fluid,
   inlet and outlet nodes of sum_k f, c_x f, c_y f) with compensated FP64;
   out[0] = mass, out[1] = momentum along j (u_x), out[2] = along -i (u_y). */
int llb_mass_momentum(llb_handle h, double out[3]);

/* ---- output writer ------------------------------------------------------- */
/* Writes the reference's velocity output files off the stepping thread:
   util::writer::write_lattice_file<2> (utils/writers/LatticeWriter.hpp:60-92),
   called by perform_lbm on save steps (Lattice.hpp:370-374), creates
   <dir>/output-<n>u_x.txt and <dir>/output-<n>u_y.txt with one text row per
   lattice row i holding u(i, j, d) for j = 0..C-1, each value in std::ostream's
   default format (printf "%.6g") followed by a space.  The files here are
   byte-identical.

   llb_writer_save_u enqueues, on the lattice's stream, a copy of u (written by
   the last LLB_STEP_MACRO step) into one of `slots` pinned host buffers and
   returns; the next steps may be enqueued at once (they run after the copy on
   the same stream).  A writer thread waits for the copy, formats the rows on
   `threads` threads and writes both files.  A call blocks only while every
   slot is still being written.  Errors of the background work (a file that
   cannot be opened, a CUDA error) are returned by the next save, by
   llb_writer_flush and by llb_writer_destroy.  The directory must exist.  One
   writer serves one calling thread at a time; flush (or destroy) the writer
   before destroying a lattice whose copies are still queued. */
typedef struct llb_writer* llb_writer_handle;
/* slots in [1, 64] (0: 3); threads in [1, 256] (0: the host's hardware
   threads, at most 16). */
int llb_writer_create(const char* dir, int32_t slots, int32_t threads, llb_writer_handle* out);
int llb_writer_save_u(llb_writer_handle w, llb_handle h, int64_t index);
/* The same files from a host array u in the reference's (R, C, 2) column-major
   layout; u is copied before the call returns. */
int llb_writer_save_host(llb_writer_handle w, const double* u, int64_t rows, int64_t cols, int64_t index);
/* Waits until every queued file is written. */
int llb_writer_flush(llb_writer_handle w);
/* Files written so far and the seconds the writer thread spent waiting for
   copies and formatting/writing. */
int llb_writer_stats(llb_writer_handle w, int64_t* files, double* wait_s, double* write_s);
int llb_writer_destroy(llb_writer_handle w);
const char* llb_writer_last_error(llb_writer_handle w);

/* ---- batches of lattices ------------------------------------------------ */
/* Many independent lattices (uneven sizes, BGK or TRT, own relaxation times,
   one storage form) advanced together by one persistent launch per step over
   a work list of lattice tiles -- or per several steps, launched
   cooperatively -- replayed from CUDA graphs.  There is no counterpart in the
   reference (its statics allow one parameter set per process); a batch is
   what a solve server runs.  Lattices join (llb_batch_add: creation, boundary
   values for steps 0.., step 0) and leave between calls.  Each lattice is an
   llb_handle sharing the batch's stream: read its results with the
   single-lattice calls on llb_batch_lattice's handle.  Stepping a lattice
   through that handle is allowed; the batch picks up its new step. */
typedef struct llb_batch* llb_batch_handle;
int llb_batch_create(int32_t device, int32_t storage, llb_batch_handle* out);
int llb_batch_destroy(llb_batch_handle b);
int llb_batch_add(llb_batch_handle b, const llb_desc* desc, const double* open_values, int32_t rows,
                  int32_t* slot);
int llb_batch_remove(llb_batch_handle b, int32_t slot);
/* Moves a lattice made by llb_create (boundary values set; initialised or
   not -- step 0 then runs on the batch's stream) into the batch, so its
   creation and upload can happen elsewhere (another thread, another stream)
   while the batch runs.  The batch owns it from then on.  A lattice whose
   nine planes reach 2^31 slots (about 200 million nodes), or with 2^16
   columns or more, is refused with LLB_E_UNSUPPORTED: the batch's kernels
   use 32-bit slot offsets and 16-bit tile indices. */
int llb_batch_attach(llb_batch_handle b, llb_handle h, int32_t* slot);
/* Takes a lattice out of the batch without destroying it: the caller owns
   the handle again (on a stream of its own that starts after the batch work
   queued so far) and destroys it with llb_destroy. */
int llb_batch_detach(llb_batch_handle b, int32_t slot, llb_handle* out);
/* Advances every lattice of the batch by nsteps. */
int llb_batch_step(llb_batch_handle b, int32_t nsteps);
int llb_batch_lattice(llb_batch_handle b, int32_t slot, llb_handle* out);
/* Launch shape: tile columns per block (1..8) and steps per launch (1: one
   launch per step, replayed from graphs; >1: cooperative multi-step launches). */
int llb_batch_set_config(llb_batch_handle b, int32_t block_y, int32_t steps_per_launch);
int llb_batch_get_config(llb_batch_handle b, int32_t* block_y, int32_t* steps_per_launch);
/* Which lattices a batch steps on compacted planes (only active nodes stored,
   one thread per slot) rather than the dense ones: LLB_LAYOUT_AUTO those with
   at least 5 % of their active nodes next to a wall, obstacle or dead node
   (the single-lattice default's rule), LLB_LAYOUT_COMPACT every lattice that
   has them, LLB_LAYOUT_DENSE none.  Attached lattices move at once, at their
   current step; results do not depend on the layout (FP64 bit for bit). */
#define LLB_LAYOUT_AUTO 0
#define LLB_LAYOUT_COMPACT 1
#define LLB_LAYOUT_DENSE 2
int llb_batch_set_layout(llb_batch_handle b, int32_t layout);
int llb_batch_get_layout(llb_batch_handle b, int32_t* layout);
/* Autotuner: times trial_steps real steps of the batch for every candidate
   layout and shape (the steps advance the lattices; every candidate computes
   the same arithmetic) and keeps the fastest. */
int llb_batch_tune(llb_batch_handle b, int32_t trial_steps, int32_t* block_y, int32_t* steps_per_launch,
                   float* ms_per_step);
int llb_batch_get_step(llb_batch_handle b, int64_t* step);
/* The lattice in `slot` stops before computing step index stop_step: later
   batch steps leave it as it is (-1: no stop).  A solve server sets each
   lattice's last step, so chunks need not end at the earliest completion. */
int llb_batch_set_stop(llb_batch_handle b, int32_t slot, int64_t stop_step);
/* Waits for the batch; LLB_E_TIMEOUT if a cooperative launch gave up a grid
   barrier.  The lattices' states are then unspecified (blocks that gave up
   skipped their later steps): remove them and add them again.  The barrier
   itself is reset, so the batch stays usable. */
int llb_batch_synchronize(llb_batch_handle b);
/* Polls of the cooperative launches' grid barrier before a block gives up and
   the launch reports LLB_E_TIMEOUT (-1: the default, 2^22).  For tests of the
   timeout path (0 makes every block but the last to arrive give up at once);
   no reference counterpart. */
int llb_batch_set_wait_limit(llb_batch_handle b, int64_t polls);
/* Without waiting: *done = 1 when everything queued on the batch has run. */
int llb_batch_query(llb_batch_handle b, int32_t* done);
/* Scheduling priority of the batch's stream (CUDA stream priorities: a lower
   number is a higher priority; clamped to the device's range, so INT32_MIN
   asks for the highest).  Blocks of a higher-priority stream are scheduled
   before waiting blocks of lower-priority streams.  Only on an empty batch. */
int llb_batch_set_stream_priority(llb_batch_handle b, int32_t priority);
int llb_batch_event_record(llb_batch_handle b, int32_t slot);
int llb_batch_event_elapsed_ms(llb_batch_handle b, int32_t slot_begin, int32_t slot_end, float* ms);
int llb_batch_info(llb_batch_handle b, int64_t* lattices, int64_t* nodes, int64_t* device_bytes);
const char* llb_batch_last_error(llb_batch_handle b);

/* ---- solve server -------------------------------------------------------- */
/* A request loop over a batch; no counterpart in the reference (one Lattice
   per process, driven by its own main()).  Requests -- a lattice description,
   its boundary values for steps 0..rows-1 and a step count -- are submitted
   from any thread and queued; they are admitted while the device bytes of the
   admitted lattices fit budget_bytes and (batched mode) the resident lattice
   nodes stay under a cap, shortest work first by default
   (llb_server_set_admission), and their state stays resident until they
   finish.  Batched mode: preparer threads create admitted lattices while the
   GPU runs, a worker advances them in two concurrent batches (lattices under
   2^20 nodes on a high-priority stream, larger ones on another) in chunks of
   max_chunk_steps -- each lattice stops on the device at its own last step --
   and a reaper thread copies results and frees.  Sequential mode: one request
   at a time, first come first served, through the plain single-lattice path.
   A request of `steps` steps (>= 2)
   ends with the state the reference's Lattice holds after perform_lbm(steps)
   and returns that call's rho and u: steps - 1 collisions and the macroscopic
   fields of the last step (llb_compute_macro).  The lattice's storage, device
   and pattern come from the server, not from the description.  Timestamps are
   seconds on a monotonic clock (llb_server_counters.clock_s is "now"). */
#define LLB_SERVE_BATCHED 0
#define LLB_SERVE_SEQUENTIAL 1
#define LLB_REQ_QUEUED 0
#define LLB_REQ_RUNNING 1
#define LLB_REQ_DONE 2
#define LLB_REQ_FAILED 3
typedef struct llb_server* llb_server_handle;
/* completed / failed requests, lattice-node updates of the completed ones,
   requests queued and admitted-but-unfinished now, device bytes charged,
   chunks launched and the lane steps they ran, the clock now, and the
   seconds the batched mode's threads spent creating lattices (preparer),
   waiting for chunks (worker) and copying results and freeing (reaper). */
typedef struct {
    int64_t completed, failed, node_steps, queued, running, bytes_in_use, chunks, batch_steps;
    double clock_s;
    double admit_s, wait_s, retire_s;
} llb_server_counters;
int llb_server_create(int32_t device, int32_t storage, int32_t mode, int64_t budget_bytes, int32_t max_chunk_steps,
                      llb_server_handle* out);
/* Admission policy of the batched mode: at most max_resident_nodes lattice
   nodes resident at once (0: the default, LLB_SERVE_DEFAULT_NODE_CAP; a
   request is always admitted when nothing runs), and the order queued
   requests are admitted in (LLB_ADMIT_SHORTEST_FIRST: least lattice nodes x
   steps first; LLB_ADMIT_FIFO: oldest first).  The byte budget applies as
   well. */
#define LLB_ADMIT_SHORTEST_FIRST 0
#define LLB_ADMIT_FIFO 1
#define LLB_SERVE_DEFAULT_NODE_CAP (32LL << 20)
int llb_server_set_admission(llb_server_handle s, int64_t max_resident_nodes, int32_t order);
/* Stops the worker after the running requests finish; queued ones fail. */
int llb_server_destroy(llb_server_handle s);
/* LLB_E_NOMEM if the lattice alone exceeds the budget.  The description's
   arrays and open_values are copied before the call returns. */
int llb_server_submit(llb_server_handle s, const llb_desc* desc, const double* open_values, int32_t rows,
                      int64_t steps, int64_t* request_id);
int llb_server_poll(llb_server_handle s, int64_t request_id, int32_t* state);
/* LLB_OK when done, LLB_E_TIMEOUT after timeout_s, LLB_E_CUDA if it failed. */
int llb_server_wait(llb_server_handle s, int64_t request_id, double timeout_s);
/* Copies rho (R*C) and u (R*C*2) (either may be NULL) and times = {submitted,
   admitted, done}; releases the request. */
int llb_server_result(llb_server_handle s, int64_t request_id, double* rho, double* u, double times[3]);
int llb_server_stats(llb_server_handle s, llb_server_counters* out);
const char* llb_server_last_error(llb_server_handle s);

/* ---- synchronisation, timing, errors ------------------------------------ */

int llb_synchronize(llb_handle h);
/* LLB_E_NUMERIC if any step since the last call produced a non-finite density
   (the reference's LLALBM_DEBUG NaN scan, Lattice.hpp:412-422), LLB_E_TIMEOUT
   if a pipelined kernel gave up a bounded wait; clears the flags. */
int llb_check_numerics(llb_handle h);
/* The same check in two halves, so the host need not wait for the step it
   just queued: _begin enqueues, on the handle's stream, a copy of the flag
   word into pinned host memory (slot in [0, 8)) and its reset, and returns;
   _end waits for that copy and returns what llb_check_numerics would have.
   A caller queues step n + 1 before it ends the check of step n, and the GPU
   never idles on the read-back.  No reference counterpart. */
int llb_check_numerics_begin(llb_handle h, int32_t slot);
int llb_check_numerics_end(llb_handle h, int32_t slot);
/* CUDA events on the handle's stream: slot in [0, 8). */
int llb_event_record(llb_handle h, int32_t slot);
int llb_event_elapsed_ms(llb_handle h, int32_t slot_begin, int32_t slot_end, float* ms);
/* Step-kernel selection, for the autotuner.  Plain steps run the TMA-pipelined
   kernel in configuration `config` (0..2: tile shape, stage count, warps; 6:
   the form's default shape with the tile's bounce bytes loaded too), the
   two-steps-per-pass kernel (3..5: the intermediate step stays in shared
   memory, so a pair of steps reads and writes the populations once; a lone
   step runs on the one-thread kernel), the one-thread-per-node kernel for
   config -1, for config -2 one thread per node of every 32-byte population
   sector that holds an active node (a list built on first use), for config -3
   one thread per slot of compacted planes that store only the fluid and open
   nodes (built on first use; the default for obstacle-rich lattices of 2^18
   nodes or more), and for config -4 the lattice resident in the shared memory
   of one thread-block cluster of 16 blocks, up to 4096 steps per launch with
   a cluster barrier between steps (lattices whose column slabs fit: about
   129 x 129 in FP64, 181 x 181 in FP32, 256 x 256 in FP16; the default up to
   12 000 nodes, 26 000 in FP16).  Lattices with partially saturated
   obstacles run on config -1 only; lattices beyond the 32-bit limits of the
   sector list or the compacted tables (2^31 slots; neighbouring columns more
   than 65 535 slots apart) have no config -2 or -3, and lattices that do not
   fit a cluster have no config -4 (LLB_E_UNSUPPORTED).  A lattice in a batch
   (llb_batch_add) refuses -3: the batch's kernels step it.  All
   configurations compute the same per-node arithmetic and give the same bits
   in every storage form. */
int llb_set_pipeline(llb_handle h, int32_t config);
int llb_get_pipeline(llb_handle h, int32_t* config);
/* Autotuner of one lattice (no reference counterpart): runs every plain-step
   configuration this lattice supports (-4..-1, 0..6) for trial_steps warm-up
   and trial_steps timed steps and keeps the fastest.  Every configuration
   gives the same bits, so these are ordinary steps of the simulation: the
   lattice advances by 2 x trial_steps per configuration tried (llb_get_step
   tells how far), and their boundary values must be set as for llb_step.
   best and ms_per_step (either may be NULL) receive the choice and its time. */
int llb_tune_pipeline(llb_handle h, int32_t trial_steps, int32_t* best, float* ms_per_step);
/* Columns of lattice nodes per thread block of the one-thread-per-node kernel
   (1..8; each block is 32 rows x block_y columns). */
int llb_set_launch_shape(llb_handle h, int32_t block_y);
/* Polls of the pipelined kernels' (configurations 0..6) waits for their
   shared-memory stages before they give up, flag LLB_E_TIMEOUT (read by
   llb_check_numerics) and return (-1: the default, 2^24).  The wait for the
   kernel's own copies in flight keeps the default, so a kernel never leaves
   with copies outstanding.  For tests of the timeout path (0 gives up at
   once); the state after a timed-out step is unspecified (re-run llb_init).
   No reference counterpart. */
int llb_set_wait_limit(llb_handle h, int64_t polls);
/* Device bytes held by the handle. */
int llb_device_bytes(llb_handle h, int64_t* bytes);
/* Message for the last error on this handle (or the last global error for NULL). */
const char* llb_last_error(llb_handle h);
int llb_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LLALBM_CUDA_H */
