/*
 * inundation_b200: C ABI of the B200 shallow-water step.
 *
 * Plain C structs of device pointers and sizes; no allocation inside any entry
 * point (the caller owns every buffer, sized by swe_workspace_bytes); every
 * function enqueues on the given stream and returns a status code (0 = ok).
 * Nothing is global, so calls on different streams with different buffers are
 * independent.
 *
 * The entry points replace the device dispatches the reference records in
 * inundation/vulkan/gpu_resident_batch.py. Each declaration names the
 * reference kernel(s) or host call it stands for (file:line).
 *
 * A mesh may hold several independent meshes ("instances", a batch): each
 * starts on a 256-cell block boundary and has its own clock, dt and CFL bound.
 * A single mesh is a batch of one.
 */
#ifndef INUNDATION_B200_H
#define INUNDATION_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *swe_stream_t; /* a cudaStream_t */

enum swe_status {
    SWE_OK = 0,
    SWE_ERR_ARGUMENT = 1,     /* a null pointer, a zero size or an unknown mode */
    SWE_ERR_CUDA = 2,         /* a CUDA launch or runtime call failed */
    SWE_ERR_TOO_LARGE = 3,    /* a size beyond a fixed limit: a block's edge tile larger than shared
                                 memory, or more cells than swe_volume_fp64_noalloc's static scratch holds */
    SWE_ERR_MATH = 4,         /* the device arithmetic lost the two-sum error term */
};

/* Control block of one instance's integer clock: 48 bytes, the layout of the
   reference's RESIDENT_CTRL_DTYPE (inundation/vulkan/gpu_resident_batch.py:64-77). */
typedef struct {
    uint64_t now_ticks;
    uint64_t stop_ticks;
    uint64_t steps;
    uint32_t dt_ticks;
    uint32_t dt_max_ticks;
    uint32_t dry_dt_ticks;
    float last_raw;
    float cfl_safety;
    uint32_t error;  /* set by the device: 1 = a bounded wait for staged data timed out,
                        2 = a grid barrier of the persistent kernel timed out */
} swe_ctrl_t;

/* Static mesh in two tile layouts (device pointers).
   Block b = cells [256 b, 256 b + 256), of which block_cells[b] are real (the
   rest pad an instance to whole blocks). Its 256-cell tile is the contiguous
   range [tile_ptr[b], tile_ptr[b + 1]) of the tile_* arrays, tile_count[b]
   records then padding to a multiple of 32: first the edges whose left cell
   is in b and right cell in b or a boundary, then those whose left cell is in
   b and right cell in another block, then the edges whose right cell is in b
   and left cell is not, each group in the reference's resident edge order
   (gpu_resident_batch.py:175).
   lcsr[k] = (position in the tile << 1) | is_right for the CSR slots k of each
   cell, in the reference's per-cell order (inundation/mesh/geometry.py:454-468,
   remapped as blocks.py:33-44).
   The 64-cell compute tiles (tile t = cells [64 t, 64 t + 64), four per block)
   are laid out the same way in the sub_* arrays, with their local CSR regrouped
   per tile from sub_lcsr[sub_lcsr_ptr[t]] (multiples of 8).
   Every per-cell array (area, n_mann and all state arrays) holds n_blocks * 256
   entries; cptr holds n_blocks * 256 + 4, flat across the batch. */
typedef struct {
    uint32_t n_cells;         /* cells, padding between instances included */
    uint32_t n_blocks;
    uint32_t max_tile_edges;  /* the largest tile_count */
    uint32_t n_inst;          /* instances in the batch */
    const int32_t *tile_cl;   /* left cell */
    const int32_t *tile_cr;   /* right cell, -1 on a wall */
    const float *tile_nx;
    const float *tile_ny;
    const float *tile_len;
    const float *tile_dzl;    /* face elevation minus the left bed */
    const float *tile_dzr;
    const uint32_t *tile_ptr;   /* n_blocks + 1 */
    const uint32_t *tile_count; /* n_blocks */
    const uint32_t *cptr;       /* n_blocks * 256 + 4 */
    const uint16_t *lcsr;       /* one per CSR slot */
    const float *area;
    const float *n_mann;
    const uint32_t *ring_ptr;   /* block two-ring CSR (blocks.py:93-118) */
    const uint32_t *ring_idx;
    const uint32_t *block_inst;  /* n_blocks: instance of each block */
    const uint32_t *block_cells; /* n_blocks: real cells of each block */
    uint32_t max_sub_edges;
    uint32_t max_sub_slots;
    const int32_t *sub_cl;
    const int32_t *sub_cr;
    const float *sub_nx;
    const float *sub_ny;
    const float *sub_len;
    const float *sub_dzl;
    const float *sub_dzr;
    const uint32_t *sub_ptr;      /* n_blocks * 4 + 1 */
    const uint32_t *sub_count;    /* n_blocks * 4 */
    const uint16_t *sub_lcsr;
    const uint32_t *sub_lcsr_ptr; /* n_blocks * 4 + 1 */
    /* Open boundary edges (inundation/vulkan/solver.py:239-243, shaders/flux.py:187-294):
       an edge with right cell -2 - k is open edge k; -1 stays a wall. open_cond holds
       two words per open edge, its condition (0 wall, 1 free outflow, 2 normal depth,
       3 stage, 4 inflow) and its value as float bits (sqrt(S)/n, the depth over the
       cell's bed, or the discharge per unit width). NULL when n_open is 0. */
    uint32_t n_open;
    const uint32_t *open_cond;
    /* The local CSR of the 256-cell tiles regrouped per tile like sub_lcsr: tile b's
       slots from blk_lcsr[blk_lcsr_ptr[b]] (multiples of 8), the array 8 slots longer than
       its last segment; max_blk_slots the longest segment. Read by stage kernel 3 only
       (may be NULL otherwise). */
    uint32_t max_blk_slots;
    const uint16_t *blk_lcsr;
    const uint32_t *blk_lcsr_ptr; /* n_blocks + 1 */
} swe_mesh_t;

/* Mutable state and the run workspace (device pointers). */
typedef struct {
    float *h, *hu, *hv, *h_lo;     /* committed state; h_lo: compensated low word */
    float *h1, *hu1, *hv1, *h1_lo; /* Heun predictor */
    float *clamp_mass;             /* per-cell positivity-clamp volume (diagnostic) */
    uint32_t *blk;                 /* 3 words per block: wet, active, forced */
    uint32_t *active_list;         /* 2 x n_blocks: active blocks of the current step (first half) */
    uint32_t *items;               /* 2 x 4 words per 64-cell tile: work items of the tiled kernels (first
                                      half); the persistent kernel queues tile ids in the second half */
    uint32_t *sched;               /* 16 words: [0] active blocks, [1] next blocks, [2] done CTAs, [3] work items,
                                      [4] next items, [6..7] uint64 cells computed over real steps; the
                                      persistent kernel's [10] step epoch, [11] start-list tiles taken and
                                      [12..15] its two tile queues' lengths and taken counts; others zero */
    uint32_t *dt_buf;              /* 4 words per instance: [0] this step's dt (float bits, 0 = no-op),
                                      [1] the next step's CFL bound, [2..3] the persistent kernel's
                                      published (dt, step epoch) pair; 16-byte aligned */
    swe_ctrl_t *ctrl;              /* one per instance */
    uint32_t *sync;                /* 64 zeroed words: the grid barrier of the persistent kernel (kernel 2;
                                      each launch zeroes word 0, its arrival counter, before it starts) */
    uint32_t *marks;               /* 2 words per block, zeroed with sched word 10 at the start of a run: word
                                      0 the epoch of the latest step the block is active in (kernel 2), word
                                      1 unused */
    float *open_vol;               /* 4 words per open edge, zeroed at the start of a run: the volume that
                                      left (hi, lo) and entered (hi, lo) the mesh through it, as exact
                                      float pairs (the per-edge form of TALLY_RESIDENT_GLSL,
                                      inundation/vulkan/shaders/resident.py:617-660); NULL when
                                      the mesh has no open edges */
} swe_state_t;

typedef struct {
    float g;
    float dry_tol;
    float cfl;
    uint32_t compensated; /* depth as a (h, h_lo) two-sum pair */
    uint32_t track_clamp; /* accumulate the clamp diagnostic */
    uint32_t active_set;  /* skip blocks outside the two-ring of wet blocks */
    uint32_t grid;        /* CTAs of the persistent stage kernels (0 = a default) */
    uint32_t kernel;      /* stage kernel: 0 = 64-cell tiles staged by bulk copies (default),
                             1 = 256-cell blocks with plain loads,
                             2 = swe_steps only: whole steps of 64-cell tiles in one persistent cooperative
                                 launch, phases separated by bounded grid barriers,
                             3 = 256-cell blocks staged by bulk copies (needs blk_lcsr) */
} swe_params_t;

/* Sparse sources (device pointers), one per cell: source k adds
   dt * rate[k] to the depth of cell cells[k] or, when hydro[k] != 0xFFFFFFFF,
   dt * (rate[k] + hscale[k] * q), q the value of hydrograph hydro[k] at the
   start of its instance's step (t = now_ticks / 2^20 s as a float).
   Hydrograph j is piecewise linear through the knots (knot_t[i], knot_q[i]),
   i in [knot_ptr[j], knot_ptr[j + 1]), and takes its end values outside them.
   hydro == NULL: constant rates only. */
typedef struct {
    const uint32_t *cells;
    const float *rate;
    const uint32_t *hydro;
    const float *hscale;
    const uint32_t *knot_ptr;
    const float *knot_t;
    const float *knot_q;
    uint32_t count;
    uint32_t n_hydro;
} swe_sources_t;

/* n_steps whole steps: swe_step n_steps times (kernel 0, 1 or 3), or one persistent cooperative launch
   running them all (kernel 2; params->grid caps its CTAs, 0 = as many as fit; status 3 when
   (4 n_steps + 1) x CTAs reaches 2^32, the range of its barrier counter). A wait of the
   persistent kernel that times out records error 2 in the control block. */
int swe_steps(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
              const swe_sources_t *sources, uint32_t n_steps, swe_stream_t stream);

/* Bytes of device workspace of a mesh of n_blocks blocks and n_inst
   instances: active list, work items, sched words, dt words and control
   blocks. */
size_t swe_workspace_bytes(uint32_t n_blocks, uint32_t n_inst);

/* Sets the shared-memory size of every per-block kernel for this mesh (call
   once, before any stream capture) and returns the persistent CTAs per SM of
   the chosen stage kernel (swe_params_t.kernel); for kernel 3, 0 when the mesh's
   largest block does not fit its shared memory (the kernel then refuses to run). */
int swe_configure(const swe_mesh_t *mesh, int kernel, int *blocks_per_sm);

/* One Heun stage over the active blocks, fused: edge fluxes of each tile into
   shared memory, the fixed-order per-cell gather and the update. stage 0 =
   predictor, 1 = corrector (adds the next step's CFL bound and the wet marks).
   Replaces flux_resident_gather + update_resident_gather[_comp]
   (inundation/vulkan/shaders/resident.py:187-291 and 401-513). */
int swe_stage(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage,
              swe_stream_t stream);

/* Sparse sources after the Heun step: compensated add, wet marks, then the
   post-source CFL bound of each wet source cell. Replaces source_resident
   (resident.py:665-733). */
int swe_apply_sources(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                      const swe_sources_t *sources, swe_stream_t stream);

/* Active flags = (wet | forced) dilated over each block's two-ring, compacted
   into active_list and the tile work items; then, when control_mode >= 0,
   step_control of every instance in the last CTA. An instance on a no-op step
   keeps its flags unless force = 1. Replaces block_dilate + step_control
   (resident.py:778-805, 813-885). */
int swe_block_dilate_compact(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                             int force, int control_mode, swe_stream_t stream);

/* Start of a run: wet flag of every block from the state (or all active).
   Replaces block_mark (resident.py:738-773). */
int swe_block_mark(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                   swe_stream_t stream);

/* Prologue CFL bound of the current state into each instance's dt word 0
   (reset to 1e30 first). Replaces dt_reset + cfl_edge_gather + cfl_gather
   (cfl.py:130-166, resident.py:528-610). */
int swe_cfl_prologue(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                     swe_stream_t stream);

/* Integer-tick step control of n_inst instances; mode 0 START, 1 STEP,
   2 RETARGET. Replaces step_control (resident.py:813-885). */
int swe_step_control(swe_ctrl_t *ctrl, uint32_t *dt_buf, uint32_t n_inst, int mode, swe_stream_t stream);

/* Whole prologue: block_mark, forced dilation, CFL bound, START
   (gpu_resident_batch.py:567-591). */
int swe_prologue(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
                 swe_stream_t stream);

/* One whole step: two stages, sources (if any), dilation and STEP control
   (gpu_resident_batch.py:489-513). */
int swe_step(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params,
             const swe_sources_t *sources, swe_stream_t stream);

/* ---- Adjoint: gradients of a gauge misfit, dt frozen ------------------------------------------
   No counterpart in the reference. The loss is sum over steps n = 1..N and
   gauges g of ((h + h_lo)(g, after step n) - obs[n - 1][g])^2; its gradient
   is taken with respect to Manning's n and the bed of every cell and to the
   discharge knots of the inflow hydrographs, with every step's dt held at
   its forward value. A run keeps checkpoints; each segment of steps is run
   again with swe_tape_record + swe_stage_taped to fill the tape, then
   reversed one step at a time by swe_adjoint_step (single-instance meshes
   without open edges: swe_stage_taped and swe_adjoint_segment refuse a mesh
   whose n_open is not 0). */

/* The record of a segment of steps (device pointers; slot k = k-th step of
   the segment, n = n_blocks * 256 padded cells). */
typedef struct {
    float *h, *hu, *hv, *h_lo; /* (capacity + 1) x n: the state at the start of every step, then at the end */
    float *s0, *s1;            /* capacity x 3 x n: each stage's gathered sums (sdh, sdhu, sdhv) */
    uint32_t *dt;              /* capacity: dt bits of every step (0 = a no-op step) */
    float *t;                  /* capacity: the hydrograph clock of every step, seconds */
    uint32_t *list;            /* capacity x n_blocks: the active blocks of every step */
    uint32_t *count;           /* capacity */
    uint32_t capacity;
} swe_tape_t;

/* Adjoint state and gradients (device pointers, n padded cells). */
typedef struct {
    float *lh, *lhu, *lhv;      /* adjoint of the state, carried from step to step */
    float *ls;                  /* 3 x n: adjoint of a stage's sums (scratch) */
    float *lsh, *lshu, *lshv;   /* adjoint of the predictor state (scratch) */
    float *uh, *ulo, *uhu, *uhv; /* the predictor state, recomputed (scratch) */
    uint32_t *mark;             /* n_blocks: tag of the step whose active blocks these are (scratch) */
    float *gn;                  /* d loss / d Manning n, per cell (accumulated) */
    float *gz;                  /* d loss / d bed elevation, per cell (accumulated) */
    double *gq;                 /* d loss / d knot discharge, per knot of swe_sources_t (accumulated) */
    uint32_t *sync;             /* NULL: one launch per phase; else 64 zeroed words for the grid barrier of a
                                   single cooperative launch per segment (word 40 set: a barrier wait timed out) */
    float cut_depth;            /* no derivative flows through a cell or face depth below this (0: the
                                   exact derivative of the discrete step) */
} swe_adjoint_t;

/* Gauges of the misfit (device pointers). */
typedef struct {
    const uint32_t *cells; /* distinct gauge cells */
    float *obs;            /* steps x count: observed (h + h_lo) after each step */
    double *loss;          /* the accumulated misfit */
    uint32_t count;
    uint32_t steps;
} swe_gauges_t;

/* Bed steps of every edge record from a bed z (n padded cells): face =
   max(zL, zR) in float64, dzL = face - zL, dzR = face - zR, as the geometry
   computes them (inundation/mesh/geometry.py:241-254). */
int swe_bed_steps(const swe_mesh_t *mesh, const float *z, float *tile_dzl, float *tile_dzr, uint32_t tile_records,
                  float *sub_dzl, float *sub_dzr, uint32_t sub_records, swe_stream_t stream);

/* swe_stage (kernel 0, 1 or 3) that also stores every computed cell's gathered sums. */
int swe_stage_taped(const swe_mesh_t *mesh, const swe_state_t *state, const swe_params_t *params, int stage,
                    float *sums, swe_stream_t stream);

/* Copies the state, dt, clock and active list at the start of a step into tape slot `slot`
   (slot == capacity: the end state only). */
int swe_tape_record(const swe_mesh_t *mesh, const swe_state_t *state, const swe_tape_t *tape, uint32_t slot,
                    swe_stream_t stream);

/* After a step: record == 1 writes (h + h_lo) at the gauges into obs row steps - 1 (the
   control block's count of real steps); record == 0 adds the squared misfit against that row to *loss. */
int swe_gauge_misfit(const swe_state_t *state, const swe_gauges_t *gauges, int record, swe_stream_t stream);

/* Reverses tape slots `slots - 1` down to 0 (slot k is the step from tape state k to k + 1):
   for each, adds the misfit's gradient at the state after the step (obs row row0 + k), then
   takes the adjoint back through the sources, the corrector and the predictor, accumulating
   gn, gz and gq. Block marks use tags tag0 + k + 1, which must not repeat within a run (give
   each segment its own range, e.g. tag0 = its first step's index). */
int swe_adjoint_segment(const swe_mesh_t *mesh, const swe_params_t *params, const swe_tape_t *tape,
                        const swe_adjoint_t *adj, const swe_sources_t *sources, const swe_gauges_t *gauges,
                        uint32_t slots, uint32_t row0, uint32_t tag0, swe_stream_t stream);

/* Sum of (h + h_lo) * area in float64, in a fixed order: partials holds
   swe_volume_partials(n) doubles. The reference does this on the host
   (inundation/workflow.py:913-922). */
uint32_t swe_volume_partials(uint32_t n_cells);
int swe_volume_fp64(const float *h, const float *h_lo, const float *area, uint32_t n_cells, double *partials,
                    double *out, swe_stream_t stream);

/* swe_volume_fp64 for callers that cannot allocate device memory (a host
   under a fixed device-memory budget, an application that owns the CUDA
   allocator, code running where cudaMalloc is not allowed). No counterpart in
   the reference, which sums the volume on the host. The partial sums live in
   a static 8 KiB device array that every GPU loading this library holds until
   exit, so n_cells is limited to 4,194,304 (SWE_ERR_TOO_LARGE above). Call it
   with the stream's device current; its first call on a device looks up the
   array's address, so make that first call before any stream capture. The
   address is kept for the life of the process: after a cudaDeviceReset the
   module may load elsewhere, so a process that resets a device must not call
   this entry point on that device again. All calls share the array: calls
   that overlap on the GPU (other streams, other threads) race and must be
   serialised by the caller. */
int swe_volume_fp64_noalloc(const float *h, const float *h_lo, const float *area, uint32_t n_cells, double *out,
                            swe_stream_t stream);

/* The two-sum of (v[0], v[1]) into v[2] (its error term) on the device: the
   reference's fast-math guard (inundation/vulkan/solver.py:449-467,
   resident.py:889-907). */
int swe_eft_probe(float *v, swe_stream_t stream);

/* The state beyond n open edges and their mass flux, on the device: case k is
   cases[6k..6k+5] = (h, hu, hv, nx, ny, HLLC mass flux) of the cell inside, with the
   condition words cond[2k], cond[2k+1] (kind, value bits); results[4k..4k+3] = (h, hu,
   hv) of the ghost and the boundary mass flux. The device half of the reference's
   probe (tests/unit/test_gpu_open_ghost.py:45-71 over shaders/flux.py:211-281). */
int swe_open_ghost_probe(const float *cases, const uint32_t *cond, float *results, uint32_t n, float g,
                         float dry_tol, swe_stream_t stream);

/* One bounded wait, on the device, for instance 0's published (dt, epoch) pair (dt words 2..3),
   the wait the persistent kernel's seats make for the step control's dt: *out = the dt bits once
   the pair carries `epoch`, or 0 after the 2 s limit, with error bit 4 set in instance 0's
   control block. For tests of the limit: no counterpart in the reference. */
int swe_dt_wait_probe(const swe_state_t *state, uint32_t epoch, uint32_t *out, swe_stream_t stream);

/* x^(-4/3) of n values on the device, the depth power of the Manning friction slope
   (Sf = g n^2 |u| h^(-4/3)) as the update evaluates it. Replaces the pow(h, 4/3) of
   update_resident_gather (resident.py:489-495), for tests of its accuracy. */
int swe_inv_pow43(const float *x, float *out, uint32_t n, swe_stream_t stream);

const char *swe_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* INUNDATION_B200_H */
