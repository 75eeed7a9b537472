/*
 * tpt_field.h -- C ABI of the B200 coarse-grid field step of tpt-sim.
 *
 * The field step is the per-tick work tpt-sim does on the 4x4-pixel cell grid
 * (`xcells x ycells`, row-major `cy * xcells + cx`):
 *
 *   - the Eulerian air solver (pressure `pv`, velocity `vx`/`vy`, ambient heat
 *     `hv`, wall masks), replacing `step_air_gpu`
 *     (crates/tpt-sim/src/air_kernel/mod.rs:120);
 *   - the FFT Newtonian gravity solve (cell mass map -> `gx`/`gy`), replacing
 *     `GravityFft::solve` (crates/tpt-sim/src/gravity_gpu/mod.rs:114) as called
 *     by `step_gravity_gpu` (crates/tpt-sim/src/gravity_kernel.rs:920).
 *
 * Conventions shared by every entry point:
 *   - the return value is a status code: TPT_OK (0) or a negative TPT_ERR_*;
 *     `tpt_last_error_string()` describes the last failure of the calling
 *     thread. Nothing aborts and no C++ exception crosses the ABI.
 *   - every buffer argument is a DEVICE pointer unless its name ends in
 *     `_host`. Grids are `xcells * ycells` elements in the reference layout.
 *   - work is stream ordered on the `tpt_stream_t` given (a `cudaStream_t`;
 *     NULL = the legacy default stream). Nothing synchronises the host.
 *   - the caller owns the field buffers; a plan or a batch owns its scratch.
 *   - a plan or batch is used from one host thread / one stream at a time.
 */
#ifndef TPT_FIELD_H
#define TPT_FIELD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same object as `cudaStream_t`, declared without the CUDA headers. */
typedef struct CUstream_st *tpt_stream_t;

/* ---- status codes ------------------------------------------------------ */
enum {
    TPT_OK = 0,
    TPT_ERR_INVALID_DIMS = -1,   /* zero, too small or too large grid      */
    TPT_ERR_NULL_POINTER = -2,   /* a required pointer is NULL             */
    TPT_ERR_CUDA = -3,           /* a CUDA runtime/driver call failed      */
    TPT_ERR_DEVICE_TIMEOUT = -4, /* a bounded device-side wait gave up     */
    TPT_ERR_INVALID_ARG = -5,    /* enum value or size out of range        */
    TPT_ERR_OUT_OF_MEMORY = -6,  /* device allocation failed               */
    TPT_ERR_UNSUPPORTED = -7     /* no sm_100 device / feature missing     */
};

/* ---- enums mirroring tpt-core (crates/tpt-core/src/particle.rs:136-165) - */
enum { /* AirMode */
    TPT_AIR_ON = 0,
    TPT_AIR_PRESSURE_OFF = 1,
    TPT_AIR_VELOCITY_OFF = 2,
    TPT_AIR_OFF = 3,
    TPT_AIR_NO_UPDATE = 4
};
enum { /* GravityMode (the configured direction, not the Newtonian field) */
    TPT_GRAVITY_VERTICAL = 0,
    TPT_GRAVITY_OFF = 1,
    TPT_GRAVITY_RADIAL = 2,
    TPT_GRAVITY_CUSTOM = 3
};
enum { /* AIRC_* convection modes */
    TPT_AIRC_NONE = 0,
    TPT_AIRC_LEGACY = 1,
    TPT_AIRC_BOUSSINESQ = 2
};
enum { /* arithmetic of the gravity solve */
    TPT_PRECISION_FP32 = 0,      /* FP32 FFT convolution                    */
    TPT_PRECISION_SPLIT_BF16 = 1 /* DFT-as-GEMM on tcgen05, 3-term bf16 split,
                                    FP32 accumulate                          */
};

/* Wall ids the field step reads (crates/tpt-core/src/constants.rs:700-735). */
enum {
    TPT_WL_WALLELEC = 1,
    TPT_WL_EWALL = 2,
    TPT_WL_FAN = 5,
    TPT_WL_WALL = 8,
    TPT_WL_GRAV = 14,
    TPT_WL_BLOCKAIR = 16
};

/* Largest grid side the entry points accept (a 8192-px canvas). */
#define TPT_MAX_CELLS_PER_SIDE 2048u

/* ---- air step ---------------------------------------------------------- */

/*
 * The `SimulationConfig` fields `step_air_gpu` reads
 * (crates/tpt-sim/src/air_kernel/mod.rs:121-141), with the reference defaults
 * listed in `tpt_air_params_default`.
 */
typedef struct tpt_air_params {
    uint32_t xcells, ycells;
    uint32_t air_mode;        /* TPT_AIR_*                                  */
    uint32_t aheat_enable;    /* 0/1: run the ambient-heat pass             */
    uint32_t convection_mode; /* TPT_AIRC_*                                 */
    uint32_t gravity_mode;    /* TPT_GRAVITY_*                              */
    float edge_pressure;
    float edge_vx, edge_vy;
    float ambient_air_temp; /* Kelvin                                      */
    float vorticity_coeff;
    float custom_gx, custom_gy;
} tpt_air_params;

/*
 * Device buffers of one air grid, the `SimBuffers` handles of the reference
 * (crates/tpt-sim/src/buffers/mod.rs:186-230). `opv/ovx/ovy/ohv` are the
 * reference's scratch grids and are overwritten. `pmap`/`elem_props` feed the
 * particle HotAir -> pressure pass (crates/tpt-sim/src/air_kernel/settle.rs:
 * 118-161); pass pmap = NULL to skip it.
 */
typedef struct tpt_air_bufs {
    float *pv, *vx, *vy, *hv;       /* state, read and written            */
    float *opv, *ovx, *ovy, *ohv;   /* scratch                            */
    uint32_t *block_air;            /* rebuilt at the end of the step     */
    uint32_t *block_airh;           /* rebuilt at the end of the step     */
    const uint32_t *wall_bmap;      /* wall id in the low byte            */
    uint32_t *wall_emap;            /* decremented once per step if > 0   */
    const uint32_t *elem_block_air; /* element stamps OR-ed into the masks */
    const uint32_t *elem_block_airh;
    const float *fan_vx, *fan_vy;   /* added where wall_bmap == WL_FAN    */
    /* optional HotAir pass */
    const uint32_t *pmap;       /* xres*yres packed words, type in bits 0..8 */
    const uint32_t *elem_props; /* n_elements rows of 32 words; word 11 is
                                   the f32 bit pattern of `hot_air`          */
    uint32_t xres, yres, n_elements;
} tpt_air_bufs;

/* Fills `p` with the reference defaults (crates/tpt-core/src/particle.rs:
 * 290-345) for an `xcells x ycells` grid. */
void tpt_air_params_default(tpt_air_params *p, uint32_t xcells, uint32_t ycells);

/*
 * One air step, replacing `step_air_gpu(&mut SimBuffers)`
 * (crates/tpt-sim/src/air_kernel/mod.rs:120-299): pressure, velocity,
 * smoothing/advection/vorticity/fans, then (if aheat_enable) ambient heat and
 * convection, the wall-mask rebuild and (if pmap) HotAir. xcells or ycells of
 * 0 returns TPT_OK without work, as the reference does (mod.rs:124-126).
 */
int tpt_air_step(const tpt_air_params *params, const tpt_air_bufs *bufs,
                 tpt_stream_t stream);

/* Largest grid (cells) tpt_air_step_static_scratch accepts: a 2048x2048-px
 * canvas, the largest the reference's UI offers. */
#define TPT_STATIC_SCRATCH_MAX_CELLS (512u * 512u)

/*
 * The same air step as tpt_air_step, for callers that cannot allocate
 * device memory -- for example an engine whose device memory all comes from
 * its own pool or graphics API, or code running where cudaMalloc is not
 * allowed. No counterpart in the reference (its SimBuffers always owns the
 * four scratch grids).
 *
 * The four scratch grids (`opv`, `ovx`, `ovy`, `ohv` of `bufs`, which are
 * ignored and may be NULL) come from one 4 MiB array in the library's own
 * device image instead, so the call allocates nothing, on the device or the
 * host. Every device that loads the library holds that array until the
 * process exits. Grids larger than TPT_STATIC_SCRATCH_MAX_CELLS cells are
 * rejected with TPT_ERR_INVALID_DIMS.
 *
 * Every call looks up the array's address in the current device's context
 * (cudaGetSymbolAddress, which allocates nothing), so the address stays
 * valid across a cudaDeviceReset. The first call on a device may load the
 * library's device code into that context: make it outside any stream
 * capture. All calls share the one array: calls whose work can overlap on the GPU (other
 * streams, other host threads) race on it and must be serialised by the
 * caller. Nothing needs clearing between calls -- each step writes every
 * scratch cell it reads.
 */
int tpt_air_step_static_scratch(const tpt_air_params *params,
                                const tpt_air_bufs *bufs, tpt_stream_t stream);

/* Host twin of the wall-mask rebuild (crates/tpt-sim/src/buffers/spatial.rs:
 * 336-352): block masks from wall ids and emap, no element stamps. */
int tpt_wall_masks_host(const uint32_t *wall_bmap_host,
                        const uint32_t *wall_emap_host,
                        uint32_t *block_air_host, uint32_t *block_airh_host,
                        size_t cells);

/* ---- gravity ----------------------------------------------------------- */

typedef struct tpt_grav_plan tpt_grav_plan;

/*
 * Plan for one grid size, replacing `FftBuffers::allocate` + `build_kernels`
 * (crates/tpt-sim/src/gravity_gpu/mod.rs:140-200). The kernel spectra are
 * built on the device in FP64 once, then rounded to the plan's precision.
 * The plan owns all of its scratch. Calls cudaMalloc; synchronises the
 * current device once at the end of creation.
 */
int tpt_grav_plan_create(uint32_t xcells, uint32_t ycells, int precision,
                         tpt_grav_plan **out);
int tpt_grav_plan_destroy(tpt_grav_plan *plan);
/* Padded transform size the plan uses (for reporting). */
int tpt_grav_plan_dims(const tpt_grav_plan *plan, uint32_t *n1, uint32_t *n2);

/*
 * One gravity solve, replacing `GravityFft::solve(bufs, mass, 1/65536)`
 * (crates/tpt-sim/src/gravity_gpu/mod.rs:114-135, 204-278):
 *   gx/gy[p] = mask[p] ? sum_m mask[m] * mass[m] * mass_scale_inv *
 *                        (-M_GRAV) * (p - m) / |p - m|^3 : 0
 * `mass_fx` is the fixed-point accumulator (mass * 65536 as i32).
 */
int tpt_grav_solve(tpt_grav_plan *plan, const int32_t *mass_fx,
                   float mass_scale_inv, const uint32_t *mask, float *gx,
                   float *gy, tpt_stream_t stream);
/* Same solve with an f32 mass grid (no fixed point). */
int tpt_grav_solve_f32(tpt_grav_plan *plan, const float *mass,
                       const uint32_t *mask, float *gx, float *gy,
                       tpt_stream_t stream);

/*
 * Host gravity-mask flood fill, replacing `rebuild_gravity_mask`
 * (crates/tpt-sim/src/gravity_kernel.rs:658-712): cells 4-connected to the
 * border through non-WL_GRAV cells get 0xFFFFFFFF, the rest 0.
 */
int tpt_grav_mask_rebuild(const uint32_t *wall_bmap_host, uint32_t *mask_host,
                          uint32_t xcells, uint32_t ycells);

/* Fixed-point mass of `m` (crates/tpt-sim/src/gravity_kernel.rs:217-229):
 * round half away from zero of m * 65536 in f32 arithmetic. */
int32_t tpt_mass_to_fixed(float m);

/* ---- gravity tick with particles -------------------------------------- */

/* Particle slots, struct of arrays (`SimBuffers::part_*`,
 * crates/tpt-sim/src/buffers/mod.rs:186-230), device pointers. */
typedef struct tpt_particles {
    uint32_t num_slots;       /* slots scanned (`used_slot_bound`)               */
    const uint32_t *ty;       /* element id; 0 = PT_NONE                         */
    const float *x, *y;       /* position in pixels                              */
    float *vx, *vy;           /* velocity, updated in place                      */
    const int32_t *life, *tmp;
    const float *temp;        /* kelvin                                          */
    const uint32_t *flags;    /* 0x08 FLAG_MOVABLE, 0x10 rigid-body pixel         */
    const uint32_t *move_lut; /* 12 words per element id (`build_move_lut`):
                                 [0] properties, [7] loss as f32 bits           */
    uint32_t n_types;         /* element ids below this have a record (PT_NUM)   */
} tpt_particles;

/* One sandbox's gravity grids (`SimBuffers`), device pointers, each
 * (xres / 4) * (yres / 4) cells; the plan's size must be that cell grid. */
typedef struct tpt_grav_state {
    uint32_t xres, yres;              /* canvas in pixels                        */
    const uint32_t *wall_bmap, *wall_emap, *grav_mask;
    int32_t *mass;                    /* this tick's accumulator (gpu_grav_mass)  */
    int32_t *mass_prev;               /* snapshot the solve reads                 */
    float *tool_mass;                 /* painted PGRV/NGRV wells, consumed; NULL = none */
    const int32_t *override_mass;     /* one-tick CEXP/GSNS mass writes; NULL = none   */
    const uint32_t *override_set;
    float *gx, *gy;                   /* the solved field                         */
    float newton_grav;                /* NEWTON_GRAVITY_SCALE (1.0)               */
} tpt_grav_state;

/*
 * One Newtonian-gravity tick around the solve, replacing the body of
 * `step_gravity_gpu` (crates/tpt-sim/src/gravity_kernel.rs:826-1010) after
 * the mask rebuild (call tpt_grav_mask_rebuild on a wall change, as the
 * reference does):
 *   0. painted wells are folded into mass_prev (`seed_gravity_tool_mass_kernel`,
 *      :241-262) and the accumulator is cleared (`seed_gravity_mass_kernel`,
 *      :217-229);
 *   1. gx/gy = the plan's solve of mass_prev (`GravityFft::solve`);
 *   2. every particle gets its element's Loss, then newton_grav * g of its
 *      cell (`apply_gravity_kernel`, :434-516), and adds its element's mass to
 *      the accumulator in fixed point (`build_gravity_mass_kernel`, :275-376),
 *      in one pass over the slots;
 *   3. the override writes replace their cells (`apply_grav_mass_override_kernel`,
 *      :379-391) and mass_prev = mass (`copy_gravity_mass_kernel`, :518-527).
 * With Newtonian gravity off the reference skips the pass; so does the caller.
 */
int tpt_grav_step(tpt_grav_plan *plan, const tpt_grav_state *state,
                  const tpt_particles *parts, tpt_stream_t stream);

/* ---- batched instances ------------------------------------------------- */

typedef struct tpt_batch tpt_batch;

/* One independent sandbox instance of a batch. */
typedef struct tpt_instance_desc {
    tpt_air_params air; /* grid size and air config of the instance     */
    uint32_t newton_grav; /* 0/1: solve gravity every tick (config flag) */
} tpt_instance_desc;

/* Device pointers of one instance's grids inside a batch's arenas. Every
 * grid has `ycells` rows of `pitch` elements (pitch = xcells rounded up to
 * 32, so each row starts on a 128-byte boundary): cell (cx, cy) is at
 * cy * pitch + cx. tpt_batch_write / tpt_batch_read convert from/to the
 * reference's dense layout (`cy * xcells + cx`). */
typedef struct tpt_instance_fields {
    float *pv, *vx, *vy, *hv;
    uint32_t *block_air, *block_airh, *wall_bmap, *wall_emap;
    uint32_t *elem_block_air, *elem_block_airh;
    float *fan_vx, *fan_vy;
    int32_t *grav_mass;  /* fixed-point mass the solve reads            */
    uint32_t *grav_mask; /* gravity propagation mask                     */
    float *gx, *gy;      /* solve output                                 */
    uint32_t pitch;      /* row stride of every grid above (elements)    */
} tpt_instance_fields;

/* Grid ids for tpt_batch_write / tpt_batch_read. */
enum {
    TPT_FIELD_PV = 0, TPT_FIELD_VX, TPT_FIELD_VY, TPT_FIELD_HV,
    TPT_FIELD_BLOCK_AIR, TPT_FIELD_BLOCK_AIRH, TPT_FIELD_WALL_BMAP,
    TPT_FIELD_WALL_EMAP, TPT_FIELD_ELEM_BLOCK_AIR, TPT_FIELD_ELEM_BLOCK_AIRH,
    TPT_FIELD_FAN_VX, TPT_FIELD_FAN_VY, TPT_FIELD_GRAV_MASS,
    TPT_FIELD_GRAV_MASK, TPT_FIELD_GX, TPT_FIELD_GY,
    TPT_FIELD_COUNT
};

/*
 * Host <-> device copy of one grid of one instance (`bytes` must equal
 * xcells*ycells*4), the batch counterpart of the reference's
 * `client.write` / `client.read` on a SimBuffers handle
 * (crates/tpt-sim/src/buffers/gpu_sync.rs:186-197, 375-396). Stream ordered
 * (cudaMemcpyAsync); synchronise the stream before touching `host` again.
 */
int tpt_batch_write(tpt_batch *batch, uint32_t instance, int field,
                    const void *host, size_t bytes, tpt_stream_t stream);
int tpt_batch_read(tpt_batch *batch, uint32_t instance, int field,
                   void *host, size_t bytes, tpt_stream_t stream);

/*
 * Host <-> device copy of one grid of EVERY instance at once: `host` holds
 * the instances' dense grids back to back in instance order, and `bytes`
 * must equal 4 * (sum of xcells*ycells). This is the bulk form of calling
 * tpt_batch_write / tpt_batch_read for each instance (the reference's
 * per-simulation `client.write` / `client.read`,
 * crates/tpt-sim/src/buffers/gpu_sync.rs:186-197, 375-396); it makes one
 * host copy and one device scatter or gather instead of one strided copy
 * per instance. The first call allocates a device staging buffer of one grid
 * of every instance, which later calls reuse: calls on one batch must be
 * ordered (one stream, or the caller's events), as its steps are. Stream
 * ordered; use pinned host memory for an asynchronous copy and synchronise
 * the stream before touching `host` again.
 */
int tpt_batch_write_field(tpt_batch *batch, int field, const void *host,
                          size_t bytes, tpt_stream_t stream);
int tpt_batch_read_field(tpt_batch *batch, int field, void *host,
                         size_t bytes, tpt_stream_t stream);

/* Forms of the batch's air tick (tpt_batch_tuning.air_form). */
enum {
    /* Two launches per tick over tiles (32x8, 64x8, 32x16 or 64x16 cells),
     * halos staged by TMA: pass A (pressure, velocity) writes opv/ovx/ovy,
     * pass B (smoothing, advection, vorticity, fans, heat, convection, masks)
     * reads them. */
    TPT_AIR_FORM_TILES = 0,
    /* One fused launch per tick: CTAs sweep down column strips with every
     * stage pipelined over the rows (no intermediate grid in memory), plus a
     * velocity pre-pass that only works for instances whose air moves far. */
    TPT_AIR_FORM_SWEEP = 1
};

/* Tuning knobs the autotuner picks (and a caller may pin). Results are the
 * same for every value: they change how the work is laid out, not what is
 * computed. A new batch starts at {32, 8, 1, 0, 0, TPT_AIR_FORM_TILES, 1}:
 * 32x8 tiles, no temporal blocking, each pass at its own residency, one
 * gravity stream, the tile form with the work queue. */
typedef struct tpt_batch_tuning {
    /* The air form's work unit. Tile form: the tile, tile_x x tile_y cells,
     * one of 32x8 (the default), 64x8, 32x16 and 64x16, one thread per cell.
     * Sweep form: a CTA of tile_x lanes (a multiple of 32 in 64..256) sweeps
     * down strips of about tile_y rows (8..2048); each lane owns a column, a
     * strip is at most tile_x - 12 columns wide (six halo columns on each
     * side), and strips of narrow instances are packed side by side into one
     * CTA. */
    uint32_t tile_x, tile_y;
    /* Temporal blocking of the tile form: ticks per block (1..50; 1 = none).
     * A block of k ticks is k + 1 launches: the first tick's velocity pass,
     * k - 1 launches that each finish one tick and start the next over 32x16
     * tiles (the velocity pass of tick t + 1 reads tick t's state from
     * shared memory), and the last tick's advection pass. The sweep form
     * takes 1. */
    uint32_t temporal_depth;
    /* Resident CTAs per SM of the air form's persistent launches (0 = as
     * many as fit). */
    uint32_t ctas_per_sm;
    /* Split-BF16 gravity of a batch holding both kinds of y stage (groups of
     * many equal-shape instances take the Toeplitz GEMM, the others the y
     * DFT pair): CTAs per launch of the DFT-pair groups' chain, which then
     * runs on a second stream beside the Toeplitz groups' chain (on the
     * remaining SMs). 0 runs the stages one after another on one stream.
     * Must be 0 for other batches; at most half the SMs. Results are the same
     * for every value. */
    uint32_t grav_side_ctas;
    uint32_t air_form;  /* TPT_AIR_FORM_TILES or TPT_AIR_FORM_SWEEP */
    /* Tile form: 1 (the default) = the persistent CTAs take tiles from an
     * atomic work queue (a counter per pass, cleared by the other pass's
     * launch), 0 = they stride the tile list statically. The sweep form
     * always takes its work items from a queue; 0 or 1. */
    uint32_t work_queue;
} tpt_batch_tuning;

/*
 * Creates a batch of `n` instances with grids allocated in packed device
 * arenas (zero-initialised), and gravity plans of `grav_precision`.
 */
int tpt_batch_create(uint32_t n, const tpt_instance_desc *descs,
                     int grav_precision, tpt_batch **out);
int tpt_batch_destroy(tpt_batch *batch);
int tpt_batch_fields(tpt_batch *batch, uint32_t instance,
                     tpt_instance_fields *out);
/*
 * Advances every instance by `ticks` field steps (air, then gravity if
 * newton_grav), the same result as calling tpt_air_step and tpt_grav_solve
 * once per tick per instance. Uses a CUDA graph per (ticks, stream) that is
 * captured on first use and replayed after.
 */
int tpt_batch_step(tpt_batch *batch, uint32_t ticks, tpt_stream_t stream);
/* Times candidate tunings on the batch's own data (state is saved and
 * restored) and keeps the fastest: the air form with its shape (tile_x x
 * tile_y), CTAs per SM and tile order, the temporal depth (tile form), then,
 * for batches with gravity, the whole step (air and gravity together) for
 * the best few air settings and every gravity branch split. The choice is cached in
 * the process per batch composition -- the instances' (xcells, ycells)
 * buckets (powers of two) with their counts, and the gravity precision -- so
 * tuning a batch of the same composition again only applies the cached
 * settings. Synchronous. */
int tpt_batch_tune(tpt_batch *batch, tpt_stream_t stream);
int tpt_batch_get_tuning(const tpt_batch *batch, tpt_batch_tuning *out);
int tpt_batch_set_tuning(tpt_batch *batch, const tpt_batch_tuning *tuning);

/* Device time of the two phases of a batch step, measured separately. */
typedef struct tpt_batch_profile {
    float air_ms;              /* `ticks` air ticks alone (all instances)  */
    float grav_ms;             /* `ticks` gravity solves alone             */
    uint32_t ticks;
    /* Air launches per tick without temporal blocking: 2 (3 in the tile
     * form with a NoUpdate + heat instance: its settle). At temporal depth
     * k, a block of n <= k ticks makes n + 1 launches (plus the n settles). */
    uint32_t air_launches_per_tick;
    uint32_t grav_launches_per_tick;
    uint64_t cells;            /* sum of xcells*ycells over instances      */
    uint64_t grav_cells;       /* same, over instances with newton_grav    */
    double grav_flops_per_tick;/* executed flops of one tick's solves      */
} tpt_batch_profile;

/*
 * Times `ticks` air ticks and `ticks` gravity solves of the batch as two
 * separate chains on `stream` (CUDA events on that stream), restoring the
 * batch state afterwards. Synchronous. For roofline reporting.
 */
int tpt_batch_profile_phases(tpt_batch *batch, uint32_t ticks,
                             tpt_stream_t stream, tpt_batch_profile *out);

/* ---- 3-D sandbox field step (crates/tpt-sim/src/voxel3d) ---------------
 *
 * The 3-D sandbox's coarse grid: 64^3 cells of 4^3 voxels, one f32 (or i32)
 * per cell, index (y << 12) | (z << 6) | x (air_kernel.rs:5-8). Voxels are
 * 256^3 u32 words, index (y << 16) | (z << 8) | x, packed as
 * ty | temp_q << 8 | life << 24 with temp = temp_q * 0.125 K
 * (step/mod.rs:125-133). Bricks are 8^3 voxels, brick id
 * (by << 10) | (bz << 5) | bx (air_kernel.rs:227-230).
 *
 * The reference's tick (engine.rs:195-208) calls, in order,
 * AirState::gather, AirState::solve, gravity::solve, gravity::clear_mass and,
 * after the element passes, gravity::gather. Each has an entry point below;
 * tpt_vox_field_step runs the first four for a list of worlds.
 */
enum {
    TPT_VOX_AXIS = 64,          /* cells per axis (AIR_AXIS)               */
    TPT_VOX_CELLS = 262144,     /* AIR_COUNT                               */
    TPT_VOX_VOXELS = 16777216,  /* VOXEL_COUNT                             */
    TPT_VOX_BRICKS = 32768,     /* BRICK_COUNT                             */
    TPT_VOX_AIR_ITERATIONS = 12,  /* AIR_JACOBI_ITERATIONS, the default    */
    TPT_VOX_GRAV_ITERATIONS = 24  /* GRAVITY_ITERATIONS (fixed)            */
};

/* How a plan runs the Jacobi solves. */
enum {
    TPT_VOX_AUTO = 0,      /* TPT_VOX_BATCHED                                */
    TPT_VOX_CLUSTER = 1,   /* one 16-CTA cluster per field, the whole grid in
                              distributed shared memory, one launch for every
                              world's sweeps                                 */
    TPT_VOX_PER_SWEEP = 2, /* one launch per pass and per sweep and world,
                              the reference's launch structure               */
    TPT_VOX_BATCHED = 3    /* one launch per sweep index for every world of
                              a call, air and gravity in the same launch,
                              programmatic dependent launches                */
};

/*
 * One world's device buffers. Every field is TPT_VOX_CELLS elements except
 * `voxel` and `aux_tmp` (TPT_VOX_VOXELS) and `sim_list` (TPT_VOX_BRICKS).
 * `sim_count` is the device word triple [n, 1, 1] the brick compaction
 * writes (step/active.rs:38-46); the gathers read n on the device.
 */
typedef struct tpt_vox_world {
    const uint32_t *voxel;     /* voxel_a                                  */
    const int32_t *aux_tmp;    /* per-voxel tmp, read by the gravity gather */
    const uint32_t *sim_list;  /* active brick ids                         */
    const uint32_t *sim_count; /* [n, 1, 1]                                */
    /* AirState (air.rs:52-80) */
    float *vx, *vy, *vz;
    float *p, *p_tmp;          /* Jacobi pressure pair                     */
    float *temp, *solid;
    int32_t *pv;               /* TPT pressure, 1/1024 fixed point         */
    /* gravity (buffers.rs:108-118) */
    int32_t *grav_mass;        /* 1/1024 fixed-point mass accumulator      */
    float *grav_potential, *grav_potential_tmp;
    float *grav_force_x, *grav_force_y, *grav_force_z;
} tpt_vox_world;

typedef struct tpt_vox_plan tpt_vox_plan;

/*
 * Creates a plan running the solves in `form` (TPT_VOX_*). CLUSTER fails
 * with TPT_ERR_UNSUPPORTED where the device cannot hold a 16-CTA cluster of
 * its kernel. The plan owns the forms' scratch (the reference's velocity
 * snapshot, air.rs:78-79, and the batched form's per-world source fields,
 * about 5 MiB per world for 16 worlds) and the gravity gather's table of
 * per-brick list counts (128 KiB); no entry point below allocates.
 */
int tpt_vox_plan_create(int form, tpt_vox_plan **out);
int tpt_vox_plan_destroy(tpt_vox_plan *plan);
/* The form the plan runs (TPT_VOX_CLUSTER or TPT_VOX_PER_SWEEP). */
int tpt_vox_plan_form(const tpt_vox_plan *plan);

/* air_clear_kernel (air_kernel.rs:182-204): zero velocity, pressure, solid
 * and pv; ambient temperature 293.15 K. Replaces AirState::new's clear. */
int tpt_vox_air_clear(const tpt_vox_world *world, tpt_stream_t stream);
/* AirState::gather (air.rs:126-148, air_kernel.rs:218-278): solid fraction
 * and mean non-empty temperature of the cells of every listed brick. */
int tpt_vox_air_gather(tpt_vox_plan *plan, const tpt_vox_world *world,
                       tpt_stream_t stream);
/* AirState::solve (air.rs:162-222): pv update, `iterations` Jacobi sweeps of
 * p / p_tmp (the reference's alternation: odd sweeps write p_tmp, even ones
 * p), then the advection of vx/vy/vz. iterations <= 65536. */
int tpt_vox_air_solve(tpt_vox_plan *plan, const tpt_vox_world *world,
                      uint32_t iterations, tpt_stream_t stream);
/* gravity::solve (gravity.rs:228-260): 24 Jacobi sweeps of the potential
 * from grav_mass, then the force field. On return grav_potential holds the
 * last sweep and grav_potential_tmp the one before, as the reference's
 * handle swap leaves them. */
int tpt_vox_grav_solve(tpt_vox_plan *plan, const tpt_vox_world *world,
                       tpt_stream_t stream);
/* gravity::clear_mass (gravity.rs:264-273). */
int tpt_vox_grav_clear_mass(tpt_vox_plan *plan, const tpt_vox_world *world,
                            tpt_stream_t stream);
/* gravity::gather (gravity.rs:276-289, 125-166): adds the fixed-point mass
 * of every listed brick's gravity elements to grav_mass. */
int tpt_vox_grav_gather(tpt_vox_plan *plan, const tpt_vox_world *world,
                        tpt_stream_t stream);
/*
 * For each of the `n` worlds: air gather, air solve (`air_iterations`),
 * gravity solve, clear mass -- the same result as calling the four entry
 * points above in that order per world. In the cluster form the solves of
 * all worlds are one launch, air and gravity clusters running side by side.
 */
int tpt_vox_field_step(tpt_vox_plan *plan, const tpt_vox_world *worlds,
                       uint32_t n, uint32_t air_iterations,
                       tpt_stream_t stream);

/* ---- save files (crates/tpt-save/src/lib.rs) ---------------------------
 *
 * A `.tptrs` file is the 8-byte magic "TPTRS001" followed by
 * zlib(bincode(SaveData)) (lib.rs:3-9, 355-372), bincode 1.3.3 with its
 * default options: little-endian fixed-width integers, u64 lengths for
 * vectors and strings, u32 enum variant indices, bool and Option tags as one
 * byte. SaveData (lib.rs:67-97) holds the SimulationConfig, the particles,
 * the eight cell grids below, the rigid bodies and (version 2) the signs.
 * These calls decode and encode it on the host, so real saves can seed the
 * field step (tpt_air_step buffers or a tpt_batch instance) and its grids
 * can be written back. Particles travel as raw 64-byte records; rigid bodies
 * and signs are kept as they were read and written back unchanged.
 */
typedef struct tpt_save tpt_save;

/* Every serialised field of SimulationConfig (crates/tpt-core/src/particle.rs:
 * 166-222) in its order; bools as 0/1 bytes, enums as their discriminant,
 * Option<f32> as a presence byte plus the value. */
typedef struct tpt_save_config {
    uint32_t xres, yres;
    uint8_t paused, aheat_enable, pretty_powder, _pad0;
    uint32_t edge_mode;    /* EdgeMode: 0 void, 1 solid, 2 loop */
    uint32_t gravity_mode; /* TPT_GRAVITY_* */
    uint32_t air_mode;     /* TPT_AIR_*     */
    float ambient_air_temp, edge_pressure;
    uint32_t display_mode, colour_mode, render_mode;
    float fire_intensity;
    uint8_t heat_enable, newton_grav, water_equal_test, _pad1;
    float vorticity_coeff;
    uint32_t convection_mode;
    float edge_velocity_x, edge_velocity_y, custom_gravity_x, custom_gravity_y;
    uint32_t temperature_scale;
    uint8_t decorations, _pad2[3];
    int32_t mouse_x, mouse_y;
    uint8_t gravity_field_enabled, gravity_zones_enabled, grid, _pad3;
    int32_t grid_size;
    uint8_t grid_checkerboard, hud, debug_hud, show_brush;
    uint8_t zoom_enabled, _pad4[3];
    int32_t zoom_window_x, zoom_window_y, zoom_factor, zoom_scope_x, zoom_scope_y, zoom_scope_size;
    uint8_t has_heat_display_limit_min, has_heat_display_limit_max, _pad5[2];
    float heat_display_limit_min, heat_display_limit_max;
    int32_t heat_display_auto_x, heat_display_auto_y, heat_display_auto_w, heat_display_auto_h;
} tpt_save_config;

/* The cell grids of a save, in SaveData order. */
enum {
    TPT_SAVE_AIR_VX = 0, TPT_SAVE_AIR_VY, TPT_SAVE_AIR_PV, TPT_SAVE_AIR_HV,
    TPT_SAVE_FAN_VX, TPT_SAVE_FAN_VY, TPT_SAVE_WALL_BMAP, TPT_SAVE_WALL_EMAP,
    TPT_SAVE_GRIDS
};
enum { TPT_SAVE_VERSION = 2, TPT_SAVE_MAX_CANVAS_DIM = 16384, TPT_SAVE_PARTICLE_BYTES = 64 };

typedef struct tpt_save_info {
    uint32_t version;
    uint32_t xcells, ycells;  /* xres / 4, yres / 4 */
    uint64_t n_particles, n_rigid_bodies, n_signs;
    uint64_t grid_len[TPT_SAVE_GRIDS]; /* elements; 0 where absent (the air
                                          grids of a pressureless save)   */
} tpt_save_info;

/* SimulationConfig::new(xres, yres) (particle.rs:224-281): the canvas
 * rounded up to a multiple of 4 and at least 64, and the defaults. */
void tpt_save_config_default(tpt_save_config *c, uint32_t xres, uint32_t yres);
/* A version-2 save of `config` with zeroed grids of its cell count and no
 * particles, rigid bodies or signs. */
int tpt_save_create(const tpt_save_config *config, tpt_save **out);
/* SaveData::from_bytes (lib.rs:374-421): magic, zlib, version 1 or 2,
 * canvas 1..16384 on each side; every malformed input is an error
 * (TPT_ERR_INVALID_ARG), never a crash. */
int tpt_save_decode(const void *bytes, size_t len, tpt_save **out);
/* SaveData::to_bytes (lib.rs:355-372): the version-2 layout, zlib at the
 * default level. `*bytes` belongs to the save and stays valid until the
 * next encode or the destroy. */
int tpt_save_encode(tpt_save *s, const void **bytes, size_t *len);
int tpt_save_destroy(tpt_save *s);
int tpt_save_get_info(const tpt_save *s, tpt_save_info *out);
int tpt_save_get_config(const tpt_save *s, tpt_save_config *out);
int tpt_save_set_config(tpt_save *s, const tpt_save_config *config);
int tpt_save_set_version(tpt_save *s, uint32_t version);
/* A grid as stored (`bytes` must be grid_len * 4) / replaced by `bytes / 4`
 * elements (0 allowed). */
int tpt_save_grid_read(const tpt_save *s, int grid, void *host, size_t bytes);
int tpt_save_grid_write(tpt_save *s, int grid, const void *host, size_t bytes);
/* The grid as SaveData::restore_into loads it (lib.rs:318-330, fit_f32 /
 * fit_u32): `cells` elements, the stored grid when its length is the
 * restored canvas's cell count, zeros otherwise. */
int tpt_save_grid_restore(const tpt_save *s, int grid, void *host, uint64_t cells);
/* Particle records (bincode of GpuParticle, particle.rs:27-44): n * 64 bytes. */
int tpt_save_particles_read(const tpt_save *s, void *host, size_t bytes);
int tpt_save_particles_write(tpt_save *s, const void *host, size_t bytes);
/* SaveData::retain_air_pressure (lib.rs:247-255): include == 0 empties the
 * four air grids. */
int tpt_save_retain_air_pressure(tpt_save *s, int include);
/* The field-step configuration SaveData::restore_into gives the engine
 * (lib.rs:262-281): SimulationConfig::new of the saved canvas with the saved
 * paused/aheat/edge/gravity/air modes, ambient temperature and edge pressure;
 * the other air fields and newton_grav at their defaults. */
int tpt_save_instance_desc(const tpt_save *s, tpt_instance_desc *out);

/* ---- 3-D save files (crates/tpt-save/src/voxel3d.rs) -------------------
 *
 * A `.tpt3` file is the magic "TPT3RS01" followed by
 * zlib(bincode(Voxel3dSaveData)) (voxel3d.rs:1-15, 216-276), the same
 * bincode 1.3.3 encoding as `.tptrs`. Voxel3dSaveData (voxel3d.rs:63-90) is
 * version 4: the Voxel3dConfig, the voxel words, the four per-voxel
 * auxiliary arrays (each empty or TPT_VOX_VOXELS long), the coarse air grid
 * (empty or a multiple of TPT_VOX_CELLS floats: vx | vy | vz | pv | t |
 * solid, pv in pressure units) and the rigid bodies (kept as read).
 */
typedef struct tpt_vox_save tpt_vox_save;

/* Voxel3dConfig (crates/tpt-core/src/voxel3d/mod.rs:96-122), serialised
 * fields in order. */
typedef struct tpt_vox_save_config {
    uint32_t dim;
    uint8_t paused, _pad0[3];
    float ambient_temp_k;
    float gravity[3];
    uint32_t edge_mode;      /* EdgeMode: 0 void, 1 solid, 2 loop */
    uint8_t air_enabled, _pad1[3];
    uint32_t air_iterations;
    float sun_dir[3];
    float exposure, render_scale;
    uint32_t ao_rays;
    uint8_t shadows, _pad2[3];
} tpt_vox_save_config;

/* The arrays of a 3-D save, in Voxel3dSaveData order. */
enum {
    TPT_VOX_SAVE_VOXELS = 0, TPT_VOX_SAVE_CTYPE, TPT_VOX_SAVE_TMP, TPT_VOX_SAVE_TMP2,
    TPT_VOX_SAVE_TMP3, TPT_VOX_SAVE_AIR, TPT_VOX_SAVE_ARRAYS
};
enum { TPT_VOX_SAVE_VERSION = 4, TPT_VOX_MAX_BODIES = 64, TPT_VOX_BODY_VOXELS = 32768 };

typedef struct tpt_vox_save_info {
    uint32_t version;
    uint64_t len[TPT_VOX_SAVE_ARRAYS]; /* elements of each array        */
    uint64_t n_bodies;
} tpt_vox_save_info;

/* Voxel3dConfig::default (mod.rs:124-141). */
void tpt_vox_save_config_default(tpt_vox_save_config *c);
/* Voxel3dSaveData::empty (voxel3d.rs:147-152): zeroed voxels, no air,
 * no auxiliary arrays, no bodies. */
int tpt_vox_save_create(const tpt_vox_save_config *config, tpt_vox_save **out);
/* Voxel3dSaveData::from_bytes (voxel3d.rs:234-253) and its layout checks
 * (validate, :155-214); every malformed input is TPT_ERR_INVALID_ARG. */
int tpt_vox_save_decode(const void *bytes, size_t len, tpt_vox_save **out);
/* Voxel3dSaveData::to_bytes (voxel3d.rs:216-231): the layout is checked
 * first. `*bytes` belongs to the save until the next encode or destroy. */
int tpt_vox_save_encode(tpt_vox_save *s, const void **bytes, size_t *len);
int tpt_vox_save_destroy(tpt_vox_save *s);
int tpt_vox_save_get_info(const tpt_vox_save *s, tpt_vox_save_info *out);
int tpt_vox_save_get_config(const tpt_vox_save *s, tpt_vox_save_config *out);
int tpt_vox_save_set_config(tpt_vox_save *s, const tpt_vox_save_config *config);
/* An array as stored (`bytes` = len * 4) / replaced (any multiple of 4). */
int tpt_vox_save_array_read(const tpt_vox_save *s, int array, void *host, size_t bytes);
int tpt_vox_save_array_write(tpt_vox_save *s, int array, const void *host, size_t bytes);
/* The air state Voxel3dEngine::load_world gives the AirState
 * (crates/tpt-sim/src/voxel3d/engine.rs:546-581): from the first six air
 * slots, pv converted to 1/1024 fixed point ((value * 1024) as i32); with no
 * air in the save, the cleared state (zero velocity, pv and solid, 293.15 K).
 * Host arrays of TPT_VOX_CELLS elements each. */
int tpt_vox_save_restore_air(const tpt_vox_save *s, float *vx, float *vy, float *vz, int32_t *pv, float *temp,
                             float *solid);

/* ---- diagnostics ------------------------------------------------------- */

/*
 * Reads and clears the library's device error word on the current device:
 * TPT_ERR_DEVICE_TIMEOUT if a bounded device-side wait (tensor-core
 * pipeline barriers) gave up since the last call, TPT_OK otherwise. The
 * kernel that timed out skipped its remaining work and released its
 * resources, so the context stays usable. Synchronises the device.
 */
int tpt_check_device_errors(void);
/*
 * Exercises that failure path without a fault: launches one device wait on
 * a barrier that nothing completes, bounded by `limit_clocks` SM clocks, in
 * the same bounded-wait code the batched kernels use. After it, the next
 * tpt_check_device_errors returns TPT_ERR_DEVICE_TIMEOUT (and clears it);
 * the context stays usable.
 */
int tpt_selftest_wait_timeout(uint32_t limit_clocks, tpt_stream_t stream);

/* Message of the last failure on the calling thread ("" if none). */
const char *tpt_last_error_string(void);
/* Number of kernel launches this library has issued (all threads). */
uint64_t tpt_kernel_launch_count(void);
/* Library version string. */
const char *tpt_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TPT_FIELD_H */
