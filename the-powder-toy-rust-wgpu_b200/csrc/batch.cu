// batch.cu -- many independent sandbox instances stepped together.
//
// Layout: every grid of every instance lives in one of three packed device
// arenas (f32, u32, i32). Instance i's grids are `ycells` rows of
// `pitch_i` elements (pitch = xcells rounded up to 32, so rows start on
// 128-byte boundaries as TMA needs); cell (cx, cy) is at cy * pitch + cx.
// The air state (pv, vx, vy, hv and the two wall masks) has a second copy
// (ping-pong) for the air tick's two forms, chosen by the tuning: the tile
// form (air_tiles.cu; two TMA-staged tile passes per tick, heat and masks in
// the ping-pong halves, pv/vx/vy in place; with temporal blocking, blocks of
// k ticks whose middle launches fuse one tick's second pass with the next
// tick's first, air_fused.cu) or the row sweep (air_sweep.cu; one launch per
// tick plus a velocity pre-pass that only works for instances flagged by the
// previous tick, every state grid in ping-pong halves). The sweep's halves
// serve the tile form as the second set of velocity-pass outputs. After an
// odd tick count one copy-back restores the canonical buffers. Gravity (instances with
// newton_grav) is independent of air in the field step
// (crates/tpt-sim/src/air_kernel/heat.rs:182-203 uses the configured
// direction, not the Newtonian field), so it runs on a second stream branch
// of the captured graph, concurrently with the air chain.
//
// N ticks are captured once into a CUDA graph (up to CHUNK = 1000 ticks per
// graph; longer steps replay it) and replayed on later calls.
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "air_launch.hpp"
#include "grav_dft.hpp"
#include "grav_plan.hpp"
#include "tmap.hpp"

using namespace tpt;

namespace {
constexpr uint32_t CHUNK = 1000;     // ticks per captured graph at most (even)
constexpr uint32_t TUNE_TICKS = 50;  // ticks of the graphs the autotuner times (even)
constexpr uint32_t MAX_DEPTH = 50;   // temporal depth at most
constexpr size_t ALIGN = 64;    // elements (256 B) between instances

enum F32 { F_PV, F_VX, F_VY, F_HV, F_PV2, F_VX2, F_VY2, F_HV2, F_OPV, F_OVX, F_OVY, F_FVX, F_FVY, F_GX, F_GY, F_N32 };
enum U32 { U_BA, U_BH, U_BA2, U_BH2, U_WALL, U_EMAP, U_EA, U_EH, U_GMASK, U_NU32 };

size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

// Where one instance's grid sits in the dense staging buffer (the
// reference's `cy * xcells + cx` layout, instances back to back) and in a
// pitched arena slot.
struct IoInst {
    size_t dense, arena;  // element offsets
    uint32_t xcells, ycells, pitch;
};

// Dense <-> pitched copy of one grid kind for instances base .. base +
// gridDim.y - 1: block (bx, k) copies rows bx, bx + gridDim.x, ... of
// instance base + k, the threads walking a row so both sides coalesce.
__global__ void k_batch_io(const IoInst *io, uint32_t base, uint32_t *arena, uint32_t *dense, int to_arena) {
    const IoInst I = io[base + blockIdx.y];
    for (uint32_t r = blockIdx.x; r < I.ycells; r += gridDim.x) {
        uint32_t *a = arena + I.arena + (size_t)r * I.pitch;
        uint32_t *d = dense + I.dense + (size_t)r * I.xcells;
        for (uint32_t c = threadIdx.x; c < I.xcells; c += blockDim.x) {
            if (to_arena)
                a[c] = d[c];
            else
                d[c] = a[c];
        }
    }
}
}  // namespace

// Default sweep shape: 224 lanes (a 400-column grid in two 200-column strips
// plus halos) by 64-row strips. Default tile form shape: 32 x 8 cells.
constexpr uint32_t DEFAULT_LANES = 224, DEFAULT_ROWS = 64;
constexpr uint32_t DEFAULT_TILE_X = 32, DEFAULT_TILE_Y = 8;

// Splits every instance into column strips of at most lanes - 2 * SW_H
// columns and row strips of about `rows` rows (sizes balanced within an
// instance), then packs the strips side by side into work items of `lanes`
// lanes: strips sorted by height, next fit, at most SW_MAXSEG per item. Items
// are returned largest first (the work queue hands them out in this order).
static std::vector<air::SweepItem> plan_sweep(const std::vector<tpt_instance_desc> &descs, uint32_t lanes,
                                              uint32_t rows) {
    struct Strip {
        uint32_t inst;
        uint16_t x0, nx, y0, ny;
    };
    std::vector<Strip> strips;
    const uint32_t maxw = lanes - 2 * air::SW_H;
    for (uint32_t i = 0; i < (uint32_t)descs.size(); ++i) {
        const uint32_t X = descs[i].air.xcells, Y = descs[i].air.ycells;
        const uint32_t nc = (X + maxw - 1) / maxw;
        const uint32_t nr = std::max<uint32_t>(1u, (Y + rows / 2) / rows);
        uint32_t x = 0;
        for (uint32_t k = 0; k < nc; ++k) {
            const uint32_t w = X / nc + (k < X % nc ? 1u : 0u);
            uint32_t y = 0;
            for (uint32_t j = 0; j < nr; ++j) {
                const uint32_t h = Y / nr + (j < Y % nr ? 1u : 0u);
                strips.push_back({i, (uint16_t)x, (uint16_t)w, (uint16_t)y, (uint16_t)h});
                y += h;
            }
            x += w;
        }
    }
    std::stable_sort(strips.begin(), strips.end(), [](const Strip &a, const Strip &b) {
        return a.ny != b.ny ? a.ny > b.ny : a.nx > b.nx;
    });
    std::vector<air::SweepItem> items;
    air::SweepItem cur{};
    uint32_t used = 0;
    for (const Strip &t : strips) {
        const uint32_t need = t.nx + 2u * air::SW_H;
        if (cur.nseg == (uint32_t)air::SW_MAXSEG || (cur.nseg && used + need > lanes)) {
            items.push_back(cur);
            cur = air::SweepItem{};
            used = 0;
        }
        air::SweepSeg &g = cur.seg[cur.nseg++];
        g.inst = t.inst;
        g.lane0 = (uint16_t)used;
        g.lanes = (uint16_t)need;
        g.x0 = t.x0;
        g.nx = t.nx;
        g.y0 = t.y0;
        g.ny = t.ny;
        cur.steps = std::max<uint32_t>(cur.steps, t.ny);
        used += need;
    }
    if (cur.nseg) items.push_back(cur);
    auto work = [](const air::SweepItem &it) {
        uint32_t lanes_used = 0;
        for (uint32_t k = 0; k < it.nseg; ++k) lanes_used += it.seg[k].lanes;
        return (uint64_t)(it.steps + 13u) * lanes_used;
    };
    std::stable_sort(items.begin(), items.end(),
                     [&](const air::SweepItem &a, const air::SweepItem &b) { return work(a) > work(b); });
    return items;
}

struct tpt_batch {
    uint32_t n = 0;
    int precision = TPT_PRECISION_FP32;
    std::vector<tpt_instance_desc> descs;
    std::vector<size_t> off;       // per-instance element offset (same in all arenas)
    std::vector<uint32_t> pitch;   // per-instance row stride (elements)
    size_t stride = 0;             // elements per grid slot of the arenas
    float *f32 = nullptr;
    uint32_t *u32 = nullptr;
    int32_t *i32 = nullptr;
    // two AirInst per instance for each form: the sweep form's (every state
    // grid in ping-pong halves) and the tile form's (pv/vx/vy in place; heat
    // and masks in ping-pong halves), and the tile form's tensor maps
    std::vector<AirInst> insts_host, insts_tile_host;
    AirInst *insts = nullptr;
    AirInst *insts_tile = nullptr;
    bool any_noupdate_heat = false;
    // AIR_TX x AIR_TY tiles (the sweep's pre-pass, the copy-back)
    air::TileRef *tiles = nullptr;
    uint32_t ntiles = 0;
    // the tile form at its current shape: tiles, tensor maps (boxes of the
    // shape) and the advection/heat pass's resident CTAs per SM
    const air::TileShape *shape = nullptr;
    air::TileRef *form_tiles = nullptr;
    uint32_t nform_tiles = 0;
    CUtensorMap *tmaps = nullptr;
    int tile_occupancy_a = 1, tile_occupancy_b = 1;  // resident CTAs per SM of pass A / pass B
    // temporal blocking (tuning.temporal_depth > 1): the B(t) + A(t + 1)
    // launches' tiles and tensor maps (their own box), built on first use
    air::TileRef *fused_tiles = nullptr;
    uint32_t nfused_tiles = 0;
    CUtensorMap *tmaps_fused = nullptr;
    int fused_occupancy = 0;
    uint32_t *tile_queue = nullptr;  // the two passes' work-queue counters
    // the sweep form of the air tick: work items (device), the queue counter
    // and the pre-pass flags ([2][n], zeroed at creation)
    air::SweepItem *items = nullptr;
    uint32_t nitems = 0;
    uint32_t *ctl = nullptr;
    uint32_t *want = nullptr;
    uint32_t sweep_lanes = 0, sweep_rows = 0;  // the shape the items are planned for
    bool any_grav = false;
    tpt_batch_tuning tuning{DEFAULT_TILE_X, DEFAULT_TILE_Y, 1, 0, 0, TPT_AIR_FORM_TILES, 1};
    int sweep_occupancy = 1;  // resident sweep CTAs per SM at sweep_lanes
    int sms = 148;
    gfft::FftSet fft;
    dft::DftSet dft;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    std::map<uint32_t, cudaGraphExec_t> graphs;
    // whole-batch grid I/O (tpt_batch_write_field / tpt_batch_read_field),
    // allocated by the first such call: the dense staging grid of every
    // instance back to back, and the per-instance placement table
    uint32_t *stage = nullptr;
    IoInst *io = nullptr;
    size_t dense_total = 0;  // cells of all instances

    float *f(int field, uint32_t i) const { return f32 + (size_t)field * stride + off[i]; }
    uint32_t *u(int field, uint32_t i) const { return u32 + (size_t)field * stride + off[i]; }
    // CTAs of the tile-walking launches (pre-pass, copy-back)
    uint32_t grid() const { return std::min<uint32_t>(ntiles, (uint32_t)sms * 4u); }
    air::SweepLaunch sweep() const {
        air::SweepLaunch L{};
        L.insts = insts;
        L.tiles = tiles;
        L.ntiles = ntiles;
        L.items = items;
        L.nitems = nitems;
        L.ninst = n;
        L.lanes = sweep_lanes;
        const uint32_t per_sm = tuning.ctas_per_sm ? tuning.ctas_per_sm : (uint32_t)sweep_occupancy;
        L.grid = std::max<uint32_t>(1u, std::min<uint32_t>(nitems, (uint32_t)sms * per_sm));
        L.prepass_grid = grid();
        L.ctl = ctl;
        L.want = want;
        return L;
    }
    // the tile form's persistent grid: ctas_per_sm per SM (0: as many as fit,
    // the residency of its advection/heat pass)
    uint32_t tile_grid(int occupancy) const {
        const uint32_t per_sm = tuning.ctas_per_sm ? tuning.ctas_per_sm : (uint32_t)occupancy;
        return std::max<uint32_t>(1u, std::min<uint32_t>(nform_tiles, (uint32_t)sms * per_sm));
    }
    uint32_t tile_grid_a() const { return tile_grid(tile_occupancy_a); }
    uint32_t tile_grid_b() const { return tile_grid(tile_occupancy_b); }
    bool sweep_form() const { return tuning.air_form == TPT_AIR_FORM_SWEEP; }
    const AirInst *form_insts() const { return sweep_form() ? insts : insts_tile; }
    uint32_t fused_grid() const {
        return std::max<uint32_t>(1u, std::min<uint32_t>(nfused_tiles, (uint32_t)sms * (uint32_t)fused_occupancy));
    }
    // `ticks` air ticks from the canonical state (tick 0 reads parity 0). The
    // tile form at temporal depth k runs blocks of k ticks as A(t0), k - 1
    // launches of B(t) + A(t + 1), and B(t0 + k - 1) with the block's
    // deferred emap decays; depth 1 is A, B per tick.
    int air_run(uint32_t ticks, cudaStream_t st) const {
        int rc = TPT_OK;
        if (sweep_form()) {
            for (uint32_t t = 0; t < ticks && rc == TPT_OK; ++t) rc = air::launch_sweep_tick(sweep(), t & 1u, st);
            return rc;
        }
        const uint32_t k = std::max<uint32_t>(1u, tuning.temporal_depth);
        for (uint32_t t = 0; t < ticks && rc == TPT_OK;) {
            const uint32_t n = std::min<uint32_t>(k, ticks - t);
            rc = shape->launch_a(insts_tile, tmaps, form_tiles, nform_tiles, tile_grid_a(), t & 1u, tile_queue,
                                 tuning.work_queue != 0, st);
            for (uint32_t j = 0; j + 1 < n && rc == TPT_OK; ++j) {
                const uint32_t p = (t + j) & 1u;
                rc = air::launch_fused_ba(insts_tile, tmaps_fused, fused_tiles, nfused_tiles, fused_grid(), p, j, st);
                if (rc == TPT_OK && any_noupdate_heat)
                    rc = shape->launch_settle(insts_tile, form_tiles, nform_tiles, tile_grid_b(), p, st);
            }
            if (rc == TPT_OK)
                rc = shape->launch_b(insts_tile, tmaps, form_tiles, nform_tiles, tile_grid_b(), (t + n - 1) & 1u, n - 1,
                                     any_noupdate_heat, tile_queue, tuning.work_queue != 0, st);
            t += n;
        }
        return rc;
    }
    int grav_solve(cudaStream_t st) const {
        return precision == TPT_PRECISION_FP32 ? fft.launch(st) : dft.launch(st);
    }

    void drop_graphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
    ~tpt_batch() {
        drop_graphs();
        cudaFree(f32);
        cudaFree(u32);
        cudaFree(i32);
        cudaFree(insts);
        cudaFree(insts_tile);
        cudaFree(tmaps);
        cudaFree(stage);
        cudaFree(io);
        cudaFree(tiles);
        cudaFree(form_tiles);
        cudaFree(fused_tiles);
        cudaFree(tmaps_fused);
        cudaFree(tile_queue);
        cudaFree(items);
        cudaFree(ctl);
        if (side) cudaStreamDestroy(side);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
};

// Records `ticks` field steps on `st` (no graph): air chain on st, gravity
// chain on the side stream, joined at the end.
static int record_ticks(tpt_batch *b, uint32_t ticks, cudaStream_t st) {
    int rc;
    if (b->any_grav) {
        TPT_CUDA(cudaEventRecord(b->fork, st));
        TPT_CUDA(cudaStreamWaitEvent(b->side, b->fork, 0));
        for (uint32_t t = 0; t < ticks; ++t) {
            rc = b->grav_solve(b->side);
            if (rc) return rc;
        }
    }
    rc = b->air_run(ticks, st);
    if (rc) return rc;
    if (ticks & 1u) {
        rc = air::launch_copy_back(b->form_insts(), b->tiles, b->ntiles, b->grid(), st);
        if (rc) return rc;
    }
    if (b->any_grav) {
        TPT_CUDA(cudaEventRecord(b->join, b->side));
        TPT_CUDA(cudaStreamWaitEvent(st, b->join, 0));
    }
    return TPT_OK;
}

static int graph_for(tpt_batch *b, uint32_t ticks, cudaGraphExec_t *out) {
    auto it = b->graphs.find(ticks);
    if (it != b->graphs.end()) {
        *out = it->second;
        return TPT_OK;
    }
    cudaStream_t cap;
    TPT_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int rc = TPT_OK;
    if (e == cudaSuccess) {
        rc = record_ticks(b, ticks, cap);
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        if (rc == TPT_OK && e2 != cudaSuccess) e = e2;
    }
    cudaStreamDestroy(cap);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        TPT_FAIL(TPT_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) TPT_FAIL(TPT_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    b->graphs[ticks] = ex;
    *out = ex;
    return TPT_OK;
}

static int field_ptr(tpt_batch *b, uint32_t i, int field, void **p) {
    switch (field) {
        case TPT_FIELD_PV: *p = b->f(F_PV, i); break;
        case TPT_FIELD_VX: *p = b->f(F_VX, i); break;
        case TPT_FIELD_VY: *p = b->f(F_VY, i); break;
        case TPT_FIELD_HV: *p = b->f(F_HV, i); break;
        case TPT_FIELD_BLOCK_AIR: *p = b->u(U_BA, i); break;
        case TPT_FIELD_BLOCK_AIRH: *p = b->u(U_BH, i); break;
        case TPT_FIELD_WALL_BMAP: *p = b->u(U_WALL, i); break;
        case TPT_FIELD_WALL_EMAP: *p = b->u(U_EMAP, i); break;
        case TPT_FIELD_ELEM_BLOCK_AIR: *p = b->u(U_EA, i); break;
        case TPT_FIELD_ELEM_BLOCK_AIRH: *p = b->u(U_EH, i); break;
        case TPT_FIELD_FAN_VX: *p = b->f(F_FVX, i); break;
        case TPT_FIELD_FAN_VY: *p = b->f(F_FVY, i); break;
        case TPT_FIELD_GRAV_MASS: *p = b->i32 + b->off[i]; break;
        case TPT_FIELD_GRAV_MASK: *p = b->u(U_GMASK, i); break;
        case TPT_FIELD_GX: *p = b->f(F_GX, i); break;
        case TPT_FIELD_GY: *p = b->f(F_GY, i); break;
        default: TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown field id %d", field);
    }
    return TPT_OK;
}

// Saved copy of the state arenas, for the calls that run trial ticks.
struct StateCopy {
    float *f = nullptr;
    uint32_t *u = nullptr;
    size_t fbytes = 0, ubytes = 0;
    int save(const tpt_batch *b, cudaStream_t st) {
        fbytes = b->stride * F_N32 * sizeof(float);
        ubytes = b->stride * U_NU32 * sizeof(uint32_t);
        TPT_CUDA(cudaMalloc(&f, fbytes));
        TPT_CUDA(cudaMalloc(&u, ubytes));
        TPT_CUDA(cudaMemcpyAsync(f, b->f32, fbytes, cudaMemcpyDeviceToDevice, st));
        TPT_CUDA(cudaMemcpyAsync(u, b->u32, ubytes, cudaMemcpyDeviceToDevice, st));
        return TPT_OK;
    }
    int restore(tpt_batch *b, cudaStream_t st) {
        TPT_CUDA(cudaMemcpyAsync(b->f32, f, fbytes, cudaMemcpyDeviceToDevice, st));
        TPT_CUDA(cudaMemcpyAsync(b->u32, u, ubytes, cudaMemcpyDeviceToDevice, st));
        TPT_CUDA(cudaStreamSynchronize(st));
        return TPT_OK;
    }
    ~StateCopy() {
        cudaFree(f);
        cudaFree(u);
    }
};

// Plans the sweep's work items for `lanes` x `rows` and uploads them; reads
// the sweep kernel's occupancy at that width.
static int set_sweep_shape(tpt_batch *b, uint32_t lanes, uint32_t rows) {
    std::vector<air::SweepItem> items = plan_sweep(b->descs, lanes, rows);
    int occ = 0;
    int rc = air::sweep_max_ctas_per_sm(lanes, &occ);
    if (rc) return rc;
    if (occ < 1) TPT_FAIL(TPT_ERR_UNSUPPORTED, "the sweep kernel does not fit an SM at %u lanes", lanes);
    air::SweepItem *d = nullptr;
    TPT_CUDA(cudaMalloc(&d, items.size() * sizeof(air::SweepItem)));
    cudaError_t e = cudaMemcpy(d, items.data(), items.size() * sizeof(air::SweepItem), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        TPT_FAIL(TPT_ERR_CUDA, "sweep item upload failed: %s", cudaGetErrorString(e));
    }
    cudaFree(b->items);
    b->items = d;
    b->nitems = (uint32_t)items.size();
    b->sweep_occupancy = occ;
    b->sweep_lanes = lanes;
    b->sweep_rows = rows;
    return TPT_OK;
}

// Tensor maps of every instance's grids that the tile form's launches stage,
// with boxes of box_w x box_h cells (TM_COUNT per instance), and the tile list
// of tiles tx x ty.
static int build_tile_maps(const tpt_batch *b, uint32_t tx, uint32_t ty, uint32_t box_w, uint32_t box_h,
                           std::vector<CUtensorMap> &tm, std::vector<air::TileRef> &tiles) {
    tm.assign((size_t)b->n * air::TM_COUNT, CUtensorMap{});
    tiles.clear();
    for (uint32_t i = 0; i < b->n; ++i) {
        const uint32_t X = b->descs[i].air.xcells, Y = b->descs[i].air.ycells, P = b->pitch[i];
        CUtensorMap *m = &tm[(size_t)i * air::TM_COUNT];
        struct Slot {
            int slot;
            const void *base;
            bool f;
        } slots[] = {
            {air::TM_PV, b->f(F_PV, i), true},         {air::TM_VX, b->f(F_VX, i), true},
            {air::TM_VY, b->f(F_VY, i), true},         {air::TM_OVX0, b->f(F_OVX, i), true},
            {air::TM_OVY0, b->f(F_OVY, i), true},      {air::TM_OPV0, b->f(F_OPV, i), true},
            {air::TM_OVX1, b->f(F_VX2, i), true},      {air::TM_OVY1, b->f(F_VY2, i), true},
            {air::TM_OPV1, b->f(F_PV2, i), true},      {air::TM_BA0, b->u(U_BA, i), false},
            {air::TM_BA1, b->u(U_BA2, i), false},      {air::TM_BH0, b->u(U_BH, i), false},
            {air::TM_BH1, b->u(U_BH2, i), false},      {air::TM_HV0, b->insts_tile_host[2 * (size_t)i].hv, true},
            {air::TM_HV1, b->insts_tile_host[2 * (size_t)i + 1].hv, true},
        };
        static_assert(sizeof(slots) / sizeof(slots[0]) == air::TM_COUNT, "every slot");
        for (const Slot &sl : slots) {
            int rc = make_grid_tmap(&m[sl.slot], sl.base, sl.f, X, Y, P, box_w, box_h);
            if (rc) return rc;
        }
        for (uint32_t y = 0; y * ty < Y; ++y)
            for (uint32_t x = 0; x * tx < X; ++x) tiles.push_back({i, (uint16_t)x, (uint16_t)y});
    }
    return TPT_OK;
}

// Uploads a tile list and its tensor maps, replacing *dt / *dm.
static int upload_tile_maps(const std::vector<CUtensorMap> &tm, const std::vector<air::TileRef> &tiles,
                            air::TileRef **dt_out, CUtensorMap **dm_out) {
    air::TileRef *dt = nullptr;
    CUtensorMap *dm = nullptr;
    cudaError_t e = cudaMalloc(&dt, tiles.size() * sizeof(air::TileRef));
    if (e == cudaSuccess) e = cudaMalloc(&dm, tm.size() * sizeof(CUtensorMap));
    if (e == cudaSuccess) e = cudaMemcpy(dt, tiles.data(), tiles.size() * sizeof(air::TileRef), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dm, tm.data(), tm.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(dt);
        cudaFree(dm);
        TPT_FAIL(TPT_ERR_CUDA, "tile form upload failed: %s", cudaGetErrorString(e));
    }
    cudaFree(*dt_out);
    cudaFree(*dm_out);
    *dt_out = dt;
    *dm_out = dm;
    return TPT_OK;
}

// Builds the tile form's tile list and tensor maps for tile shape `sh` (the
// boxes are the tile plus a 4-cell x and 3-cell y halo) and uploads them.
static int set_tile_shape(tpt_batch *b, const air::TileShape *sh) {
    int occ_a = 0, occ_b = 0;
    int rc = sh->prepare(&occ_a, &occ_b);
    if (rc) return rc;
    if (occ_a < 1 || occ_b < 1) TPT_FAIL(TPT_ERR_UNSUPPORTED, "the %ux%u tile kernels do not fit an SM", sh->tx, sh->ty);
    std::vector<air::TileRef> tiles;
    std::vector<CUtensorMap> tm;
    rc = build_tile_maps(b, sh->tx, sh->ty, sh->tx + 8, sh->ty + 6, tm, tiles);
    if (rc) return rc;
    rc = upload_tile_maps(tm, tiles, &b->form_tiles, &b->tmaps);
    if (rc) return rc;
    b->nform_tiles = (uint32_t)tiles.size();
    b->shape = sh;
    b->tile_occupancy_a = occ_a;
    b->tile_occupancy_b = occ_b;
    return TPT_OK;
}

// The temporally blocked launches' tiles and tensor maps (boxes of the tile
// plus an 8-cell x and 5-cell y halo), once per batch.
static int set_fused(tpt_batch *b) {
    if (b->fused_tiles) return TPT_OK;
    int occ = 0;
    int rc = air::fused_tile_prepare(&occ);
    if (rc) return rc;
    if (occ < 1) TPT_FAIL(TPT_ERR_UNSUPPORTED, "the temporally blocked air kernel does not fit an SM");
    std::vector<air::TileRef> tiles;
    std::vector<CUtensorMap> tm;
    rc = build_tile_maps(b, air::FUSED_TX, air::FUSED_TY, air::FUSED_TX + 16, air::FUSED_TY + 10, tm, tiles);
    if (rc) return rc;
    rc = upload_tile_maps(tm, tiles, &b->fused_tiles, &b->tmaps_fused);
    if (rc) return rc;
    b->nfused_tiles = (uint32_t)tiles.size();
    b->fused_occupancy = occ;
    return TPT_OK;
}

extern "C" {

int tpt_batch_create(uint32_t n, const tpt_instance_desc *descs, int precision, tpt_batch **out) {
    if (!out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_create: out is NULL");
    *out = nullptr;
    if (n == 0) TPT_FAIL(TPT_ERR_INVALID_DIMS, "tpt_batch_create: no instances");
    if (!descs) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_create: descs is NULL");
    if (precision != TPT_PRECISION_FP32 && precision != TPT_PRECISION_SPLIT_BF16)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown precision %d", precision);
    for (uint32_t i = 0; i < n; ++i) {
        const tpt_air_params &p = descs[i].air;
        if (p.xcells < 3 || p.ycells < 3 || p.xcells > TPT_MAX_CELLS_PER_SIDE || p.ycells > TPT_MAX_CELLS_PER_SIDE)
            TPT_FAIL(TPT_ERR_INVALID_DIMS, "instance %u: grid %ux%u outside 3..%u", i, p.xcells, p.ycells,
                     TPT_MAX_CELLS_PER_SIDE);
        if (p.air_mode > 4u || p.convection_mode > 2u || p.gravity_mode > 3u || p.aheat_enable > 1u)
            TPT_FAIL(TPT_ERR_INVALID_ARG, "instance %u: enum field out of range", i);
    }
    int rc = require_sm100();
    if (rc) return rc;
    if (!tensor_map_encoder()) TPT_FAIL(TPT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
    tpt_batch *b = new (std::nothrow) tpt_batch();
    if (!b) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    auto bail = [&](int code) {
        delete b;
        return code;
    };
    b->n = n;
    b->precision = precision;
    b->descs.assign(descs, descs + n);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    size_t total = 0;
    b->off.resize(n);
    b->pitch.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        b->pitch[i] = (uint32_t)round_up(descs[i].air.xcells, 32);
        b->off[i] = total;
        total += round_up((size_t)b->pitch[i] * descs[i].air.ycells, ALIGN);
    }
    b->stride = total;
    cudaError_t e = cudaMalloc(&b->f32, total * F_N32 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->u32, total * U_NU32 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->i32, total * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(b->f32, 0, total * F_N32 * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(b->u32, 0, total * U_NU32 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(b->i32, 0, total * sizeof(int32_t));
    if (e != cudaSuccess) {
        set_error("batch arena allocation (%zu cells) failed: %s", total, cudaGetErrorString(e));
        return bail(e == cudaErrorMemoryAllocation ? TPT_ERR_OUT_OF_MEMORY : TPT_ERR_CUDA);
    }
    // two AirInst per instance: parity 0 reads canonical hv/masks and writes
    // the second copies; parity 1 the reverse.
    std::vector<air::TileRef> tiles;
    b->insts_host.resize(2 * (size_t)n);
    b->insts_tile_host.resize(2 * (size_t)n);
    std::vector<JobShape> gshapes;
    std::vector<uint32_t> gidx;
    for (uint32_t i = 0; i < n; ++i) {
        const tpt_air_params &p = descs[i].air;
        AirInst I = make_air_inst(p);
        I.pitch = b->pitch[i];
        I.opv = b->f(F_OPV, i);
        I.ovx = b->f(F_OVX, i);
        I.ovy = b->f(F_OVY, i);
        I.ohv = nullptr;
        I.wall = b->u(U_WALL, i);
        I.emap = b->u(U_EMAP, i);
        I.eair = b->u(U_EA, i);
        I.eairh = b->u(U_EH, i);
        I.fvx = b->f(F_FVX, i);
        I.fvy = b->f(F_FVY, i);
        for (int par = 0; par < 2; ++par) {
            AirInst J = I;
            J.pv = b->f(par ? F_PV2 : F_PV, i);
            J.vx = b->f(par ? F_VX2 : F_VX, i);
            J.vy = b->f(par ? F_VY2 : F_VY, i);
            J.pv_out = b->f(par ? F_PV : F_PV2, i);
            J.vx_out = b->f(par ? F_VX : F_VX2, i);
            J.vy_out = b->f(par ? F_VY : F_VY2, i);
            if (p.aheat_enable) {
                J.hv = b->f(par ? F_HV2 : F_HV, i);
                J.hv_out = b->f(par ? F_HV : F_HV2, i);
            } else {  // heat never changes: one buffer for both halves
                J.hv = J.hv_out = b->f(F_HV, i);
            }
            J.bair = b->u(par ? U_BA2 : U_BA, i);
            J.bairh = b->u(par ? U_BH2 : U_BH, i);
            J.bair_out = b->u(par ? U_BA : U_BA2, i);
            J.bairh_out = b->u(par ? U_BH : U_BH2, i);
            b->insts_host[2 * (size_t)i + par] = J;
            // the tile form: pv/vx/vy in their canonical buffers, updated in place
            AirInst T = J;
            T.pv = b->f(F_PV, i);
            T.vx = b->f(F_VX, i);
            T.vy = b->f(F_VY, i);
            T.pv_out = T.vx_out = T.vy_out = nullptr;
            // the velocity pass's outputs alternate between two sets by tick
            // parity (the sweep's ping-pong halves serve as the second set)
            T.opv = b->f(par ? F_PV2 : F_OPV, i);
            T.ovx = b->f(par ? F_VX2 : F_OVX, i);
            T.ovy = b->f(par ? F_VY2 : F_OVY, i);
            b->insts_tile_host[2 * (size_t)i + par] = T;
        }
        if (p.air_mode == 4u && p.aheat_enable) b->any_noupdate_heat = true;
        for (uint32_t ty = 0; ty * AIR_TY < p.ycells; ++ty)
            for (uint32_t tx = 0; tx * AIR_TX < p.xcells; ++tx) tiles.push_back({i, (uint16_t)tx, (uint16_t)ty});
        if (descs[i].newton_grav) {
            gshapes.push_back({p.xcells, p.ycells});
            gidx.push_back(i);
        }
    }
    b->ntiles = (uint32_t)tiles.size();
    e = cudaMalloc(&b->insts, b->insts_host.size() * sizeof(AirInst));
    if (e == cudaSuccess) e = cudaMalloc(&b->insts_tile, b->insts_tile_host.size() * sizeof(AirInst));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->insts_tile, b->insts_tile_host.data(), b->insts_tile_host.size() * sizeof(AirInst),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->tiles, tiles.size() * sizeof(air::TileRef));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->insts, b->insts_host.data(), b->insts_host.size() * sizeof(AirInst), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->tiles, tiles.data(), tiles.size() * sizeof(air::TileRef), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->tile_queue, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(b->tile_queue, 0, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->ctl, (1 + 2 * (size_t)n) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(b->ctl, 0, (1 + 2 * (size_t)n) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        set_error("batch setup failed: %s", cudaGetErrorString(e));
        return bail(TPT_ERR_CUDA);
    }
    b->want = b->ctl + 1;
    rc = set_tile_shape(b, air::tile_shape(DEFAULT_TILE_X, DEFAULT_TILE_Y));
    if (rc) return bail(rc);
    rc = set_sweep_shape(b, DEFAULT_LANES, DEFAULT_ROWS);
    if (rc) return bail(rc);
    b->any_grav = !gshapes.empty();
    if (b->any_grav) {
        if (precision == TPT_PRECISION_FP32) {
            rc = b->fft.create(gshapes);
            if (rc) return bail(rc);
            for (size_t j = 0; j < gidx.size(); ++j) {
                uint32_t i = gidx[j];
                b->fft.set_io(j, b->i32 + b->off[i], nullptr, 1.0f / 65536.0f, b->u(U_GMASK, i), b->f(F_GX, i),
                              b->f(F_GY, i), b->pitch[i]);
            }
            rc = b->fft.upload_jobs();
        } else {
            rc = b->dft.create(gshapes);
            for (size_t j = 0; rc == TPT_OK && j < gidx.size(); ++j) {
                uint32_t i = gidx[j];
                dft::SolveIO io{b->i32 + b->off[i], nullptr, b->u(U_GMASK, i), b->f(F_GX, i), b->f(F_GY, i),
                                1.0f / 65536.0f, b->pitch[i]};
                rc = b->dft.set_io(j, io);
            }
        }
        if (rc) return bail(rc);
    }
    *out = b;
    return TPT_OK;
}

int tpt_batch_destroy(tpt_batch *b) {
    delete b;
    return TPT_OK;
}

int tpt_batch_fields(tpt_batch *b, uint32_t i, tpt_instance_fields *o) {
    if (!b || !o) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_fields: NULL pointer");
    if (i >= b->n) TPT_FAIL(TPT_ERR_INVALID_ARG, "instance %u out of range (batch of %u)", i, b->n);
    o->pv = b->f(F_PV, i);
    o->vx = b->f(F_VX, i);
    o->vy = b->f(F_VY, i);
    o->hv = b->f(F_HV, i);
    o->block_air = b->u(U_BA, i);
    o->block_airh = b->u(U_BH, i);
    o->wall_bmap = b->u(U_WALL, i);
    o->wall_emap = b->u(U_EMAP, i);
    o->elem_block_air = b->u(U_EA, i);
    o->elem_block_airh = b->u(U_EH, i);
    o->fan_vx = b->f(F_FVX, i);
    o->fan_vy = b->f(F_FVY, i);
    o->grav_mass = b->i32 + b->off[i];
    o->grav_mask = b->u(U_GMASK, i);
    o->gx = b->f(F_GX, i);
    o->gy = b->f(F_GY, i);
    o->pitch = b->pitch[i];
    return TPT_OK;
}

// Copies between a dense host grid (xcells per row) and the pitched grid.
static int batch_copy(tpt_batch *b, uint32_t i, int field, void *host, size_t bytes, bool to_device,
                      tpt_stream_t stream) {
    if (!b || !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_%s: NULL pointer", to_device ? "write" : "read");
    if (i >= b->n) TPT_FAIL(TPT_ERR_INVALID_ARG, "instance %u out of range", i);
    const size_t X = b->descs[i].air.xcells, Y = b->descs[i].air.ycells;
    if (bytes != X * Y * 4) TPT_FAIL(TPT_ERR_INVALID_ARG, "bytes %zu != %zu cells * 4", bytes, X * Y);
    void *p;
    int rc = field_ptr(b, i, field, &p);
    if (rc) return rc;
    const size_t dpitch = (size_t)b->pitch[i] * 4;
    if (to_device) {
        TPT_CUDA(cudaMemcpy2DAsync(p, dpitch, host, X * 4, X * 4, Y, cudaMemcpyHostToDevice, (cudaStream_t)stream));
    } else {
        TPT_CUDA(cudaMemcpy2DAsync(host, X * 4, p, dpitch, X * 4, Y, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    }
    return TPT_OK;
}

int tpt_batch_write(tpt_batch *b, uint32_t i, int field, const void *host, size_t bytes, tpt_stream_t stream) {
    return batch_copy(b, i, field, const_cast<void *>(host), bytes, true, stream);
}

int tpt_batch_read(tpt_batch *b, uint32_t i, int field, void *host, size_t bytes, tpt_stream_t stream) {
    return batch_copy(b, i, field, host, bytes, false, stream);
}

// The staging buffer and placement table of the whole-batch calls.
static int ensure_io(tpt_batch *b) {
    if (b->stage) return TPT_OK;
    std::vector<IoInst> io(b->n);
    size_t dense = 0;
    for (uint32_t i = 0; i < b->n; ++i) {
        io[i] = {dense, b->off[i], b->descs[i].air.xcells, b->descs[i].air.ycells, b->pitch[i]};
        dense += (size_t)io[i].xcells * io[i].ycells;
    }
    cudaError_t e = cudaMalloc(&b->io, io.size() * sizeof(IoInst));
    if (e == cudaSuccess) e = cudaMemcpy(b->io, io.data(), io.size() * sizeof(IoInst), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->stage, dense * sizeof(uint32_t));
    if (e != cudaSuccess) {
        cudaFree(b->io);
        cudaFree(b->stage);
        b->io = nullptr;
        b->stage = nullptr;
        set_error("staging buffer of %zu cells: %s", dense, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? TPT_ERR_OUT_OF_MEMORY : TPT_ERR_CUDA;
    }
    b->dense_total = dense;
    return TPT_OK;
}

// One grid kind of every instance between a dense host buffer and the arena:
// one host copy of the whole buffer plus one scatter or gather launch.
static int batch_copy_field(tpt_batch *b, int field, void *host, size_t bytes, bool to_device,
                            tpt_stream_t stream) {
    const char *name = to_device ? "tpt_batch_write_field" : "tpt_batch_read_field";
    if (!b || !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "%s: NULL pointer", name);
    void *base;
    int rc = field_ptr(b, 0, field, &base);  // instance 0 starts its arena slot
    if (rc) return rc;
    rc = ensure_io(b);
    if (rc) return rc;
    if (bytes != b->dense_total * 4)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "%s: bytes %zu != %zu cells * 4", name, bytes, b->dense_total);
    cudaStream_t st = (cudaStream_t)stream;
    if (to_device) TPT_CUDA(cudaMemcpyAsync(b->stage, host, bytes, cudaMemcpyHostToDevice, st));
    uint32_t maxy = 1;
    for (const auto &d : b->descs) maxy = std::max(maxy, d.air.ycells);
    for (uint32_t first = 0; first < b->n; first += 65535u) {
        const uint32_t k = std::min<uint32_t>(b->n - first, 65535u);
        const uint32_t bx = std::min<uint32_t>(maxy, std::max<uint32_t>(1u, (uint32_t)b->sms * 8u / k));
        k_batch_io<<<dim3(bx, k), 128, 0, st>>>(b->io, first, (uint32_t *)base, b->stage, to_device ? 1 : 0);
        TPT_LAUNCHED();
    }
    if (!to_device) TPT_CUDA(cudaMemcpyAsync(host, b->stage, bytes, cudaMemcpyDeviceToHost, st));
    return TPT_OK;
}

int tpt_batch_write_field(tpt_batch *b, int field, const void *host, size_t bytes, tpt_stream_t stream) {
    return batch_copy_field(b, field, const_cast<void *>(host), bytes, true, stream);
}

int tpt_batch_read_field(tpt_batch *b, int field, void *host, size_t bytes, tpt_stream_t stream) {
    return batch_copy_field(b, field, host, bytes, false, stream);
}

int tpt_batch_step(tpt_batch *b, uint32_t ticks, tpt_stream_t stream) {
    if (!b) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_step: batch is NULL");
    if (ticks == 0) return TPT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t full = ticks / CHUNK, rest = ticks % CHUNK;
    cudaGraphExec_t g;
    int rc;
    if (full) {
        rc = graph_for(b, CHUNK, &g);
        if (rc) return rc;
        for (uint32_t c = 0; c < full; ++c) {
            TPT_CUDA(cudaGraphLaunch(g, st));
        }
    }
    if (rest) {
        rc = graph_for(b, rest, &g);
        if (rc) return rc;
        TPT_CUDA(cudaGraphLaunch(g, st));
    }
    return TPT_OK;
}

int tpt_batch_get_tuning(const tpt_batch *b, tpt_batch_tuning *t) {
    if (!b || !t) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_get_tuning: NULL pointer");
    *t = b->tuning;
    return TPT_OK;
}

int tpt_batch_set_tuning(tpt_batch *b, const tpt_batch_tuning *t) {
    if (!b || !t) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_set_tuning: NULL pointer");
    if (t->air_form != TPT_AIR_FORM_TILES && t->air_form != TPT_AIR_FORM_SWEEP)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "air_form %u is neither TPT_AIR_FORM_TILES nor TPT_AIR_FORM_SWEEP", t->air_form);
    const bool sweep = t->air_form == TPT_AIR_FORM_SWEEP;
    const air::TileShape *sh = nullptr;
    if (sweep) {
        if (t->tile_x < 64 || t->tile_x > (uint32_t)air::SWEEP_MAX_LANES || t->tile_x % 32u)
            TPT_FAIL(TPT_ERR_INVALID_ARG, "tile_x (sweep lanes) %u must be a multiple of 32 in 64..%d", t->tile_x,
                     air::SWEEP_MAX_LANES);
        if (t->tile_y < 8 || t->tile_y > TPT_MAX_CELLS_PER_SIDE)
            TPT_FAIL(TPT_ERR_INVALID_ARG, "tile_y (rows per strip) %u must be in 8..%u", t->tile_y,
                     TPT_MAX_CELLS_PER_SIDE);
    } else {
        sh = air::tile_shape(t->tile_x, t->tile_y);
        if (!sh)
            TPT_FAIL(TPT_ERR_INVALID_ARG, "tile %ux%u is not a tile form shape (32x8, 64x8, 32x16, 64x16)", t->tile_x,
                     t->tile_y);
    }
    if (t->temporal_depth < 1 || t->temporal_depth > MAX_DEPTH)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "temporal_depth %u must be in 1..%u", t->temporal_depth, MAX_DEPTH);
    if (sweep && t->temporal_depth != 1)
        TPT_FAIL(TPT_ERR_UNSUPPORTED, "temporal blocking is built for the tile form; the sweep form takes depth 1");
    if (t->ctas_per_sm > 32) TPT_FAIL(TPT_ERR_INVALID_ARG, "ctas_per_sm must be 0 (as many as fit) .. 32");
    if (t->work_queue > 1u) TPT_FAIL(TPT_ERR_INVALID_ARG, "work_queue must be 0 (static striding) or 1 (queue)");
    const bool split = b->any_grav && b->precision == TPT_PRECISION_SPLIT_BF16 && b->dft.can_split();
    if (t->grav_side_ctas && !split)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "grav_side_ctas must be 0: the batch's gravity has one kind of y stage");
    if (sweep && (t->tile_x != b->sweep_lanes || t->tile_y != b->sweep_rows)) {
        int rc = set_sweep_shape(b, t->tile_x, t->tile_y);
        if (rc) return rc;
    }
    if (sweep && t->ctas_per_sm > (uint32_t)b->sweep_occupancy)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "ctas_per_sm %u exceeds the %d sweep CTAs of %u lanes that fit an SM",
                 t->ctas_per_sm, b->sweep_occupancy, t->tile_x);
    if (!sweep && sh != b->shape) {
        int rc = set_tile_shape(b, sh);
        if (rc) return rc;
    }
    if (t->temporal_depth > 1) {
        int rc = set_fused(b);
        if (rc) return rc;
    }
    if (split) {
        int rc = b->dft.set_side_ctas(t->grav_side_ctas);
        if (rc) return rc;
    }
    b->drop_graphs();
    b->tuning = *t;
    return TPT_OK;
}

int tpt_batch_profile_phases(tpt_batch *b, uint32_t ticks, tpt_stream_t stream, tpt_batch_profile *out) {
    if (!b || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_profile_phases: NULL pointer");
    if (ticks == 0 || (ticks & 1u)) TPT_FAIL(TPT_ERR_INVALID_ARG, "ticks must be even and > 0");
    cudaStream_t st = (cudaStream_t)stream;
    StateCopy saved;
    int rc = saved.save(b, st);
    if (rc) return rc;
    memset(out, 0, sizeof(*out));
    out->ticks = ticks;
    for (uint32_t i = 0; i < b->n; ++i) {
        uint64_t c = (uint64_t)b->descs[i].air.xcells * b->descs[i].air.ycells;
        out->cells += c;
        if (b->descs[i].newton_grav) out->grav_cells += c;
    }
    // sweep form: velocity pre-pass (flagged instances only) + sweep; tile
    // form: pass A + pass B (+ a settle pass when an instance is NoUpdate with
    // ambient heat)
    out->air_launches_per_tick = b->sweep_form() ? 2 : (b->any_noupdate_heat ? 3 : 2);
    out->grav_launches_per_tick = b->any_grav ? (b->precision == TPT_PRECISION_FP32 ? 3 : b->dft.launches()) : 0;
    out->grav_flops_per_tick = b->any_grav && b->precision != TPT_PRECISION_FP32 ? b->dft.flops() : 0.0;
    cudaEvent_t e0, e1, e2;
    TPT_CUDA(cudaEventCreate(&e0));
    TPT_CUDA(cudaEventCreate(&e1));
    TPT_CUDA(cudaEventCreate(&e2));
    if (rc == TPT_OK) rc = b->air_run(2, st);  // warm-up
    cudaEventRecord(e0, st);
    if (rc == TPT_OK) rc = b->air_run(ticks, st);
    cudaEventRecord(e1, st);
    for (uint32_t t = 0; t < ticks && rc == TPT_OK && b->any_grav; ++t) rc = b->grav_solve(st);
    cudaEventRecord(e2, st);
    if (rc == TPT_OK) {
        cudaEventSynchronize(e2);
        cudaEventElapsedTime(&out->air_ms, e0, e1);
        cudaEventElapsedTime(&out->grav_ms, e1, e2);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    int rc2 = saved.restore(b, st);
    return rc ? rc : rc2;
}

// Tuned settings per batch composition: the shapes' (W, H) buckets
// (powers of two) with their counts, and the gravity precision. A batch whose
// instances fall in the same buckets reuses the tuned settings without
// timing.
struct TuneKey {
    int precision;
    std::vector<std::pair<uint32_t, uint32_t>> buckets;  // (log2 W << 8 | log2 H, count), sorted
    bool operator<(const TuneKey &o) const {
        return precision != o.precision ? precision < o.precision : buckets < o.buckets;
    }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, tpt_batch_tuning> g_tune_cache;

static uint32_t log2_bucket(uint32_t v) {
    uint32_t k = 0;
    while ((2u << k) <= v) ++k;
    return k;
}

static TuneKey tune_key(const tpt_batch *b) {
    std::map<uint32_t, uint32_t> h;
    for (const auto &d : b->descs) ++h[log2_bucket(d.air.xcells) << 8 | log2_bucket(d.air.ycells)];
    TuneKey k;
    k.precision = b->any_grav ? b->precision : -1;
    k.buckets.assign(h.begin(), h.end());
    return k;
}

int tpt_batch_tune(tpt_batch *b, tpt_stream_t stream) {
    if (!b) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_batch_tune: batch is NULL");
    const TuneKey key = tune_key(b);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return tpt_batch_set_tuning(b, &it->second);
    }
    cudaStream_t st = (cudaStream_t)stream;
    StateCopy saved;
    int src = saved.save(b, st);
    if (src) return src;
    // Phase 1: the air form and its layout, by timing 20 air ticks of each
    // candidate: the tile form at every tile shape, with static striding and
    // with the atomic work queue, at each pass's own residency (0) and at 4,
    // 6 and 8 CTAs per SM (32x8; the larger tiles at 0 and 2); the sweep form
    // at a few shapes (lanes per CTA x rows per strip) with as many CTAs as
    // fit.
    struct Cand {
        uint32_t form, x, y, per_sm, queue;
    };
    std::vector<Cand> cands;
    for (int k = 0; k < air::TILE_SHAPES; ++k) {
        const air::TileShape *sh = air::tile_shapes()[k];
        const bool base = sh->tx == DEFAULT_TILE_X && sh->ty == DEFAULT_TILE_Y;
        for (uint32_t q : {1u, 0u})
            for (uint32_t c : base ? std::vector<uint32_t>{0u, 4u, 6u, 8u} : std::vector<uint32_t>{0u, 2u})
                cands.push_back({TPT_AIR_FORM_TILES, sh->tx, sh->ty, c, q});
    }
    for (auto sh : {std::make_pair(224u, 64u), std::make_pair(256u, 64u), std::make_pair(256u, 32u)})
        cands.push_back({TPT_AIR_FORM_SWEEP, sh.first, sh.second, 0u, 0u});
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    tpt_batch_tuning best = b->tuning;
    float best_ms = 1e30f;
    int rc = TPT_OK;
    std::vector<std::pair<float, tpt_batch_tuning>> timed;  // phase 1's air-only times
    for (const Cand &cd : cands) {
        tpt_batch_tuning t = b->tuning;
        t.air_form = cd.form;
        t.tile_x = cd.x;
        t.tile_y = cd.y;
        t.ctas_per_sm = cd.per_sm;
        t.temporal_depth = 1;
        t.work_queue = cd.queue;
        rc = tpt_batch_set_tuning(b, &t);
        if (rc) break;
        const uint32_t trial = 20;
        for (int rep = 0; rep < 2 && rc == TPT_OK; ++rep) {  // warm-up, then timed
            cudaEventRecord(e0, st);
            rc = b->air_run(trial, st);
            cudaEventRecord(e1, st);
        }
        if (rc) break;
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        timed.push_back({ms, t});
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    // Phase 1b, for the tile form at the chosen layout, on the same 20 ticks:
    // the temporal depth (ticks per block of fused B(t) + A(t + 1) launches).
    for (uint32_t depth : {2u, 4u, 10u, 20u}) {
        if (rc || best.air_form != TPT_AIR_FORM_TILES) break;
        tpt_batch_tuning t = best;
        t.temporal_depth = depth;
        rc = tpt_batch_set_tuning(b, &t);
        if (rc) break;
        for (int rep = 0; rep < 2 && rc == TPT_OK; ++rep) {  // warm-up, then timed
            cudaEventRecord(e0, st);
            rc = b->air_run(20, st);
            cudaEventRecord(e1, st);
        }
        if (rc) break;
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    // Phase 2, for batches with gravity: the whole step -- a graph of
    // TUNE_TICKS ticks as a step captures it, air and gravity chains
    // together -- since the gravity
    // chain runs on the SMs the air launches leave idle, the air layout that
    // is fastest alone need not be fastest beside it. Finalists: the air
    // settings within 5% of the fastest air-only time (at most four), each
    // with every gravity split (CTAs of the DFT-pair groups' branch on its
    // own stream, as a percentage of the SMs; 0 = one stream) when the batch
    // has both kinds of y stage.
    if (rc == TPT_OK && b->any_grav) {
        std::stable_sort(timed.begin(), timed.end(),
                         [](const std::pair<float, tpt_batch_tuning> &x, const std::pair<float, tpt_batch_tuning> &y) {
                             return x.first < y.first;
                         });
        std::vector<tpt_batch_tuning> finalists{best};
        for (const auto &tt : timed) {
            if (finalists.size() >= 4 || tt.first > 1.05f * timed.front().first) break;
            if (memcmp(&tt.second, &best, sizeof(best)) != 0) finalists.push_back(tt.second);
        }
        const bool split = b->precision == TPT_PRECISION_SPLIT_BF16 && b->dft.can_split();
        const uint32_t cap = split ? b->dft.max_side_ctas() : 0u;
        std::vector<uint32_t> pcts{0u};
        if (split)
            for (uint32_t pct : {10u, 15u, 20u, 25u, 33u, 40u, 50u}) pcts.push_back(pct);
        float step_best = 1e30f;
        tpt_batch_tuning chosen = best;
        for (const tpt_batch_tuning &fin : finalists) {
            for (uint32_t pct : pcts) {
                if (rc) break;
                tpt_batch_tuning t = fin;
                t.grav_side_ctas =
                    pct ? std::min<uint32_t>(cap, std::max<uint32_t>(1u, (uint32_t)b->sms * pct / 100u)) : 0u;
                rc = tpt_batch_set_tuning(b, &t);
                cudaGraphExec_t ex = nullptr;
                if (rc == TPT_OK) rc = graph_for(b, TUNE_TICKS, &ex);
                float ms = 1e30f;
                for (int rep = 0; rep < 3 && rc == TPT_OK; ++rep) {  // warm-up, then the faster of two
                    cudaEventRecord(e0, st);
                    if (cudaGraphLaunch(ex, st) != cudaSuccess) {
                        set_error("graph launch failed while tuning");
                        rc = TPT_ERR_CUDA;
                    }
                    cudaEventRecord(e1, st);
                    cudaEventSynchronize(e1);
                    float r = 0;
                    cudaEventElapsedTime(&r, e0, e1);
                    if (rep > 0 && r < ms) ms = r;
                }
                if (rc) break;
                if (ms < step_best) {
                    step_best = ms;
                    chosen = t;
                }
            }
        }
        best = chosen;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rrc = saved.restore(b, st);
    if (rc) return rc;
    if (rrc) return rrc;
    rc = tpt_batch_set_tuning(b, &best);
    if (rc == TPT_OK) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = best;
    }
    return rc;
}

}  // extern "C"
