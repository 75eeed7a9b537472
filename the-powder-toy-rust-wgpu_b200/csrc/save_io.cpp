// save_io.cpp -- `.tptrs` save files on the host (crates/tpt-save/src/lib.rs):
// the 8-byte magic "TPTRS001", then zlib(bincode(SaveData)).
//
// bincode 1.3.3 with its default options (what `bincode::serialize` /
// `bincode::deserialize` use): little-endian fixed-width integers and floats,
// a u64 element count before a vector and a u64 byte count before a string,
// a u32 variant index for an enum, one byte 0/1 for a bool (other values are
// an error) and for an Option's presence, struct fields in declaration order
// with `#[serde(skip)]` fields left out, trailing bytes after the value
// ignored.
#include <stdint.h>
#include <string.h>
#include <zlib.h>

#include <new>
#include <vector>

#include "common.cuh"

struct tpt_save {
    uint32_t version = TPT_SAVE_VERSION;
    tpt_save_config config{};
    std::vector<uint8_t> particles;       // n * 64 bytes, the bincode of each GpuParticle
    std::vector<uint32_t> grid[TPT_SAVE_GRIDS];  // f32 grids as their bit patterns
    std::vector<uint8_t> rigid, signs;    // the encoded elements, kept as read
    uint64_t n_rigid = 0, n_signs = 0;
    std::vector<uint8_t> encoded;         // the last tpt_save_encode result
};

namespace {

using tpt::set_error;

// ------------------------------------------------------------- writer ----
struct Writer {
    std::vector<uint8_t> b;
    void bytes(const void *p, size_t n) { b.insert(b.end(), (const uint8_t *)p, (const uint8_t *)p + n); }
    void u8(uint8_t v) { b.push_back(v); }
    void u32(uint32_t v) {
        const uint8_t x[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
        bytes(x, 4);
    }
    void i32(int32_t v) { u32((uint32_t)v); }
    void f32(float v) {
        uint32_t u;
        memcpy(&u, &v, 4);
        u32(u);
    }
    void u64(uint64_t v) {
        u32((uint32_t)v);
        u32((uint32_t)(v >> 32));
    }
    void boolean(uint8_t v) { u8(v ? 1 : 0); }
    void opt_f32(uint8_t has, float v) {
        u8(has ? 1 : 0);
        if (has) f32(v);
    }
};

// ------------------------------------------------------------- reader ----
// Every read checks the remaining length; the first failure sticks.
struct Reader {
    const uint8_t *p;
    size_t n, i = 0;
    const char *err = nullptr;
    bool fail(const char *what) {
        if (!err) err = what;
        return false;
    }
    bool take(void *dst, size_t k) {
        if (err) return false;
        if (n - i < k) return fail("unexpected end of the payload");
        memcpy(dst, p + i, k);
        i += k;
        return true;
    }
    bool u8(uint8_t &v) { return take(&v, 1); }
    bool u32(uint32_t &v) {
        uint8_t x[4];
        if (!take(x, 4)) return false;
        v = (uint32_t)x[0] | (uint32_t)x[1] << 8 | (uint32_t)x[2] << 16 | (uint32_t)x[3] << 24;
        return true;
    }
    bool i32(int32_t &v) {
        uint32_t u;
        if (!u32(u)) return false;
        v = (int32_t)u;
        return true;
    }
    bool f32(float &v) {
        uint32_t u;
        if (!u32(u)) return false;
        memcpy(&v, &u, 4);
        return true;
    }
    bool u64(uint64_t &v) {
        uint32_t lo, hi;
        if (!u32(lo) || !u32(hi)) return false;
        v = (uint64_t)hi << 32 | lo;
        return true;
    }
    bool boolean(uint8_t &v) {
        if (!u8(v)) return false;
        if (v > 1) return fail("invalid bool byte");
        return true;
    }
    bool variant(uint32_t &v, uint32_t count) {
        if (!u32(v)) return false;
        if (v >= count) return fail("invalid enum variant index");
        return true;
    }
    bool opt_f32(uint8_t &has, float &v) {
        if (!u8(has)) return false;
        if (has > 1) return fail("invalid Option tag");
        v = 0.0f;
        return has ? f32(v) : true;
    }
    // A vector's element count, checked against the bytes left.
    bool count(uint64_t &c, size_t min_elem_bytes) {
        if (!u64(c)) return false;
        if (min_elem_bytes && c > (n - i) / min_elem_bytes) return fail("vector length beyond the payload");
        return true;
    }
};

// SimulationConfig (particle.rs:166-222); mod_elements_enabled is
// #[serde(skip)] and not in the stream.
void put_config(Writer &w, const tpt_save_config &c) {
    w.u32(c.xres);
    w.u32(c.yres);
    w.boolean(c.paused);
    w.boolean(c.aheat_enable);
    w.boolean(c.pretty_powder);
    w.u32(c.edge_mode);
    w.u32(c.gravity_mode);
    w.u32(c.air_mode);
    w.f32(c.ambient_air_temp);
    w.f32(c.edge_pressure);
    w.u32(c.display_mode);
    w.u32(c.colour_mode);
    w.u32(c.render_mode);
    w.f32(c.fire_intensity);
    w.boolean(c.heat_enable);
    w.boolean(c.newton_grav);
    w.boolean(c.water_equal_test);
    w.f32(c.vorticity_coeff);
    w.u32(c.convection_mode);
    w.f32(c.edge_velocity_x);
    w.f32(c.edge_velocity_y);
    w.f32(c.custom_gravity_x);
    w.f32(c.custom_gravity_y);
    w.u32(c.temperature_scale);
    w.boolean(c.decorations);
    w.i32(c.mouse_x);
    w.i32(c.mouse_y);
    w.boolean(c.gravity_field_enabled);
    w.boolean(c.gravity_zones_enabled);
    w.boolean(c.grid);
    w.i32(c.grid_size);
    w.boolean(c.grid_checkerboard);
    w.boolean(c.hud);
    w.boolean(c.debug_hud);
    w.boolean(c.show_brush);
    w.boolean(c.zoom_enabled);
    w.i32(c.zoom_window_x);
    w.i32(c.zoom_window_y);
    w.i32(c.zoom_factor);
    w.i32(c.zoom_scope_x);
    w.i32(c.zoom_scope_y);
    w.i32(c.zoom_scope_size);
    w.opt_f32(c.has_heat_display_limit_min, c.heat_display_limit_min);
    w.opt_f32(c.has_heat_display_limit_max, c.heat_display_limit_max);
    w.i32(c.heat_display_auto_x);
    w.i32(c.heat_display_auto_y);
    w.i32(c.heat_display_auto_w);
    w.i32(c.heat_display_auto_h);
}

bool get_config(Reader &r, tpt_save_config &c) {
    c = tpt_save_config{};
    r.u32(c.xres);
    r.u32(c.yres);
    r.boolean(c.paused);
    r.boolean(c.aheat_enable);
    r.boolean(c.pretty_powder);
    r.variant(c.edge_mode, 3);     // EdgeMode (particle.rs:123-129)
    r.variant(c.gravity_mode, 4);  // GravityMode (:135-142)
    r.variant(c.air_mode, 5);      // AirMode (:149-157)
    r.f32(c.ambient_air_temp);
    r.f32(c.edge_pressure);
    r.u32(c.display_mode);
    r.u32(c.colour_mode);
    r.u32(c.render_mode);
    r.f32(c.fire_intensity);
    r.boolean(c.heat_enable);
    r.boolean(c.newton_grav);
    r.boolean(c.water_equal_test);
    r.f32(c.vorticity_coeff);
    r.u32(c.convection_mode);
    r.f32(c.edge_velocity_x);
    r.f32(c.edge_velocity_y);
    r.f32(c.custom_gravity_x);
    r.f32(c.custom_gravity_y);
    r.u32(c.temperature_scale);
    r.boolean(c.decorations);
    r.i32(c.mouse_x);
    r.i32(c.mouse_y);
    r.boolean(c.gravity_field_enabled);
    r.boolean(c.gravity_zones_enabled);
    r.boolean(c.grid);
    r.i32(c.grid_size);
    r.boolean(c.grid_checkerboard);
    r.boolean(c.hud);
    r.boolean(c.debug_hud);
    r.boolean(c.show_brush);
    r.boolean(c.zoom_enabled);
    r.i32(c.zoom_window_x);
    r.i32(c.zoom_window_y);
    r.i32(c.zoom_factor);
    r.i32(c.zoom_scope_x);
    r.i32(c.zoom_scope_y);
    r.i32(c.zoom_scope_size);
    r.opt_f32(c.has_heat_display_limit_min, c.heat_display_limit_min);
    r.opt_f32(c.has_heat_display_limit_max, c.heat_display_limit_max);
    r.i32(c.heat_display_auto_x);
    r.i32(c.heat_display_auto_y);
    r.i32(c.heat_display_auto_w);
    r.i32(c.heat_display_auto_h);
    return !r.err;
}

bool get_words(Reader &r, std::vector<uint32_t> &v) {
    uint64_t c;
    if (!r.count(c, 4)) return false;
    v.resize((size_t)c);
    for (auto &x : v) r.u32(x);
    return !r.err;
}

// One RigidBody2D (particle.rs:420-436; `materialised` is skipped) with its
// Vec<RigidPixel> (:392-403, nine 4-byte fields), validated and copied out.
bool skip_rigid(Reader &r) {
    uint32_t u;
    uint8_t b;
    float f;
    r.u32(u);      // id
    r.boolean(b);  // active
    for (int k = 0; k < 10; ++k) r.f32(f);  // cm_x .. inv_inertia
    uint64_t px;
    if (!r.count(px, 36)) return false;
    for (uint64_t k = 0; k < px * 9; ++k) r.u32(u);
    return !r.err;
}

// One Sign (crates/tpt-core/src/sign.rs:27-33): x, y, text (UTF-8), ju.
bool utf8_ok(const uint8_t *s, size_t n) {
    size_t i = 0;
    while (i < n) {
        const uint8_t c = s[i];
        size_t k;
        uint32_t cp;
        if (c < 0x80) {
            ++i;
            continue;
        } else if ((c & 0xE0) == 0xC0) {
            k = 1;
            cp = c & 0x1F;
        } else if ((c & 0xF0) == 0xE0) {
            k = 2;
            cp = c & 0x0F;
        } else if ((c & 0xF8) == 0xF0) {
            k = 3;
            cp = c & 0x07;
        } else {
            return false;
        }
        if (n - i <= k) return false;
        for (size_t j = 1; j <= k; ++j) {
            if ((s[i + j] & 0xC0) != 0x80) return false;
            cp = cp << 6 | (s[i + j] & 0x3F);
        }
        const uint32_t min[4] = {0, 0x80, 0x800, 0x10000};
        if (cp < min[k] || cp > 0x10FFFF || (cp >= 0xD800 && cp <= 0xDFFF)) return false;
        i += k + 1;
    }
    return true;
}

bool skip_sign(Reader &r) {
    int32_t v;
    r.i32(v);
    r.i32(v);
    uint64_t len;
    if (!r.count(len, 1)) return false;
    if (!utf8_ok(r.p + r.i, (size_t)len)) return r.fail("sign text is not UTF-8");
    r.i += (size_t)len;
    uint8_t ju;
    r.u8(ju);
    return !r.err;
}

// The encoded elements of a vector whose elements are walked by `skip`.
template <typename Skip>
bool get_raw_vec(Reader &r, std::vector<uint8_t> &raw, uint64_t &count, size_t min_elem, Skip skip) {
    if (!r.count(count, min_elem)) return false;
    const size_t start = r.i;
    for (uint64_t k = 0; k < count; ++k)
        if (!skip(r)) return false;
    raw.assign(r.p + start, r.p + r.i);
    return true;
}

// The zlib stream after an 8-byte magic, inflated to its end (a stream cut
// short is an error; bytes after its end are ignored, as flate2 does).
int inflate_after_magic(const void *bytes, size_t len, const char *magic, const char *what,
                        std::vector<uint8_t> &payload) {
    const uint8_t *b = (const uint8_t *)bytes;
    if (len <= 8) TPT_FAIL(TPT_ERR_INVALID_ARG, "%s is too short to contain a header", what);
    if (memcmp(b, magic, 8) != 0) TPT_FAIL(TPT_ERR_INVALID_ARG, "not a %s: bad magic header", what);
    z_stream zs{};
    if (inflateInit(&zs) != Z_OK) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "zlib inflateInit failed");
    zs.next_in = const_cast<Bytef *>(b + 8);
    zs.avail_in = (uInt)(len - 8 > 0xFFFFFFFFu ? 0xFFFFFFFFu : len - 8);
    int zr = Z_OK;
    std::vector<uint8_t> chunk(1 << 20);
    while (zr == Z_OK) {
        zs.next_out = chunk.data();
        zs.avail_out = (uInt)chunk.size();
        zr = inflate(&zs, Z_NO_FLUSH);
        if (zr != Z_OK && zr != Z_STREAM_END) break;
        payload.insert(payload.end(), chunk.data(), chunk.data() + (chunk.size() - zs.avail_out));
        if (zr == Z_OK && zs.avail_in == 0 && zs.avail_out != 0) {
            zr = Z_BUF_ERROR;  // input ended inside the stream
            break;
        }
    }
    inflateEnd(&zs);
    if (zr != Z_STREAM_END) TPT_FAIL(TPT_ERR_INVALID_ARG, "failed to decompress %s (zlib %d)", what, zr);
    return TPT_OK;
}

// magic + zlib(payload) at the default level into `out`.
int deflate_with_magic(const std::vector<uint8_t> &payload, const char *magic, std::vector<uint8_t> &out) {
    uLongf cap = compressBound((uLong)payload.size());
    out.resize(8 + (size_t)cap);
    memcpy(out.data(), magic, 8);
    if (compress2(out.data() + 8, &cap, payload.data(), (uLong)payload.size(), Z_DEFAULT_COMPRESSION) != Z_OK)
        TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "failed to compress save data");
    out.resize(8 + (size_t)cap);
    return TPT_OK;
}

int decode_payload(const uint8_t *p, size_t n, tpt_save &s) {
    Reader r{p, n};
    r.u32(s.version);  // the version probe (SaveDataVersion, lib.rs:124-128)
    if (r.err) TPT_FAIL(TPT_ERR_INVALID_ARG, "failed to deserialize save data: %s", r.err);
    if (s.version == 0 || s.version > TPT_SAVE_VERSION)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "unsupported save file version %u (this build supports 1..=%u)", s.version,
                 (unsigned)TPT_SAVE_VERSION);
    get_config(r, s.config);
    uint64_t np = 0;
    if (r.count(np, 64)) {
        s.particles.resize((size_t)np * 64);
        r.take(s.particles.data(), s.particles.size());
    }
    for (int g = 0; g < TPT_SAVE_GRIDS && !r.err; ++g) get_words(r, s.grid[g]);
    if (!r.err) get_raw_vec(r, s.rigid, s.n_rigid, 53, skip_rigid);
    // Version 1 (SaveDataV1, lib.rs:139-154) ends before the signs.
    if (!r.err && s.version >= 2) get_raw_vec(r, s.signs, s.n_signs, 17, skip_sign);
    if (r.err) TPT_FAIL(TPT_ERR_INVALID_ARG, "failed to deserialize save data: %s", r.err);
    if (s.config.xres == 0 || s.config.yres == 0 || s.config.xres > TPT_SAVE_MAX_CANVAS_DIM ||
        s.config.yres > TPT_SAVE_MAX_CANVAS_DIM)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "save file has an invalid canvas size %ux%u", s.config.xres, s.config.yres);
    return TPT_OK;
}

uint32_t align_dim(uint32_t v) {  // particle.rs:383-386: at least 64, a multiple of CELL = 4
    if (v < 64u) v = 64u;
    return (v + 3u) / 4u * 4u;
}

}  // namespace

extern "C" {

void tpt_save_config_default(tpt_save_config *c, uint32_t xres, uint32_t yres) {
    if (!c) return;
    *c = tpt_save_config{};
    c->xres = align_dim(xres);
    c->yres = align_dim(yres);
    c->ambient_air_temp = 295.15f;  // DEFAULT_TEMP_K
    c->render_mode = 0x1u | 0x2u | 0x4u | 0x40u;  // RENDER_BASC | FIRE | SPRK | EFFE
    c->fire_intensity = 1.0f;
    c->heat_enable = 1;
    c->vorticity_coeff = 0.1f;
    c->convection_mode = TPT_AIRC_BOUSSINESQ;
    c->custom_gravity_y = 1.0f;
    c->decorations = 1;
    c->mouse_x = -1;
    c->mouse_y = -1;
    c->grid_size = 1;
    c->hud = 1;
    c->show_brush = 1;
    c->zoom_factor = 8;
    c->zoom_scope_size = 32;
    c->has_heat_display_limit_min = 1;
    c->heat_display_limit_min = 0.0f;     // MIN_TEMP
    c->has_heat_display_limit_max = 1;
    c->heat_display_limit_max = 9999.0f;  // MAX_TEMP
    c->heat_display_auto_w = (int32_t)c->xres;
    c->heat_display_auto_h = (int32_t)c->yres;
}

int tpt_save_create(const tpt_save_config *config, tpt_save **out) {
    if (!config || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_create: NULL argument");
    *out = nullptr;
    if (config->xres == 0 || config->yres == 0 || config->xres > TPT_SAVE_MAX_CANVAS_DIM ||
        config->yres > TPT_SAVE_MAX_CANVAS_DIM)
        TPT_FAIL(TPT_ERR_INVALID_DIMS, "tpt_save_create: canvas %ux%u", config->xres, config->yres);
    tpt_save *s = new (std::nothrow) tpt_save();
    if (!s) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    s->config = *config;
    const size_t cells = (size_t)(config->xres / 4u) * (config->yres / 4u);
    for (auto &g : s->grid) g.assign(cells, 0u);
    *out = s;
    return TPT_OK;
}

int tpt_save_decode(const void *bytes, size_t len, tpt_save **out) {
    if (!out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_decode: out is NULL");
    *out = nullptr;
    if (!bytes && len) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_decode: bytes is NULL");
    std::vector<uint8_t> payload;
    int rc = inflate_after_magic(bytes, len, "TPTRS001", "Powder Toy (Rust) save file", payload);
    if (rc) return rc;
    tpt_save *s = new (std::nothrow) tpt_save();
    if (!s) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    rc = decode_payload(payload.data(), payload.size(), *s);
    if (rc) {
        delete s;
        return rc;
    }
    *out = s;
    return TPT_OK;
}

int tpt_save_encode(tpt_save *s, const void **bytes, size_t *len) {
    if (!s || !bytes || !len) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_encode: NULL argument");
    Writer w;
    w.u32(s->version);
    put_config(w, s->config);
    w.u64(s->particles.size() / 64);
    w.bytes(s->particles.data(), s->particles.size());
    for (const auto &g : s->grid) {
        w.u64(g.size());
        for (uint32_t x : g) w.u32(x);
    }
    w.u64(s->n_rigid);
    w.bytes(s->rigid.data(), s->rigid.size());
    w.u64(s->n_signs);
    w.bytes(s->signs.data(), s->signs.size());
    const int rc = deflate_with_magic(w.b, "TPTRS001", s->encoded);
    if (rc) return rc;
    *bytes = s->encoded.data();
    *len = s->encoded.size();
    return TPT_OK;
}

int tpt_save_destroy(tpt_save *s) {
    delete s;
    return TPT_OK;
}

int tpt_save_get_info(const tpt_save *s, tpt_save_info *out) {
    if (!s || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_get_info: NULL argument");
    *out = tpt_save_info{};
    out->version = s->version;
    out->xcells = s->config.xres / 4u;
    out->ycells = s->config.yres / 4u;
    out->n_particles = s->particles.size() / 64;
    out->n_rigid_bodies = s->n_rigid;
    out->n_signs = s->n_signs;
    for (int g = 0; g < TPT_SAVE_GRIDS; ++g) out->grid_len[g] = s->grid[g].size();
    return TPT_OK;
}

int tpt_save_get_config(const tpt_save *s, tpt_save_config *out) {
    if (!s || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_get_config: NULL argument");
    *out = s->config;
    return TPT_OK;
}

int tpt_save_set_config(tpt_save *s, const tpt_save_config *c) {
    if (!s || !c) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_set_config: NULL argument");
    if (c->edge_mode > 2u || c->gravity_mode > 3u || c->air_mode > 4u)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_save_set_config: enum value out of range");
    s->config = *c;
    return TPT_OK;
}

int tpt_save_set_version(tpt_save *s, uint32_t version) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_set_version: save is NULL");
    s->version = version;
    return TPT_OK;
}

int tpt_save_grid_read(const tpt_save *s, int grid, void *host, size_t bytes) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_grid_read: save is NULL");
    if (grid < 0 || grid >= TPT_SAVE_GRIDS) TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown save grid %d", grid);
    const auto &g = s->grid[grid];
    if (bytes != g.size() * 4) TPT_FAIL(TPT_ERR_INVALID_ARG, "grid %d holds %zu bytes, not %zu", grid, g.size() * 4, bytes);
    if (bytes && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_grid_read: host is NULL");
    if (bytes) memcpy(host, g.data(), bytes);
    return TPT_OK;
}

int tpt_save_grid_write(tpt_save *s, int grid, const void *host, size_t bytes) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_grid_write: save is NULL");
    if (grid < 0 || grid >= TPT_SAVE_GRIDS) TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown save grid %d", grid);
    if (bytes % 4) TPT_FAIL(TPT_ERR_INVALID_ARG, "grid bytes %zu is not a multiple of 4", bytes);
    if (bytes && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_grid_write: host is NULL");
    auto &g = s->grid[grid];
    g.resize(bytes / 4);
    if (bytes) memcpy(g.data(), host, bytes);
    return TPT_OK;
}

int tpt_save_grid_restore(const tpt_save *s, int grid, void *host, uint64_t cells) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_grid_restore: save is NULL");
    if (grid < 0 || grid >= TPT_SAVE_GRIDS) TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown save grid %d", grid);
    if (cells && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_grid_restore: host is NULL");
    const auto &g = s->grid[grid];
    if (g.size() == cells) memcpy(host, g.data(), (size_t)cells * 4);
    else memset(host, 0, (size_t)cells * 4);
    return TPT_OK;
}

int tpt_save_particles_read(const tpt_save *s, void *host, size_t bytes) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_particles_read: save is NULL");
    if (bytes != s->particles.size())
        TPT_FAIL(TPT_ERR_INVALID_ARG, "the particles are %zu bytes, not %zu", s->particles.size(), bytes);
    if (bytes && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_particles_read: host is NULL");
    if (bytes) memcpy(host, s->particles.data(), bytes);
    return TPT_OK;
}

int tpt_save_particles_write(tpt_save *s, const void *host, size_t bytes) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_particles_write: save is NULL");
    if (bytes % 64) TPT_FAIL(TPT_ERR_INVALID_ARG, "particle bytes %zu is not a multiple of 64", bytes);
    if (bytes && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_particles_write: host is NULL");
    s->particles.assign((const uint8_t *)host, (const uint8_t *)host + bytes);
    return TPT_OK;
}

int tpt_save_retain_air_pressure(tpt_save *s, int include) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_retain_air_pressure: save is NULL");
    if (!include)
        for (int g = TPT_SAVE_AIR_VX; g <= TPT_SAVE_AIR_HV; ++g) s->grid[g].clear();
    return TPT_OK;
}

int tpt_save_instance_desc(const tpt_save *s, tpt_instance_desc *out) {
    if (!s || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_save_instance_desc: NULL argument");
    tpt_save_config c;
    tpt_save_config_default(&c, s->config.xres, s->config.yres);
    *out = tpt_instance_desc{};
    tpt_air_params &a = out->air;
    a.xcells = c.xres / 4u;
    a.ycells = c.yres / 4u;
    a.air_mode = s->config.air_mode;          // copied from the save (lib.rs:266-276)
    a.aheat_enable = s->config.aheat_enable;
    a.gravity_mode = s->config.gravity_mode;
    a.ambient_air_temp = s->config.ambient_air_temp;
    a.edge_pressure = s->config.edge_pressure;
    a.convection_mode = c.convection_mode;     // SimulationConfig::new defaults
    a.edge_vx = c.edge_velocity_x;
    a.edge_vy = c.edge_velocity_y;
    a.vorticity_coeff = c.vorticity_coeff;
    a.custom_gx = c.custom_gravity_x;
    a.custom_gy = c.custom_gravity_y;
    out->newton_grav = c.newton_grav;
    return TPT_OK;
}

}  // extern "C"

// ============================================================ .tpt3 ====
// The 3-D sandbox's saves (crates/tpt-save/src/voxel3d.rs): "TPT3RS01" +
// zlib(bincode(Voxel3dSaveData)), version 4 only.

struct tpt_vox_save {
    uint32_t version = TPT_VOX_SAVE_VERSION;
    tpt_vox_save_config config{};
    std::vector<uint32_t> arr[TPT_VOX_SAVE_ARRAYS];  // voxels, ctype, tmp, tmp2, tmp3 (words), air (f32 bits)
    std::vector<uint8_t> bodies;                      // the encoded Voxel3dBodySave elements, kept as read
    uint64_t n_bodies = 0;
    std::vector<uint8_t> encoded;
};

namespace {

// Voxel3dConfig (crates/tpt-core/src/voxel3d/mod.rs:96-122); fixed-size
// arrays are their elements in order.
void put_vox_config(Writer &w, const tpt_vox_save_config &c) {
    w.u32(c.dim);
    w.boolean(c.paused);
    w.f32(c.ambient_temp_k);
    for (float g : c.gravity) w.f32(g);
    w.u32(c.edge_mode);
    w.boolean(c.air_enabled);
    w.u32(c.air_iterations);
    for (float d : c.sun_dir) w.f32(d);
    w.f32(c.exposure);
    w.f32(c.render_scale);
    w.u32(c.ao_rays);
    w.boolean(c.shadows);
}

bool get_vox_config(Reader &r, tpt_vox_save_config &c) {
    c = tpt_vox_save_config{};
    r.u32(c.dim);
    r.boolean(c.paused);
    r.f32(c.ambient_temp_k);
    for (float &g : c.gravity) r.f32(g);
    r.variant(c.edge_mode, 3);
    r.boolean(c.air_enabled);
    r.u32(c.air_iterations);
    for (float &d : c.sun_dir) r.f32(d);
    r.f32(c.exposure);
    r.f32(c.render_scale);
    r.u32(c.ao_rays);
    r.boolean(c.shadows);
    return !r.err;
}

// One Voxel3dBodySave (voxel3d.rs:42-57): 16 floats, ty, Vec<u32>.
bool skip_body(Reader &r) {
    uint32_t u;
    for (int k = 0; k < 17; ++k) r.u32(u);
    uint64_t n;
    if (!r.count(n, 4)) return false;
    for (uint64_t k = 0; k < n; ++k) r.u32(u);
    return !r.err;
}

// Voxel3dSaveData::validate (voxel3d.rs:155-214), the reference's messages.
int vox_validate(const tpt_vox_save &s) {
    if (s.version != TPT_VOX_SAVE_VERSION)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "unsupported voxel save version %u (this build supports %u)", s.version,
                 (unsigned)TPT_VOX_SAVE_VERSION);
    if (s.arr[TPT_VOX_SAVE_VOXELS].size() != (size_t)TPT_VOX_VOXELS)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "voxel save holds %zu voxels, expected %u", s.arr[TPT_VOX_SAVE_VOXELS].size(),
                 (unsigned)TPT_VOX_VOXELS);
    const char *names[] = {"ctype", "tmp", "tmp2", "tmp3"};
    for (int a = TPT_VOX_SAVE_CTYPE; a <= TPT_VOX_SAVE_TMP3; ++a) {
        const size_t n = s.arr[a].size();
        if (n != 0 && n != (size_t)TPT_VOX_VOXELS)
            TPT_FAIL(TPT_ERR_INVALID_ARG, "voxel save holds %zu %s words, expected 0 or %u", n, names[a - 1],
                     (unsigned)TPT_VOX_VOXELS);
    }
    if (s.arr[TPT_VOX_SAVE_AIR].size() % (size_t)TPT_VOX_CELLS)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "voxel save air grid has %zu cells, expected a multiple of %u",
                 s.arr[TPT_VOX_SAVE_AIR].size(), (unsigned)TPT_VOX_CELLS);
    if (s.n_bodies > (uint64_t)TPT_VOX_MAX_BODIES)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "voxel save holds %llu rigid bodies, at most %u are supported",
                 (unsigned long long)s.n_bodies, (unsigned)TPT_VOX_MAX_BODIES);
    Reader r{s.bodies.data(), s.bodies.size()};
    for (uint64_t b = 0; b < s.n_bodies; ++b) {
        uint32_t u;
        for (int k = 0; k < 17; ++k) r.u32(u);
        uint64_t n = 0;
        r.u64(n);
        if (n > (uint64_t)TPT_VOX_BODY_VOXELS)
            TPT_FAIL(TPT_ERR_INVALID_ARG, "rigid body %llu local grid holds %llu voxels, at most %u are supported",
                     (unsigned long long)b, (unsigned long long)n, (unsigned)TPT_VOX_BODY_VOXELS);
        r.i += (size_t)n * 4;
    }
    return TPT_OK;
}

}  // namespace

extern "C" {

void tpt_vox_save_config_default(tpt_vox_save_config *c) {
    if (!c) return;
    *c = tpt_vox_save_config{};
    c->dim = 256;  // VOXEL_DIM
    c->ambient_temp_k = 293.15f;
    c->gravity[1] = -9.81f;
    c->air_enabled = 1;
    c->air_iterations = 12;
    c->sun_dir[0] = 0.5f;
    c->sun_dir[1] = 0.70710677f;
    c->sun_dir[2] = 0.5f;
    c->exposure = 1.0f;
    c->render_scale = 1.0f;
    c->ao_rays = 2;
    c->shadows = 1;
}

int tpt_vox_save_create(const tpt_vox_save_config *config, tpt_vox_save **out) {
    if (!config || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_create: NULL argument");
    *out = nullptr;
    if (config->edge_mode > 2u) TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_vox_save_create: edge_mode out of range");
    tpt_vox_save *s = new (std::nothrow) tpt_vox_save();
    if (!s) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    s->config = *config;
    s->arr[TPT_VOX_SAVE_VOXELS].assign((size_t)TPT_VOX_VOXELS, 0u);
    *out = s;
    return TPT_OK;
}

int tpt_vox_save_decode(const void *bytes, size_t len, tpt_vox_save **out) {
    if (!out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_decode: out is NULL");
    *out = nullptr;
    if (!bytes && len) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_decode: bytes is NULL");
    std::vector<uint8_t> payload;
    int rc = inflate_after_magic(bytes, len, "TPT3RS01", "Powder Toy 3D voxel save", payload);
    if (rc) return rc;
    tpt_vox_save *s = new (std::nothrow) tpt_vox_save();
    if (!s) TPT_FAIL(TPT_ERR_OUT_OF_MEMORY, "host allocation failed");
    Reader r{payload.data(), payload.size()};
    r.u32(s->version);
    get_vox_config(r, s->config);
    for (auto &a : s->arr) get_words(r, a);
    if (!r.err) get_raw_vec(r, s->bodies, s->n_bodies, 76, skip_body);
    if (r.err) {
        delete s;
        TPT_FAIL(TPT_ERR_INVALID_ARG, "failed to deserialize voxel save data: %s", r.err);
    }
    rc = vox_validate(*s);
    if (rc) {
        delete s;
        return rc;
    }
    *out = s;
    return TPT_OK;
}

int tpt_vox_save_encode(tpt_vox_save *s, const void **bytes, size_t *len) {
    if (!s || !bytes || !len) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_encode: NULL argument");
    int rc = vox_validate(*s);
    if (rc) return rc;
    Writer w;
    w.u32(s->version);
    put_vox_config(w, s->config);
    for (const auto &a : s->arr) {
        w.u64(a.size());
        w.bytes(a.data(), a.size() * 4);  // little-endian words, the host's order
    }
    w.u64(s->n_bodies);
    w.bytes(s->bodies.data(), s->bodies.size());
    rc = deflate_with_magic(w.b, "TPT3RS01", s->encoded);
    if (rc) return rc;
    *bytes = s->encoded.data();
    *len = s->encoded.size();
    return TPT_OK;
}

int tpt_vox_save_destroy(tpt_vox_save *s) {
    delete s;
    return TPT_OK;
}

int tpt_vox_save_get_info(const tpt_vox_save *s, tpt_vox_save_info *out) {
    if (!s || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_get_info: NULL argument");
    *out = tpt_vox_save_info{};
    out->version = s->version;
    for (int a = 0; a < TPT_VOX_SAVE_ARRAYS; ++a) out->len[a] = s->arr[a].size();
    out->n_bodies = s->n_bodies;
    return TPT_OK;
}

int tpt_vox_save_get_config(const tpt_vox_save *s, tpt_vox_save_config *out) {
    if (!s || !out) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_get_config: NULL argument");
    *out = s->config;
    return TPT_OK;
}

int tpt_vox_save_set_config(tpt_vox_save *s, const tpt_vox_save_config *c) {
    if (!s || !c) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_set_config: NULL argument");
    if (c->edge_mode > 2u) TPT_FAIL(TPT_ERR_INVALID_ARG, "tpt_vox_save_set_config: edge_mode out of range");
    s->config = *c;
    return TPT_OK;
}

int tpt_vox_save_array_read(const tpt_vox_save *s, int array, void *host, size_t bytes) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_array_read: save is NULL");
    if (array < 0 || array >= TPT_VOX_SAVE_ARRAYS) TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown voxel save array %d", array);
    const auto &a = s->arr[array];
    if (bytes != a.size() * 4)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "array %d holds %zu bytes, not %zu", array, a.size() * 4, bytes);
    if (bytes && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_array_read: host is NULL");
    if (bytes) memcpy(host, a.data(), bytes);
    return TPT_OK;
}

int tpt_vox_save_array_write(tpt_vox_save *s, int array, const void *host, size_t bytes) {
    if (!s) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_array_write: save is NULL");
    if (array < 0 || array >= TPT_VOX_SAVE_ARRAYS) TPT_FAIL(TPT_ERR_INVALID_ARG, "unknown voxel save array %d", array);
    if (bytes % 4) TPT_FAIL(TPT_ERR_INVALID_ARG, "array bytes %zu is not a multiple of 4", bytes);
    if (bytes && !host) TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_array_write: host is NULL");
    auto &a = s->arr[array];
    a.resize(bytes / 4);
    if (bytes) memcpy(a.data(), host, bytes);
    return TPT_OK;
}

int tpt_vox_save_restore_air(const tpt_vox_save *s, float *vx, float *vy, float *vz, int32_t *pv, float *temp,
                             float *solid) {
    if (!s || !vx || !vy || !vz || !pv || !temp || !solid)
        TPT_FAIL(TPT_ERR_NULL_POINTER, "tpt_vox_save_restore_air: NULL argument");
    const size_t c = (size_t)TPT_VOX_CELLS;
    const auto &air = s->arr[TPT_VOX_SAVE_AIR];
    if (air.empty()) {  // AirState::new (air.rs:93-123)
        for (size_t i = 0; i < c; ++i) {
            vx[i] = vy[i] = vz[i] = solid[i] = 0.0f;
            pv[i] = 0;
            temp[i] = 293.15f;
        }
        return TPT_OK;
    }
    if (air.size() != 6 * c)
        TPT_FAIL(TPT_ERR_INVALID_ARG, "voxel3d: expected 0 or %zu air floats, got %zu", 6 * c, air.size());
    float *dst[6] = {vx, vy, vz, nullptr, temp, solid};
    for (int f = 0; f < 6; ++f) {
        const uint32_t *src = air.data() + (size_t)f * c;
        if (f != 3) {
            memcpy(dst[f], src, c * 4);
            continue;
        }
        for (size_t i = 0; i < c; ++i) {  // (value * PV_SCALE) as i32, saturating, NaN -> 0
            float v;
            memcpy(&v, &src[i], 4);
            const float q = v * 1024.0f;
            pv[i] = q != q ? 0 : q >= 2147483648.0f ? INT32_MAX : q < -2147483648.0f ? INT32_MIN : (int32_t)q;
        }
    }
    return TPT_OK;
}

}  // extern "C"
