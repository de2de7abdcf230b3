// state_io.cpp - simulation snapshots: a JSON header followed by raw
// little-endian arrays (no counterpart in the reference, which keeps its
// state in GL textures only).
//
// Layout: one line of JSON (padded with spaces to a multiple of 64 bytes,
// ending in '\n'), then the sections it lists, each at its "offset" (bytes
// from the start of the file) with its "bytes" length:
//   vx, vy[, vz]   FP32 face velocities, shapes [nz][ny][nx+1] ...
//   density        FP32 [channels][nz][ny][nx]
//   temperature    FP32 [nz][ny][nx]
//   pressure       FP32 [nz][ny][nx] (the next solve's warm start)
//   emitters, obstacles, boxes   the ABI records (ss_emitter, ...) as stored
// A viewer reads the JSON and maps the FP32 sections directly.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ss_internal.h"

using namespace ss;

namespace {

struct Section {
    std::string name;
    std::string dtype;
    std::vector<long long> shape;
    long long count = 0;
    const void* host = nullptr;
    size_t bytes = 0;
    size_t offset = 0;
};

std::string json_shape(const std::vector<long long>& s) {
    std::string o = "[";
    for (size_t i = 0; i < s.size(); ++i) o += (i ? ", " : "") + std::to_string(s[i]);
    return o + "]";
}

// value of "key": <number> after position pos in the header (own writer's output)
bool find_number(const std::string& h, size_t pos, const char* key, long long* out) {
    const std::string k = std::string("\"") + key + "\":";
    const size_t p = h.find(k, pos);
    if (p == std::string::npos) return false;
    return sscanf(h.c_str() + p + k.size(), " %lld", out) == 1;
}

bool section_of(const std::string& h, const char* name, long long* offset, long long* bytes) {
    const std::string k = std::string("\"name\": \"") + name + "\"";
    const size_t p = h.find(k);
    if (p == std::string::npos) return false;
    return find_number(h, p, "offset", offset) && find_number(h, p, "bytes", bytes);
}

}  // namespace

extern "C" {

int ss_save_state(ss_sim* s, const char* path, void* stream) {
    if (!s || !path) return set_error(SS_E_INVALID, "NULL argument");
    std::vector<std::vector<float>> store;
    std::vector<Section> secs;
    const long long nx = s->nx, ny = s->ny, nz = s->nz;
    auto add_field = [&](const char* name, int field, std::vector<long long> shape) -> int {
        size_t n = 1;
        for (long long d : shape) n *= (size_t)d;
        store.emplace_back(n);
        const int rc = ss_get_field(s, field, store.back().data(), n, stream);
        if (rc) return rc;
        Section sec;
        sec.name = name; sec.dtype = "<f4"; sec.shape = shape; sec.count = (long long)n;
        sec.host = store.back().data(); sec.bytes = n * sizeof(float);
        secs.push_back(sec);
        return SS_OK;
    };
    int rc = add_field("vx", SS_FIELD_VX, {nz, ny, nx + 1});
    if (!rc) rc = add_field("vy", SS_FIELD_VY, {nz, ny + 1, nx});
    if (!rc && s->dim == 3) rc = add_field("vz", SS_FIELD_VZ, {nz + 1, ny, nx});
    if (!rc) rc = add_field("density", SS_FIELD_DENSITY, {(long long)s->nch, nz, ny, nx});
    if (!rc) rc = add_field("temperature", SS_FIELD_TEMPERATURE, {nz, ny, nx});
    if (!rc) rc = add_field("pressure", SS_FIELD_PRESSURE, {nz, ny, nx});
    if (rc) return rc;
    auto add_records = [&](const char* name, const void* p, size_t count, size_t size) {
        Section sec;
        sec.name = name; sec.dtype = "record"; sec.shape = {(long long)count}; sec.count = (long long)count;
        sec.host = p; sec.bytes = count * size;
        secs.push_back(sec);
    };
    add_records("emitters", s->em.data(), s->em.size(), sizeof(ss_emitter));
    add_records("obstacles", s->ob.data(), s->ob.size(), sizeof(ss_obstacle));
    add_records("boxes", s->bx.data(), s->bx.size(), sizeof(ss_box));

    // header length first (offsets depend on it): fixed-width offsets keep it stable
    auto header = [&](size_t data_start) {
        std::string h = "{\"format\": \"smokesim-state\", \"version\": 1, \"endian\": \"little\", \"dim\": " +
                        std::to_string(s->dim) + ", \"n\": [" + std::to_string(nx) + ", " + std::to_string(ny) + ", " +
                        std::to_string(nz) + "], \"cell_size\": " + std::to_string(s->h) +
                        ", \"density_channels\": " + std::to_string(s->nch) + ", \"enclosed\": " +
                        std::to_string(s->enclosed) + ", \"record_bytes\": {\"emitter\": " +
                        std::to_string(sizeof(ss_emitter)) + ", \"obstacle\": " + std::to_string(sizeof(ss_obstacle)) +
                        ", \"box\": " + std::to_string(sizeof(ss_box)) + "}, \"sections\": [";
        size_t off = data_start;
        for (size_t i = 0; i < secs.size(); ++i) {
            char num[64];
            snprintf(num, sizeof num, "%20zu", off);   // fixed width (JSON allows the spaces)
            h += (i ? ", " : "") + std::string("{\"name\": \"") + secs[i].name + "\", \"dtype\": \"" + secs[i].dtype +
                 "\", \"shape\": " + json_shape(secs[i].shape) + ", \"offset\": " + num +
                 ", \"bytes\": " + std::to_string(secs[i].bytes) + "}";
            secs[i].offset = off;
            off += (secs[i].bytes + 63) / 64 * 64;
        }
        h += "]}";
        return h;
    };
    std::string h = header(0);
    const size_t hlen = (h.size() + 1 + 63) / 64 * 64;
    h = header(hlen);
    h.append(hlen - 1 - h.size(), ' ');
    h += '\n';
    FILE* f = fopen(path, "wb");
    if (!f) return set_error(SS_E_INVALID, std::string("cannot open ") + path);
    bool ok = fwrite(h.data(), 1, h.size(), f) == h.size();
    const char pad[64] = {};
    for (const Section& sec : secs) {
        if (!ok) break;
        ok = fseek(f, (long)sec.offset, SEEK_SET) == 0 && (sec.bytes == 0 || fwrite(sec.host, 1, sec.bytes, f) == sec.bytes);
        const size_t tail = (sec.bytes + 63) / 64 * 64 - sec.bytes;
        if (ok && tail) ok = fwrite(pad, 1, tail, f) == tail;
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) return set_error(SS_E_INVALID, std::string("write failed: ") + path);
    return SS_OK;
}

int ss_load_state(ss_sim* s, const char* path, void* stream) {
    if (!s || !path) return set_error(SS_E_INVALID, "NULL argument");
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(SS_E_INVALID, std::string("cannot open ") + path);
    std::string h;
    for (int c; (c = fgetc(f)) != EOF && c != '\n' && h.size() < (1u << 20);) h.push_back((char)c);
    auto fail = [&](const std::string& why) {
        fclose(f);
        return set_error(SS_E_INVALID, "state file " + std::string(path) + ": " + why);
    };
    if (h.find("\"format\": \"smokesim-state\"") == std::string::npos) return fail("not a smokesim-state file");
    long long dim = 0, ch = 0, eb = 0, ob = 0, bb = 0;
    if (!find_number(h, 0, "dim", &dim) || !find_number(h, 0, "density_channels", &ch)) return fail("header");
    const size_t pn = h.find("\"n\": [");
    long long n[3] = {0, 0, 0};
    if (pn == std::string::npos || sscanf(h.c_str() + pn + 6, "%lld, %lld, %lld", &n[0], &n[1], &n[2]) != 3)
        return fail("header grid size");
    if (dim != s->dim || n[0] != s->nx || n[1] != s->ny || n[2] != s->nz || ch != s->nch)
        return fail("grid description differs from this simulation's");
    if (!find_number(h, 0, "emitter", &eb) || !find_number(h, 0, "obstacle", &ob) || !find_number(h, 0, "box", &bb) ||
        eb != (long long)sizeof(ss_emitter) || ob != (long long)sizeof(ss_obstacle) || bb != (long long)sizeof(ss_box))
        return fail("record layout differs from this library's");
    auto read = [&](const char* name, std::vector<unsigned char>& out) -> bool {
        long long off = 0, bytes = 0;
        if (!section_of(h, name, &off, &bytes) || off < 0 || bytes < 0) return false;
        out.resize((size_t)bytes);
        return fseek(f, (long)off, SEEK_SET) == 0 && (bytes == 0 || fread(out.data(), 1, (size_t)bytes, f) == (size_t)bytes);
    };
    std::vector<unsigned char> buf, emb, obb, bxb;
    if (!read("emitters", emb) || !read("obstacles", obb) || !read("boxes", bxb)) return fail("scene sections");
    struct F { const char* name; int field; };
    const F fields[] = {{"vx", SS_FIELD_VX}, {"vy", SS_FIELD_VY}, {"vz", SS_FIELD_VZ}, {"density", SS_FIELD_DENSITY},
                        {"temperature", SS_FIELD_TEMPERATURE}, {"pressure", SS_FIELD_PRESSURE}};
    std::vector<std::pair<int, std::vector<unsigned char>>> data;
    for (const F& fd : fields) {
        if (fd.field == SS_FIELD_VZ && s->dim != 3) continue;
        if (!read(fd.name, buf)) return fail(std::string("section ") + fd.name);
        data.emplace_back(fd.field, buf);
    }
    fclose(f);
    // the scene first (it rebuilds the solid map), then the fields
    int rc = ss_set_scene(s, (const ss_emitter*)emb.data(), (int)(emb.size() / sizeof(ss_emitter)),
                          (const ss_obstacle*)obb.data(), (int)(obb.size() / sizeof(ss_obstacle)),
                          (const ss_box*)bxb.data(), (int)(bxb.size() / sizeof(ss_box)), stream);
    if (rc) return rc;
    for (auto& d : data) {
        rc = ss_set_field(s, d.first, (const float*)d.second.data(), d.second.size() / sizeof(float), stream);
        if (rc) return rc;
    }
    return SS_OK;
}

}  // extern "C"
