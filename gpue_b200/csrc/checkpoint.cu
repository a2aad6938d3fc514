// checkpoint.cu -- binary snapshots of a context for checkpoint and resume.
//
// GPUE itself only writes text dumps (FileIO::writeOut, src/fileIO.cu:13-72)
// and restarts from them with -r; those lose the imaginary-time
// renormalisation still pending on the device and the energy the next
// early-stop check compares with.  A snapshot keeps the state exactly as the
// context holds it, so a resumed run continues bit for bit:
//
//   offset 0   SnapshotHeader (fixed size, little endian, version 1)
//   then       the state, npoints complex values of `dtype`, x fastest,
//              without the pending factor applied
//
// The header carries the grid and physics parameters (gpue_params) the state
// belongs to; a load into a context whose parameters differ (apart from
// precision and device) is refused, as is a payload whose checksum (64-bit
// FNV-1a over 8-byte words) does not match.  Saves go to "<path>.tmp" and are
// renamed over <path>, so an interrupted save leaves the previous snapshot.

#include <cstdint>
#include <cstdio>
#include <vector>

#include "engine_internal.h"

using namespace gpue_eng;

namespace {

constexpr char kMagic[8] = {'G', 'P', 'U', 'E', 'S', 'N', 'A', 'P'};
constexpr uint32_t kVersion = 1;

struct SnapshotHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    int32_t dtype;          // GPUE_C128 / GPUE_C64
    int32_t gstate;         // caller's phase
    int64_t step;           // caller's step index
    int64_t npoints;
    double last_energy;     // energy of the latest check (the early-stop reference)
    int32_t pending_scale;  // 1: `scale` still multiplies the state
    int32_t pad;
    double scale;
    gpue_params params;
    uint64_t checksum;
};

uint64_t fnv1a_words(const void* p, size_t bytes) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 1469598103934665603ull;
    size_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 1099511628211ull;
    }
    for (; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

// The parameters a state depends on: every field but precision, device and
// the reserved words (compared field by field: the struct has tail padding).
bool same_physics(const gpue_params& a, const gpue_params& b, std::string& what) {
    if (a.dimnum != b.dimnum || a.xDim != b.xDim || a.yDim != b.yDim || a.zDim != b.zDim) {
        what = "grid";
        return false;
    }
    if (a.xMax != b.xMax || a.yMax != b.yMax || a.zMax != b.zMax) {
        what = "box";
        return false;
    }
    const double da[] = {a.hbar, a.mass, a.omegaX, a.omegaY, a.omegaZ, a.gammaY, a.x0_shift,
                         a.y0_shift, a.z0_shift, a.omega, a.interaction, a.gDenConst, a.gdt,
                         a.dt};
    const double db[] = {b.hbar, b.mass, b.omegaX, b.omegaY, b.omegaZ, b.gammaY, b.x0_shift,
                         b.y0_shift, b.z0_shift, b.omega, b.interaction, b.gDenConst, b.gdt,
                         b.dt};
    const int ia[] = {a.gpe, a.corotating, a.gauge, a.ramp, a.ramp_type};
    const int ib[] = {b.gpe, b.corotating, b.gauge, b.ramp, b.ramp_type};
    for (size_t k = 0; k < sizeof da / sizeof da[0]; ++k)
        if (da[k] != db[k]) {
            what = "parameters";
            return false;
        }
    for (size_t k = 0; k < sizeof ia / sizeof ia[0]; ++k)
        if (ia[k] != ib[k]) {
            what = "parameters";
            return false;
        }
    return true;
}

}  // namespace

gpue_status gpue_snapshot_save(gpue_ctx* c, const char* path, int32_t gstate, int64_t step) {
    if (!c || !path) return GPUE_ERR_INVALID_ARG;
    if (!c->have_wfc) return fail(c, GPUE_ERR_STATE, "no wavefunction set");
    CK(cudaSetDevice(c->device));
    const int sp = c->polished ? GPUE_PREC_FP64 : c->prec;
    const size_t es = sp == GPUE_PREC_FP32 ? 8 : 16;
    SnapshotHeader h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.header_bytes = sizeof h;
    h.dtype = sp == GPUE_PREC_FP32 ? GPUE_C64 : GPUE_C128;
    h.gstate = gstate;
    h.step = step;
    h.npoints = c->N;
    h.last_energy = c->last_energy;
    h.pending_scale = c->pending_scale ? 1 : 0;
    std::memcpy(&h.params, &c->p, sizeof h.params);
    std::vector<unsigned char> payload(es * (size_t)c->N);
    CK(cudaMemcpyAsync(payload.data(), state_of(c, sp), payload.size(), cudaMemcpyDeviceToHost,
                       c->stream));
    if (c->pending_scale)
        CK(cudaMemcpyAsync(&h.scale, c->scal + kScale, sizeof h.scale, cudaMemcpyDeviceToHost,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    h.checksum = fnv1a_words(payload.data(), payload.size());
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return fail(c, GPUE_ERR_INVALID_ARG, "cannot write %s", tmp.c_str());
    const bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
                    std::fwrite(payload.data(), 1, payload.size(), f) == payload.size();
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) {
        std::remove(tmp.c_str());
        return fail(c, GPUE_ERR_INVALID_ARG, "short write to %s", tmp.c_str());
    }
    if (std::rename(tmp.c_str(), path) != 0)
        return fail(c, GPUE_ERR_INVALID_ARG, "cannot rename %s to %s", tmp.c_str(), path);
    return GPUE_OK;
}

gpue_status gpue_snapshot_load(gpue_ctx* c, const char* path, int32_t* gstate, int64_t* step) {
    if (!c || !path) return GPUE_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(c, GPUE_ERR_INVALID_ARG, "cannot open %s", path);
    SnapshotHeader h;
    if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 ||
        h.version != kVersion || h.header_bytes != sizeof h) {
        std::fclose(f);
        return fail(c, GPUE_ERR_INVALID_ARG, "%s is not a version-%u snapshot", path, kVersion);
    }
    std::string what;
    if (h.npoints != c->N || !same_physics(h.params, c->p, what)) {
        std::fclose(f);
        return fail(c, GPUE_ERR_INVALID_ARG, "%s was saved with a different %s", path,
                    what.empty() ? "grid" : what.c_str());
    }
    if (h.dtype != GPUE_C128 && h.dtype != GPUE_C64) {
        std::fclose(f);
        return fail(c, GPUE_ERR_INVALID_ARG, "%s: unknown dtype %d", path, h.dtype);
    }
    std::vector<unsigned char> payload((h.dtype == GPUE_C64 ? 8 : 16) * (size_t)h.npoints);
    const bool got = std::fread(payload.data(), 1, payload.size(), f) == payload.size();
    std::fclose(f);
    if (!got) return fail(c, GPUE_ERR_INVALID_ARG, "%s is truncated", path);
    if (fnv1a_words(payload.data(), payload.size()) != h.checksum)
        return fail(c, GPUE_ERR_INVALID_ARG, "%s: checksum mismatch", path);
    gpue_status st = gpue_set_wfc(c, payload.data(), GPUE_MEM_HOST, h.dtype);
    if (st) return st;
    // the deferred renormalisation is a factor, whatever the element type
    if (h.pending_scale) {
        CK(cudaMemcpyAsync(c->scal + kScale, &h.scale, sizeof h.scale, cudaMemcpyHostToDevice,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->pending_scale = true;
    }
    c->last_energy = h.last_energy;
    if (gstate) *gstate = h.gstate;
    if (step) *step = h.step;
    return GPUE_OK;
}
