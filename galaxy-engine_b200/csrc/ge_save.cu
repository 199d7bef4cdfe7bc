// ge_save.cu -- reader of Galaxy Engine scene files (host code only).
//
// SaveSystem::saveSystem / deserializeParticleSystem (src/UX/saveSystem.cpp:
// 285-362, include/UX/saveSystem.h:120-290) write a YAML parameter block,
// the line "---PARTICLE BINARY DATA---", then little-endian binary data:
//   uint32 version (190; 180 files are read by the same code), uint32
//   globalId, globalShapeId, globalWallId, uint32 particle count, then per
//   particle the ParticlePhysics(3D) and ParticleRendering(3D) members
//   (include/Particles/particle.h), each written with its own sizeof, in the
//   order of saveSystem.cpp:314-360 (2D) / :371-410 (3D).
// The dimension is the YAML's is3DMode (saveSystem.cpp:75).  A 2D record is
// 180 bytes, a 3D record 208.  This reader returns the members the gravity
// step uses (position, velocity, acceleration, mass, temperature, id, pin
// flag) as structure-of-arrays for ge_upload / ge_upload_temp /
// ge_upload_pinned; the particles come in the file's order.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "ge_bh.h"

namespace {

const char *kSep = "---PARTICLE BINARY DATA---";

struct Layout {
    int dims;
    size_t record;   // bytes per particle
    size_t pos, vel, acc, mass, temp, id, pinned;
};

// byte offsets of the members the reader uses; the record is the members'
// sizes summed in the file's order (vecD = D floats, Color = 4 bytes,
// bool = 1, uint64 mortonKey = 8)
Layout layout(int D) {
    Layout L{};
    L.dims = D;
    const size_t v = 4 * (size_t)D;
    size_t o = 0;
    L.pos = o; o += v;           // pos
    o += v;                      // predPos
    L.vel = o; o += v;           // vel
    o += v;                      // prevVel
    o += v;                      // predVel
    L.acc = o; o += v;           // acc
    L.mass = o; o += 4;          // mass
    o += 4 + 4;                  // press, pressTmp
    o += v;                      // pressF
    o += 4 * 7;                  // dens, predDens, sphMass, restDens, stiff, visc, cohesion
    L.temp = o; o += 4;          // temp
    o += 4 + 4;                  // ke, prevKe
    o += 8;                      // mortonKey
    L.id = o; o += 4;            // id
    o += 1 + 1;                  // isHotPoint, hasSolidified
    o += 4 * 4;                  // color, pColor, sColor, sphColor
    o += 4;                      // size
    o += 8;                      // uniqueColor .. isGrabbed (8 bools)
    o += 4 + 4 + 4 + 4 + 4;      // previousSize, neighbors, totalRadius, lifeSpan, sphLabel
    L.pinned = o; o += 1;        // isPinned
    o += 1;                      // isBeingDrawn
    o += 4 + 4;                  // spawnCorrectIter, turbulence
    L.record = o;
    return L;
}

struct Header {
    uint32_t version = 0, gid = 0, gshape = 0, gwall = 0, count = 0;
    int dims = 2;
    std::streampos data;   // first particle record
};

int read_header(std::ifstream &f, Header &h) {
    std::string line;
    bool found = false, is3d = false;
    while (std::getline(f, line)) {
        if (line.find(kSep) != std::string::npos) {
            found = true;
            break;
        }
        const size_t k = line.find("is3DMode:");
        if (k != std::string::npos) {
            const std::string val = line.substr(k + 9);
            is3d = val.find("true") != std::string::npos;
        }
    }
    if (!found) return GE_ERR_ARG;
    uint32_t w[5];
    f.read(reinterpret_cast<char *>(w), sizeof(w));
    if (!f) return GE_ERR_ARG;
    h.version = w[0];
    h.gid = w[1];
    h.gshape = w[2];
    h.gwall = w[3];
    h.count = w[4];
    h.dims = is3d ? 3 : 2;
    h.data = f.tellg();
    if (h.version != 190 && h.version != 180) return GE_ERR_UNSUPPORTED;
    return GE_OK;
}

}  // namespace

extern "C" {

int ge_save_read_info(const char *path, ge_save_info *info) {
    if (!path || !info) return GE_ERR_ARG;
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f.is_open()) return GE_ERR_ARG;
    Header h;
    const int rc = read_header(f, h);
    std::memset(info, 0, sizeof(*info));
    info->version = h.version;
    if (rc) return rc;
    info->dims = h.dims;
    info->n = h.count;
    info->global_id = h.gid;
    info->global_shape_id = h.gshape;
    info->global_wall_id = h.gwall;
    info->record_bytes = (int32_t)layout(h.dims).record;
    return GE_OK;
}

int ge_save_read(const char *path, int64_t cap, float *x, float *y, float *z, float *vx,
                 float *vy, float *vz, float *ax, float *ay, float *az, float *m, float *temp,
                 uint32_t *id, uint8_t *pinned) {
    if (!path) return GE_ERR_ARG;
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f.is_open()) return GE_ERR_ARG;
    Header h;
    int rc = read_header(f, h);
    if (rc) return rc;
    if ((int64_t)h.count > cap) return GE_ERR_CAPACITY;
    const Layout L = layout(h.dims);
    const int D = h.dims;
    float *pos[3] = {x, y, D == 3 ? z : nullptr};
    float *vel[3] = {vx, vy, D == 3 ? vz : nullptr};
    float *acc[3] = {ax, ay, D == 3 ? az : nullptr};
    std::vector<unsigned char> buf;
    const size_t chunk = 65536;
    for (uint32_t base = 0; base < h.count; base += (uint32_t)chunk) {
        const size_t cnt = std::min<size_t>(chunk, h.count - base);
        buf.resize(cnt * L.record);
        f.read(reinterpret_cast<char *>(buf.data()), (std::streamsize)buf.size());
        if ((size_t)f.gcount() != buf.size()) return GE_ERR_ARG;   // truncated file
        for (size_t k = 0; k < cnt; k++) {
            const unsigned char *r = buf.data() + k * L.record;
            const size_t i = base + k;
            for (int a = 0; a < D; a++) {
                if (pos[a]) std::memcpy(&pos[a][i], r + L.pos + 4 * a, 4);
                if (vel[a]) std::memcpy(&vel[a][i], r + L.vel + 4 * a, 4);
                if (acc[a]) std::memcpy(&acc[a][i], r + L.acc + 4 * a, 4);
            }
            if (m) std::memcpy(&m[i], r + L.mass, 4);
            if (temp) std::memcpy(&temp[i], r + L.temp, 4);
            if (id) std::memcpy(&id[i], r + L.id, 4);
            if (pinned) pinned[i] = r[L.pinned] ? 1u : 0u;
        }
    }
    return GE_OK;
}

}  // extern "C"
