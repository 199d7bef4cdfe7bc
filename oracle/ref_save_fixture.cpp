/*
 * ref_save_fixture.cpp -- writes the save-file fixtures under tests/golden/
 * through the reference's own particle types.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/Makefile target `save-fixture`).  The
 * particles are the reference's ParticlePhysics / ParticleRendering (2D) and
 * ParticlePhysics3D / ParticleRendering3D (3D) structs from its checkout
 * (include/Particles/particle.h), made by their own parameterised
 * constructors, so every member's type and size in the file comes from the
 * reference's declarations (compiled against ref_shim/ge_ref_shim.h, the
 * glm / raylib stand-in).  The file layout is the format of
 * SaveSystem::saveSystem (src/UX/saveSystem.cpp:285-410): a YAML parameter
 * block, the separator, the version and three id counters, the particle
 * count, then per particle its members in that format's order, each written
 * with sizeof() of the reference's member.  After the particles the writer
 * puts the constraint count (0 here), where the reader of this library stops.
 *
 * Member values are exact in float (quarter multiples, small integers) and
 * follow from the particle index, so the test can restate them:
 *   pos    = ((i % 37) * 0.25 - 4, (i / 37) * 0.5 - 2 (, (i % 11) * 0.125 - 0.5))
 *   vel    = ((i % 5) * 0.125 - 0.25, (i % 7) * 0.0625 - 0.1875 (, (i % 3) * 0.25 - 0.25))
 *   acc    = (i % 3 - 1, i % 4 - 2 (, i % 5 - 2)) * 0.5
 *   mass   = 1 + (i % 9)           (the constructor's argument)
 *   temp   = 100 + i               (assigned after construction)
 *   id     = 1000 + i
 *   pinned = i % 13 == 0           (ParticleRendering::isPinned)
 * Usage: ref_save_fixture <out2d.bin> <out3d.bin> <count>
 */
#include "Particles/particle.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

uint32_t globalId = 0;

namespace {

// save format version 190 (include/UX/saveSystem.h:37-38)
constexpr uint32_t kVersion = 190;
const char *kSeparator = "\n---PARTICLE BINARY DATA---\n";

template <typename T>
void put(FILE *f, const T &v) {
    std::fwrite(&v, sizeof(v), 1, f);
}

template <typename P, typename R>
void put_record(FILE *f, const P &p, const R &r) {
    put(f, p.pos); put(f, p.predPos); put(f, p.vel); put(f, p.prevVel); put(f, p.predVel);
    put(f, p.acc); put(f, p.mass); put(f, p.press); put(f, p.pressTmp); put(f, p.pressF);
    put(f, p.dens); put(f, p.predDens); put(f, p.sphMass); put(f, p.restDens); put(f, p.stiff);
    put(f, p.visc); put(f, p.cohesion); put(f, p.temp); put(f, p.ke); put(f, p.prevKe);
    put(f, p.mortonKey); put(f, p.id); put(f, p.isHotPoint); put(f, p.hasSolidified);
    put(f, r.color); put(f, r.pColor); put(f, r.sColor); put(f, r.sphColor); put(f, r.size);
    put(f, r.uniqueColor); put(f, r.isSolid); put(f, r.canBeSubdivided); put(f, r.canBeResized);
    put(f, r.isDarkMatter); put(f, r.isSPH); put(f, r.isSelected); put(f, r.isGrabbed);
    put(f, r.previousSize); put(f, r.neighbors); put(f, r.totalRadius); put(f, r.lifeSpan);
    put(f, r.sphLabel); put(f, r.isPinned); put(f, r.isBeingDrawn); put(f, r.spawnCorrectIter);
    put(f, r.turbulence);
}

void header(FILE *f, bool d3, uint32_t count) {
    std::string yaml = std::string("G: 6.674e-11\nis3DMode: ") + (d3 ? "true" : "false") +
                       "\ntheta: 0.8\nsoftening: 1.5\n";
    std::fwrite(yaml.data(), 1, yaml.size(), f);
    std::fwrite(kSeparator, 1, std::strlen(kSeparator), f);
    const uint32_t gid = 1000 + count, shape = 0, wall = 0;
    put(f, kVersion); put(f, gid); put(f, shape); put(f, wall); put(f, count);
}

float pos_x(uint32_t i) { return (float)(i % 37) * 0.25f - 4.0f; }
float pos_y(uint32_t i) { return (float)(i / 37) * 0.5f - 2.0f; }
float pos_z(uint32_t i) { return (float)(i % 11) * 0.125f - 0.5f; }
float vel_x(uint32_t i) { return (float)(i % 5) * 0.125f - 0.25f; }
float vel_y(uint32_t i) { return (float)(i % 7) * 0.0625f - 0.1875f; }
float vel_z(uint32_t i) { return (float)(i % 3) * 0.25f - 0.25f; }

int write2d(const char *path, uint32_t n) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return 1;
    header(f, false, n);
    Color c{(unsigned char)10, (unsigned char)20, (unsigned char)30, (unsigned char)255};
    for (uint32_t i = 0; i < n; i++) {
        ParticlePhysics p(glm::vec2(pos_x(i), pos_y(i)), glm::vec2(vel_x(i), vel_y(i)),
                          1.0f + (float)(i % 9), 0.0f, 0.0f, 0.0f, 0.0f);
        p.acc = glm::vec2(((float)(i % 3) - 1.0f) * 0.5f, ((float)(i % 4) - 2.0f) * 0.5f);
        p.temp = 100.0f + (float)i;
        p.id = 1000 + i;
        ParticleRendering r(c, 1.0f, false, false, false, true, true, false, true, -1.0f, 0);
        r.isPinned = (i % 13) == 0;
        put_record(f, p, r);
    }
    put(f, (uint32_t)0);   // constraints
    std::fclose(f);
    return 0;
}

int write3d(const char *path, uint32_t n) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return 1;
    header(f, true, n);
    Color c{(unsigned char)40, (unsigned char)50, (unsigned char)60, (unsigned char)255};
    for (uint32_t i = 0; i < n; i++) {
        ParticlePhysics3D p(glm::vec3(pos_x(i), pos_y(i), pos_z(i)),
                            glm::vec3(vel_x(i), vel_y(i), vel_z(i)), 1.0f + (float)(i % 9),
                            0.0f, 0.0f, 0.0f, 0.0f);
        p.acc = glm::vec3(((float)(i % 3) - 1.0f) * 0.5f, ((float)(i % 4) - 2.0f) * 0.5f,
                          ((float)(i % 5) - 2.0f) * 0.5f);
        p.temp = 100.0f + (float)i;
        p.id = 1000 + i;
        ParticleRendering3D r(c, 1.0f, false, false, false, true, true, false, true, -1.0f, 0);
        r.isPinned = (i % 13) == 0;
        put_record(f, p, r);
    }
    put(f, (uint32_t)0);   // constraints
    std::fclose(f);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <out2d.bin> <out3d.bin> <count>\n", argv[0]);
        return 2;
    }
    const uint32_t n = (uint32_t)std::strtoul(argv[3], nullptr, 10);
    std::printf("sizeof ParticlePhysics %zu, ParticleRendering %zu, ParticlePhysics3D %zu, "
                "ParticleRendering3D %zu\n", sizeof(ParticlePhysics), sizeof(ParticleRendering),
                sizeof(ParticlePhysics3D), sizeof(ParticleRendering3D));
    if (write2d(argv[1], n) || write3d(argv[2], n)) {
        std::fprintf(stderr, "cannot write the fixtures\n");
        return 1;
    }
    return 0;
}
