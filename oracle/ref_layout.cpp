/*
 * ref_layout.cpp -- prints the byte layout of the reference's particle
 * records (include/Particles/particle.h) as the compiler lays it out, for the
 * test that pins ge_aos_layout_default to it.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/Makefile target `ref` writes its output
 * to _ref/particle_layout.txt).  One line per record type:
 *   <dims> stride pos vel acc prevVel mass id temp rendering_stride isPinned
 */
#include "Particles/particle.h"

#include <cstddef>
#include <cstdio>

uint32_t globalId = 0;

int main() {
    std::printf("2 %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(ParticlePhysics),
                offsetof(ParticlePhysics, pos), offsetof(ParticlePhysics, vel),
                offsetof(ParticlePhysics, acc), offsetof(ParticlePhysics, prevVel),
                offsetof(ParticlePhysics, mass), offsetof(ParticlePhysics, id),
                offsetof(ParticlePhysics, temp), sizeof(ParticleRendering),
                offsetof(ParticleRendering, isPinned));
    std::printf("3 %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(ParticlePhysics3D),
                offsetof(ParticlePhysics3D, pos), offsetof(ParticlePhysics3D, vel),
                offsetof(ParticlePhysics3D, acc), offsetof(ParticlePhysics3D, prevVel),
                offsetof(ParticlePhysics3D, mass), offsetof(ParticlePhysics3D, id),
                offsetof(ParticlePhysics3D, temp), sizeof(ParticleRendering3D),
                offsetof(ParticleRendering3D, isPinned));
    return 0;
}
