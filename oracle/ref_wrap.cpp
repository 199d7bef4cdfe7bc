/*
 * ref_wrap.cpp -- C entry points around the reference's own, unmodified
 * Physics/morton.cpp and Physics/quadtree.cpp (compiled from the reference
 * checkout by oracle/Makefile into oracle/_ref/libgeref.so).
 *
 * TEST INFRASTRUCTURE ONLY: pins the oracle's restatement (ge_oracle.c)
 * against the reference code itself.  Each entry fills the reference's
 * particle vectors, calls the reference member function and copies the
 * result out.
 */
#include "Physics/morton.h"
#include "Physics/quadtree.h"

#include <cstring>

// Globals that the reference defines in globalLogic.cpp:20-23.
std::vector<Node> globalNodes;
std::vector<Node3D> globalNodes3D;
uint32_t globalId = 0;

static Morton g_morton;

extern "C" {

// Morton::computeMortonKeys (morton.cpp:27-38); bb = {x, y, size}
void ref_keys2d(int64_t n, const float *x, const float *y, const float *bb, uint64_t *keys) {
    std::vector<ParticlePhysics> p(n);
    for (int64_t i = 0; i < n; i++) p[i].pos = glm::vec2(x[i], y[i]);
    glm::vec3 b(bb[0], bb[1], bb[2]);
    g_morton.computeMortonKeys(p, b);
    for (int64_t i = 0; i < n; i++) keys[i] = p[i].mortonKey;
}

// Morton::computeMortonKeys3D (morton.cpp:92-112); bb = {x, y, z, size}
void ref_keys3d(int64_t n, const float *x, const float *y, const float *z, const float *bb,
                uint64_t *keys) {
    std::vector<ParticlePhysics3D> p(n);
    for (int64_t i = 0; i < n; i++) p[i].pos = glm::vec3(x[i], y[i], z[i]);
    glm::vec4 b(bb[0], bb[1], bb[2], bb[3]);
    g_morton.computeMortonKeys3D(p, b);
    for (int64_t i = 0; i < n; i++) keys[i] = p[i].mortonKey;
}

// Morton::sortParticlesByMortonKey (morton.cpp:40-63): returns, for each
// output slot, the input index that landed there (through the id field).
void ref_sort2d(int64_t n, const uint64_t *keys, uint32_t *order) {
    std::vector<ParticlePhysics> p(n);
    std::vector<ParticleRendering> r(n);
    for (int64_t i = 0; i < n; i++) { p[i].mortonKey = keys[i]; p[i].id = (uint32_t)i; }
    g_morton.sortParticlesByMortonKey(p, r);
    for (int64_t i = 0; i < n; i++) order[i] = p[i].id;
}

static void copy_nodes2d(int64_t cap, float *pos, float *size, float *com, float *mass,
                         uint32_t *start, uint32_t *end, uint32_t *next, uint32_t *child) {
    for (int64_t k = 0; k < (int64_t)globalNodes.size() && k < cap; k++) {
        const Node &nd = globalNodes[k];
        pos[2 * k] = nd.pos.x; pos[2 * k + 1] = nd.pos.y;
        com[2 * k] = nd.centerOfMass.x; com[2 * k + 1] = nd.centerOfMass.y;
        size[k] = nd.size; mass[k] = nd.gridMass;
        start[k] = nd.startIndex; end[k] = nd.endIndex; next[k] = nd.next;
        for (int q = 0; q < 4; q++) child[4 * k + q] = nd.subGrids[q & 1][(q >> 1) & 1];
    }
}

// globalNodes.clear(); Quadtree root(p, r, bb)  (globalLogic.cpp:1175-1177)
// over particles already in the order given.  Returns the node count.
int64_t ref_build_quadtree(int64_t n, const float *x, const float *y, const float *m,
                           const float *bb, int64_t cap, float *pos, float *size, float *com,
                           float *mass, uint32_t *start, uint32_t *end, uint32_t *next,
                           uint32_t *child) {
    std::vector<ParticlePhysics> p(n);
    std::vector<ParticleRendering> r(n);
    for (int64_t i = 0; i < n; i++) {
        p[i].pos = glm::vec2(x[i], y[i]);
        p[i].mass = m[i];
        p[i].temp = 0.0f;
    }
    glm::vec3 b(bb[0], bb[1], bb[2]);
    globalNodes.clear();
    { Quadtree root(p, r, b); }
    copy_nodes2d(cap, pos, size, com, mass, start, end, next, child);
    return (int64_t)globalNodes.size();
}

// globalNodes3D.clear(); Octree root3D(...)  (globalLogic.cpp:1600-1602)
int64_t ref_build_octree(int64_t n, const float *x, const float *y, const float *z,
                         const float *m, const float *bb, int64_t cap, float *pos, float *size,
                         float *com, float *mass, uint32_t *start, uint32_t *end,
                         uint32_t *next, uint32_t *child) {
    std::vector<ParticlePhysics3D> p(n);
    std::vector<ParticleRendering3D> r(n);
    for (int64_t i = 0; i < n; i++) {
        p[i].pos = glm::vec3(x[i], y[i], z[i]);
        p[i].mass = m[i];
        p[i].temp = 0.0f;
    }
    globalNodes3D.clear();
    { Octree root3D(p, r, glm::vec3(bb[0], bb[1], bb[2]), bb[3]); }
    for (int64_t k = 0; k < (int64_t)globalNodes3D.size() && k < cap; k++) {
        const Node3D &nd = globalNodes3D[k];
        pos[3 * k] = nd.pos.x; pos[3 * k + 1] = nd.pos.y; pos[3 * k + 2] = nd.pos.z;
        com[3 * k] = nd.centerOfMass.x; com[3 * k + 1] = nd.centerOfMass.y;
        com[3 * k + 2] = nd.centerOfMass.z;
        size[k] = nd.size; mass[k] = nd.gridMass;
        start[k] = nd.startIndex; end[k] = nd.endIndex; next[k] = nd.next;
        for (int q = 0; q < 8; q++) child[8 * k + q] = nd.subGrids[q & 1][(q >> 1) & 1][(q >> 2) & 1];
    }
    return (int64_t)globalNodes3D.size();
}

}  // extern "C"
