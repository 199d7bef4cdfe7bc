/*
 * ge_oracle.h -- CPU restatement of Galaxy Engine's per-frame gravity path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle: the tests, the smoke
 * check and the CPU-baseline leg of bench.py call it as the checker.  The
 * product library (galaxy-engine_b200/libgebh.so) never links or calls it.
 *
 * Every function restates the reference algorithm from the cited lines of
 * NarcisCalin/Galaxy-Engine (paths relative to the reference checkout):
 *
 *   bounding box      GalaxyEngine/src/globalLogic.cpp:1083-1099 (2D), :1460-1477 (3D)
 *   Morton keys       GalaxyEngine/src/Physics/morton.cpp:3-38 (2D), :67-112 (3D)
 *   key sort          GalaxyEngine/src/Physics/morton.cpp:40-63, :114-138
 *   quadtree build    GalaxyEngine/src/Physics/quadtree.cpp:5-107, include/Physics/quadtree.h:31-129
 *   octree build      GalaxyEngine/src/Physics/quadtree.cpp:109-292, include/Physics/quadtree.h:134-197
 *   2D tree walk      GalaxyEngine/src/Physics/physics.cpp:91-205 (scalar), :207-352 (AVX2)
 *   3D tree walk      GalaxyEngine/src/Physics/physics3D.cpp:131-253 (scalar), :255-414 (AVX2)
 *   direct sum        GalaxyEngine/src/Physics/physics.cpp:392-540, physics3D.cpp:416-623
 *   leapfrog halves   GalaxyEngine/src/Physics/physics.cpp:1069-1125, physics3D.cpp:740-804, :1158-1168
 *   frame order       GalaxyEngine/src/globalLogic.cpp:1155-1370 (2D), :1584-1719 (3D)
 *
 * Conventions that differ from the reference, on purpose:
 *   - the key sort is STABLE by (key, current index).  The reference uses
 *     std::sort, whose order among equal keys is unspecified; a stable order
 *     is the canonical permutation the GPU build reproduces bit-exactly.
 *   - the softening term added to r^2 is passed explicitly as eps2.  The 2D
 *     reference walk adds softening^2 (physics.cpp:100,123); the 3D walk adds
 *     softening un-squared (physics3D.cpp:166,221).
 *   - the gridTemp / particle temperature terms are carried only when
 *     temperature is enabled (reference default: off, parameters.h:147).
 *
 * Node arrays are the reference's `globalNodes` content in DFS pre-order,
 * stored structure-of-arrays: child[q] with q = xbit | ybit<<1 (| zbit<<2),
 * the reference's subGrids[xbit][ybit]([zbit]); UINT32_MAX marks an empty slot.
 */
#ifndef GE_ORACLE_H
#define GE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int   dims;            /* 2 or 3 */
    float G;
    float theta;
    float eps2;            /* value added to r^2 in the tree walk */
    float dt;              /* myVar.timeFactor */
    uint32_t leaf_cap;     /* reference: 4  (quadtree.cpp:16) */
    float size_gate;       /* reference: 2.0f */
    float min_size;        /* reference: 1e-6f */
    int   periodic;        /* isPeriodicBoundaryEnabled && !infiniteDomain */
    float domain[3];       /* domainSize / domainSize3D */
    int   temp_enabled;    /* isTempEnabled */
    float heat_cond;       /* globalHeatConductivity */
    float naive_soft;      /* softening added un-squared by the direct-sum path */
    int   direct_below;    /* scalar frame (walk 0): direct sum below this many particles */
} or_params;

typedef struct {
    int64_t  cap;          /* node capacity of every array below */
    int64_t  count;        /* nodes written */
    int      dims;
    int      overflow;     /* set when cap was too small */
    int      max_depth;
    float   *pos;          /* [cap*dims] cell corner */
    float   *size;         /* [cap] */
    float   *com;          /* [cap*dims] */
    float   *mass;         /* [cap] */
    float   *temp;         /* [cap] gridTemp (0 unless temp given) */
    uint32_t *start, *end, *next;
    uint32_t *child;       /* [cap*(1<<dims)] */
} or_tree;

/* --- bounding box ---------------------------------------------------- */
void or_bbox2d(int64_t n, const float *x, const float *y, float out[3]);
void or_bbox3d(int64_t n, const float *x, const float *y, const float *z, float out[4]);

/* --- Morton keys ----------------------------------------------------- */
uint64_t or_scale_to_grid2d(float p, float lo, float hi);
uint64_t or_scale_to_grid3d(float p, float lo, float hi);
void or_keys2d(int64_t n, const float *x, const float *y, const float bb[3], uint64_t *keys);
void or_keys3d(int64_t n, const float *x, const float *y, const float *z, const float bb[4], uint64_t *keys);

/* stable (key, index) order: perm[k] = index of the k-th smallest */
void or_sort_perm(int64_t n, const uint64_t *keys, uint32_t *perm);

/* --- tree build over already-sorted particles ------------------------ */
int  or_tree_alloc(or_tree *t, int dims, int64_t cap);
void or_tree_free(or_tree *t);
/* bb = {x, y, size} (2D) or {x, y, z, size} (3D); temp may be NULL */
int or_build_quadtree(or_tree *t, int64_t n, const float *x, const float *y,
                      const float *m, const float *temp, const float bb[3],
                      uint32_t leaf_cap, float size_gate, float min_size);
int or_build_octree(or_tree *t, int64_t n, const float *x, const float *y, const float *z,
                    const float *m, const float *temp, const float bb[4],
                    uint32_t leaf_cap, float size_gate, float min_size);

/* --- force ------------------------------------------------------------ */
/* Temperature (temp_enabled): the reference updates temp[i] in place inside
 * an OpenMP-parallel loop while other threads read it as their temp[j]
 * (physics.cpp:145-158, 183-191), so its result depends on thread timing.
 * The oracle fixes one order: every particle reads the other particles'
 * temperatures, and the nodes' sums, as they were before the walk, and
 * accumulates its own in its walk order; the device walk does the same. */
/* scalar walk (parity oracle).  temp may be NULL when temp_enabled == 0.
 * inter (optional, [n]) receives the per-particle interaction count:
 * accepted monopoles + leaf pairs j != i.  cond (optional, [n]) receives
 * sum|F_k| / |sum F_k|, the cancellation factor of that particle's sum. */
void or_walk2d(int64_t n, const float *x, const float *y, const float *m, float *temp,
               const or_tree *t, const or_params *p, float *ax, float *ay,
               uint32_t *inter, float *cond, int nthreads);
void or_walk3d(int64_t n, const float *x, const float *y, const float *z, const float *m,
               float *temp, const or_tree *t, const or_params *p,
               float *ax, float *ay, float *az, uint32_t *inter, float *cond, int nthreads);
/* AVX2 walk: the path the application runs on AVX2 hosts (timed baseline) */
void or_walk2d_avx2(int64_t n, const float *x, const float *y, const float *m,
                    const or_tree *t, const or_params *p, float *ax, float *ay, int nthreads);
void or_walk3d_avx2(int64_t n, const float *x, const float *y, const float *z, const float *m,
                    const or_tree *t, const or_params *p, float *ax, float *ay, float *az,
                    int nthreads);
/* O(N^2) direct sum, used by the application for N < 5000 */
void or_naive2d(int64_t n, const float *x, const float *y, const float *m,
                const or_params *p, float *ax, float *ay, int nthreads);
void or_naive3d(int64_t n, const float *x, const float *y, const float *z, const float *m,
                const or_params *p, float *ax, float *ay, float *az, int nthreads);
/* FP64 direct sum for the targets listed in idx (eps2 added to r^2, j != i) */
void or_direct_f64(int dims, int64_t n, const float *x, const float *y, const float *z,
                   const float *m, double G, double eps2, int64_t nt, const int64_t *idx,
                   double *ax, double *ay, double *az, int nthreads);

/* --- mixed-precision walk (checker of GE_PREC_MIXED; ge_oracle_mixed.c) --
 * FP64 node moments (mom: [count * (6 | 10)] = mass, com, second moments
 * about the com: 2D xx xy yy, 3D xx yy zz xy xz yz), then the walk with the
 * offset-corrected opening test and the softened quadrupole, accelerations
 * in FP64.  inter (optional, [n]) receives the interaction counts. */
int or_moments_mixed(const or_tree *t, const float *x, const float *y, const float *z,
                     const float *m, double *mom);
void or_walk_mixed(int64_t n, const float *x, const float *y, const float *z, const float *m,
                   const or_tree *t, const or_params *p, double *ax, double *ay, double *az,
                   uint32_t *inter, int nthreads);
/* the same with the group walk: groups of group_size consecutive particles
 * share one opening test against their bounding box (ge_oracle_mixed.c) */
void or_walk_group(int64_t n, const float *x, const float *y, const float *z, const float *m,
                   const or_tree *t, const or_params *p, int group_size, double *ax, double *ay,
                   double *az, uint32_t *inter, int nthreads);

/* --- trajectory preview (particlesSpawning.cpp:443-500, :1000-1060) ----
 * nprobes probe particles (pos/vel [nprobes*dims], mass [nprobes]) stepped
 * `steps` times against the fixed tree t built over particles x, y, z, with
 * the older walk (physics.cpp:4-90, physics3D.cpp:49-120); eps2 is the
 * softening added to r^2 (squared in both 2D and 3D in that walk).
 * path [nprobes*steps*dims] receives each step's position. */
void or_predict_trajectory(const or_tree *t, const float *x, const float *y, const float *z,
                           const or_params *p, float eps2, int64_t nprobes, const float *pos,
                           const float *vel, const float *mass, int32_t steps, float *path,
                           int nthreads);

/* --- gravity field display (include/Physics/field.h:59-80, 106-222) -----
 * strength [amount_x * amount_y] (index j + i * amount_y) and rgba (RGBA8,
 * one pixel per cell) of the field view over the 2D domain. */
int or_gravity_field(int64_t n, const float *x, const float *y, const float *m, float G,
                     float dom_x, float dom_y, int periodic, int res, float softness,
                     float threshold, float stretch, float exposure, int two_color,
                     const float low[3], const float high[3], float *strength, uint32_t *rgba,
                     int *amount_x, int *amount_y, int nthreads);

/* FP64 potential energy by direct summation (energy pass reference) */
double or_potential_f64(int dims, int64_t n, const float *x, const float *y, const float *z,
                        const float *m, double G, double eps2, int nthreads);

/* --- leapfrog --------------------------------------------------------- */
void or_integrate_start(int dims, int64_t n, float *x, float *y, float *z,
                        float *vx, float *vy, float *vz, const float *ax, const float *ay,
                        const float *az, float *pvx, float *pvy, float *pvz,
                        const uint8_t *pinned, const or_params *p);
void or_integrate_end(int dims, int64_t n, float *vx, float *vy, float *vz,
                      const float *ax, const float *ay, const float *az,
                      const uint8_t *pinned, const or_params *p);

/* SPH neighbour grid: SPH::newGridGPU (SPH.h:533-590) -- the cell-key
 * shader (:101-152), the bitonic network as gpuBitonicSort drives it
 * (:247-296, :337-367) and the offsets shaders (:369-400, :455-470).
 * Outputs keys/index/cell_x/cell_y [n] in the network's order and
 * offsets [table]. */
void or_sph_grid(int64_t n, const float *x, const float *y, float cell, uint32_t table,
                 uint32_t *keys, uint32_t *index, int32_t *cell_x, int32_t *cell_y,
                 uint32_t *offsets);

/* --- one full frame of the gravity path -------------------------------
 * State arrays are in the current particle order and are permuted into
 * Morton order, exactly as the application's particle vectors are.  z, vz,
 * az, pvz are ignored in 2D; pvx..pvz, temp, pinned may be NULL.
 * walk: 0 = scalar tree walk (scalar direct sum below p->direct_below
 * particles), 1 = AVX2 tree walk, 2 = application dispatch (direct sum below
 * 5000 particles, AVX2 walk otherwise).
 * stage_ms (optional, [8]): integrateStart, bbox, keys, sort+gather, build,
 * walk, integrateEnd, total.  Returns 0, or -1 on allocation failure. */
int or_frame(const or_params *p, int64_t n, float *x, float *y, float *z,
             float *vx, float *vy, float *vz, float *ax, float *ay, float *az,
             float *m, uint32_t *id, float *pvx, float *pvy, float *pvz,
             float *temp, uint8_t *pinned, int walk, int nthreads,
             double *stage_ms, uint64_t *interactions, int64_t *nodes);

#ifdef __cplusplus
}
#endif
#endif
