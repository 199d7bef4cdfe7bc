/*
 * ge_bh.h -- C ABI of the B200 Barnes-Hut gravity step (libgebh.so).
 *
 * Drop-in for Galaxy Engine's per-frame gravity path (paths relative to the
 * NarcisCalin/Galaxy-Engine checkout):
 *
 *   integrateStart -> boundingBox -> computeMortonKeys -> sortParticlesByMortonKey
 *   -> Quadtree/Octree build -> calculateForceFromGrid -> integrateEnd
 *   (GalaxyEngine/src/globalLogic.cpp:1155-1370 in 2D, :1584-1719 in 3D)
 *
 * Conventions
 *   - Every call returns a ge_status; 0 is success.  ge_last_error() returns a
 *     message for the last failure on that context.
 *   - Host buffers are caller-owned and only read/written during the call.
 *     Device state is owned by the context and stays resident between calls.
 *   - Particles are kept in Morton order: every step re-sorts them, exactly as
 *     the reference re-sorts its particle vectors every frame.  The uint32
 *     `id` array travels with the particles so results can be matched by id.
 *   - One host thread per context; different contexts are independent.  All
 *     device work of a context runs on its stream (ge_set_stream).
 *   - No entry point falls back to the CPU: without a usable CUDA device,
 *     ge_create fails with GE_ERR_NO_DEVICE.
 */
#ifndef GE_BH_H
#define GE_BH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GE_ABI_VERSION 1

typedef enum {
    GE_OK = 0,
    GE_ERR_ARG = 1,        /* invalid argument */
    GE_ERR_NO_DEVICE = 2,  /* no CUDA device / wrong architecture */
    GE_ERR_CUDA = 3,       /* CUDA runtime error (see ge_last_error) */
    GE_ERR_CAPACITY = 4,   /* node or stack capacity exceeded; raise node_cap_factor */
    GE_ERR_STATE = 5,      /* call made in the wrong state (e.g. no particles) */
    GE_ERR_TIMEOUT = 6,    /* a bounded device-side wait gave up */
    GE_ERR_OOM = 7,        /* device allocation failed or HBM budget exceeded */
    GE_ERR_UNSUPPORTED = 8 /* option not supported by this build */
} ge_status;

typedef enum {
    GE_PREC_FAST = 0,   /* FP32; MAC and tree arithmetic exactly as the reference,
                           force terms with rsqrt and FMA */
    GE_PREC_EXACT = 1,  /* FP32 with the reference's own rounding for every
                           operation (1/sqrtf, no contraction); for parity checks */
    GE_PREC_MIXED = 2   /* FP32 interactions on cell-relative positions, Kahan-
                           compensated accumulation and leapfrog update */
} ge_precision;

/*
 * Parameters.  Replaces the reference's UpdateVariables fields used on the
 * gravity path (GalaxyEngine/include/parameters.h:97-129,138,147,318).
 */
typedef struct {
    int32_t dims;            /* 2 (quadtree) or 3 (octree) */
    int32_t precision;       /* ge_precision */
    float G;                 /* myVar.G */
    float theta;             /* myVar.theta */
    float eps2;              /* value added to r^2: softening^2 in the 2D walk
                                (physics.cpp:100), softening in 3D (physics3D.cpp:166) */
    float dt;                /* myVar.timeFactor */
    uint32_t leaf_cap;       /* max particles in a leaf below the size gate (reference: 4) */
    float size_gate;         /* reference: 2.0f (quadtree.cpp:16) */
    float min_size;          /* reference: 1e-6f */
    float node_cap_factor;   /* node capacity = factor * N + 1024 (reference reserves 4N / 8N) */
    int32_t periodic;        /* periodic wrap (isPeriodicBoundaryEnabled && !infiniteDomain) */
    float domain[3];         /* domainSize / domainSize3D */
    int32_t track_prev_vel;  /* keep prevVel as the reference does (integrateStart) */
    int32_t group_size;      /* GE_PREC_MIXED walk: particles that share one traversal
                                (32, 64 or 128; 0 = every particle walks alone) */
    int32_t temp_enabled;    /* heat exchange in the walk (myVar.isTempEnabled, default off;
                                GE_PREC_EXACT / GE_PREC_FAST); temperatures via ge_upload_temp */
    float heat_cond;         /* myVar.globalHeatConductivity (parameters.h:120) */
    int32_t direct_below;    /* a simulation of fewer particles takes its accelerations
                                from the O(N^2) direct sum instead of the walk, as the
                                application does below 5000 (globalLogic.cpp:1321-1346,
                                3D :1677-1702; naiveGravity physics.cpp:392-434, 3D
                                physics3D.cpp:416-469); 0 = always walk, INT32_MAX =
                                always direct (myVar.naive); no heat exchange there;
                                GE_PREC_EXACT / GE_PREC_FAST */
    float direct_eps2;       /* value the direct sum adds to r^2: softening, un-squared
                                in 2D and 3D (physics.cpp:422, physics3D.cpp:455) */
    int32_t no_graph;        /* 1: ge_step launches every kernel itself; 0 (default):
                                pairs of steps replay a captured CUDA graph */
    int32_t walk_kind;       /* GE_PREC_FAST tree walk (same interaction set either way):
                                0 (default) every particle walks the depth-first layout
                                on its own; 1 the 32 particles of a warp walk together
                                (a shared node stack, nodes decided for the whole warp
                                against its bounding box, a staged source list, per-
                                particle walks only for the undecided subtrees); 1
                                needs eps2 > 0 and no periodic wrap or heat exchange,
                                otherwise the per-particle walk runs */
} ge_params;

typedef struct {
    int64_t n;               /* particles */
    int64_t nodes;           /* nodes in the last tree */
    int32_t depth;           /* levels in the last tree */
    int32_t steps;           /* steps run on this context */
    uint64_t interactions;   /* accepted monopoles + leaf pairs (j != i) in the last
                                force pass, when counting is enabled */
    float bbox[4];           /* last root box: x, y, (z,) size */
    float ms_last_step;      /* device time of the last ge_step call / nsteps */
    float stage_ms[8];       /* last ge_profile_step: kick+bbox, keys, sort, permute,
                                build, walk, total, unused */
} ge_stats;

typedef struct ge_ctx ge_ctx;

/* --- lifecycle -------------------------------------------------------- */
/* Fills the reference defaults: theta 0.8, softening 1.5 (eps2 = 2.25 in 2D,
   1.5 in 3D, direct_eps2 = 1.5), dt 0.045, G 6.674e-11, leaf_cap 4, size_gate 2,
   min_size 1e-6; direct_below 0 (the application's own dispatch is 5000). */
void ge_params_default(ge_params *p, int dims);
int ge_create(const ge_params *p, ge_ctx **out);
int ge_destroy(ge_ctx *ctx);
const char *ge_last_error(const ge_ctx *ctx);
int ge_set_params(ge_ctx *ctx, const ge_params *p);
/* Run the context's work on an existing cudaStream_t (NULL: the context's own). */
int ge_set_stream(ge_ctx *ctx, void *cuda_stream);
int ge_sync(ge_ctx *ctx);
int ge_get_stats(ge_ctx *ctx, ge_stats *out);
int ge_abi_version(void);

/* --- state I/O (host SoA buffers; z/vz/az ignored in 2D; NULL = skip) -- */
/* replaces Physics::flattenParticles (physics.cpp:354-390): the state goes to
   the device once and stays resident.  Accelerations start at 0 as in the
   reference's fresh particles (particle.h:49); ax/ay/az may seed them. */
int ge_upload(ge_ctx *ctx, int64_t n, const float *x, const float *y, const float *z,
              const float *vx, const float *vy, const float *vz, const float *m,
              const uint32_t *id, const float *ax, const float *ay, const float *az);
/* replaces Physics::readFlattenBack (physics.cpp:542-565) */
int ge_download(ge_ctx *ctx, float *x, float *y, float *z, float *vx, float *vy, float *vz,
                float *ax, float *ay, float *az, float *m, uint32_t *id);
/* optional per-particle pin flags (ParticleRendering::isPinned, particle.h:100),
   in the current particle order; NULL clears them */
int ge_upload_pinned(ge_ctx *ctx, const uint8_t *pinned);
int ge_download_prev_vel(ge_ctx *ctx, float *pvx, float *pvy, float *pvz);
/* particle temperatures (ParticlePhysics::temp), in the current particle
   order; with temp_enabled each step's walk exchanges heat as the reference
   does (physics.cpp:145-158, 183-191; physics3D.cpp:190-201, 230-237): an
   accepted node by its average temperature, a leaf's particles one by one,
   temp_i += heat_cond * (T - temp_i) / distance * dt.  The reference changes
   temp_i in place while other threads read it; here every particle reads the
   others' temperatures (and the node averages) as they were before the walk
   and accumulates its own in walk order. */
int ge_upload_temp(ge_ctx *ctx, const float *temp);
int ge_download_temp(ge_ctx *ctx, float *temp);

/* --- the reference's particle records (array of structures) --------------
 * The reference keeps its particles as two record arrays,
 * std::vector<ParticlePhysics> and std::vector<ParticleRendering>
 * (include/Particles/particle.h:5-140; ParticlePhysics3D /
 * ParticleRendering3D :142-277), copies the gravity members into SoA
 * vectors before the walk (Physics::flattenParticles, src/Physics/
 * physics.cpp:354-390) and back after it (readFlattenBack, :542-565), and
 * reorders both arrays by Morton key every frame (morton.cpp:40-63).
 * ge_frame_aos is one frame (as ge_frame_host) on those records as they
 * are: the members are read from the n physics records (and the pin flags
 * from the rendering records; rend may be NULL), and after the frame the
 * updated members -- pos, vel, acc, and prevVel with track_prev_vel, temp
 * with temp_enabled -- are written back into each particle's own record, so
 * the caller's arrays keep their order and their other members.  The
 * records go to the device in one copy per array and the changed bytes of
 * each record come back in one pitched copy (page-locked arrays copy
 * fastest).  order (optional, n entries) receives the Morton order the
 * reference would have moved its arrays to: order[k] = the record in slot k.
 * The layout gives the byte offsets of the members read and written (-1:
 * not present); ge_aos_layout_default fills the reference's (the offsets of
 * the structs in particle.h, pinned by a test that compiles that header).
 * Positions, velocities and accelerations are float vectors of dims
 * components; mass and temp floats; id uint32; isPinned one byte. */
typedef struct {
    int32_t stride;        /* bytes per physics record (sizeof ParticlePhysics[3D]) */
    int32_t off_pos, off_vel, off_acc;
    int32_t off_prev_vel;  /* written back with track_prev_vel; -1: none */
    int32_t off_mass, off_id;
    int32_t off_temp;      /* read and written back with temp_enabled; -1: none */
    int32_t r_stride;      /* bytes per rendering record (sizeof ParticleRendering[3D]) */
    int32_t r_off_pinned;  /* isPinned; -1: no pin flags */
} ge_aos_layout;
void ge_aos_layout_default(ge_aos_layout *layout, int dims);
int ge_frame_aos(ge_ctx *ctx, int64_t n, void *phys, const void *rend,
                 const ge_aos_layout *layout, uint32_t *order);

/* --- checkpoint / resume --------------------------------------------------
 * No counterpart in the reference, whose scene files (SaveSystem,
 * src/UX/saveSystem.cpp:285-410) keep no compensation terms.  The particle
 * state with every term the next step reads, as caller-owned host arrays in
 * the current particle order (all simulations, slot order); any pointer may
 * be NULL (z members ignored in 2D):
 *   x y z vx vy vz ax ay az m id   as ge_download / ge_upload
 *   kx ky kz kvx kvy kvz           GE_PREC_MIXED: the Kahan compensation terms
 *                                  of positions and velocities
 *   pvx pvy pvz                    prevVel (track_prev_vel)
 *   temp, pinned                   temperatures and pin flags
 * ge_download_state fills zeros for what the context does not hold (the
 * compensation terms outside GE_PREC_MIXED, prevVel without track_prev_vel,
 * temperatures or pin flags never uploaded).  ge_upload_state replaces the
 * context's particles by one simulation of n particles, as ge_upload does,
 * then sets every array given (compensation terms: GE_PREC_MIXED only, else
 * GE_ERR_STATE).  A context restored from a snapshot, with the same
 * parameters, steps on bit for bit as the context that wrote it. */
typedef struct {
    float *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
    uint32_t *id;
    float *kx, *ky, *kz, *kvx, *kvy, *kvz;
    float *pvx, *pvy, *pvz;
    float *temp;
    uint8_t *pinned;
} ge_state_arrays;
int ge_download_state(ge_ctx *ctx, const ge_state_arrays *s);
int ge_upload_state(ge_ctx *ctx, int64_t n, const ge_state_arrays *s);

/* --- the fused step ---------------------------------------------------- */
/* nsteps full frames on the resident state (globalLogic.cpp:1155-1370 /
   :1584-1719 with dt != 0), all on the device. */
int ge_step(ge_ctx *ctx, int32_t nsteps);
/* The same in two halves: ge_step_async enqueues the frames on the context's
   stream and returns at once; ge_step_wait waits for them and reports
   errors and timing.  Contexts on different streams then step concurrently.
   Between the two calls only ge_step_wait, ge_sync and ge_get_stats may be
   used on the context. */
int ge_step_async(ge_ctx *ctx, int32_t nsteps);
int ge_step_wait(ge_ctx *ctx);
/* Autotuner of the mixed mode's group walk (no counterpart in the
   reference).  On the resident state, times the force pass -- tree build,
   node moments and the group walk, best of `reps` after a warm-up -- for
   every group_size in {32, 64, 128} and leaf_cap in {1, 4, 8, 16}, keeps the
   fastest in the context's parameters (ge_set_params can override it) and
   recomputes the accelerations with it.  Positions and velocities are not
   changed.  ms[4 * g + l] is the time of group size g and leaf capacity l in
   those orders.  GE_ERR_STATE outside GE_PREC_MIXED: the other modes keep the
   reference's leaf capacity. */
typedef struct {
    int32_t group_size, leaf_cap;   /* chosen */
    int32_t tried;                  /* configurations measured */
    int32_t reserved;
    float ms[12];
} ge_tune_result;
int ge_autotune(ge_ctx *ctx, int32_t reps, ge_tune_result *out);
/* one frame with per-stage CUDA-event timing into ge_stats.stage_ms */
int ge_profile_step(ge_ctx *ctx);
/* One frame on HOST buffers: upload, step, download, all inside the call.
   This is the reference-facing drop-in for the gravity block of
   updateScene(): arrays are updated in place and come back in Morton order
   (id says which particle is where), like the reference's pParticles. */
int ge_frame_host(ge_ctx *ctx, int64_t n, float *x, float *y, float *z, float *vx, float *vy,
                  float *vz, float *ax, float *ay, float *az, float *m, uint32_t *id);

/* --- stage calls mirroring the reference surface (for parity tests) ---- */
/* Physics::integrateStart (physics.cpp:1069-1112) */
int ge_integrate_start(ge_ctx *ctx);
/* boundingBox / boundingBox3D (globalLogic.cpp:1083-1099 / :1460-1477); out:
   {x, y, size} in 2D, {x, y, z, size} in 3D */
int ge_bounding_box(ge_ctx *ctx, float *out);
/* Morton::computeMortonKeys[3D] (morton.cpp:27-38 / :92-112) for the current
   order and root box; keys_out (optional) receives them */
int ge_compute_morton_keys(ge_ctx *ctx, uint64_t *keys_out);
/* Morton::sortParticlesByMortonKey[3D] (morton.cpp:40-63 / :114-138): stable
   radix sort of the keys and the gather of the whole state; perm_out
   (optional) receives the index each slot came from */
int ge_sort_by_morton_key(ge_ctx *ctx, uint32_t *perm_out);
/* Quadtree / Octree construction with mass and centre of mass
   (quadtree.cpp:5-292) over the current (sorted) order */
int ge_build_tree(ge_ctx *ctx);
/* Physics::calculateForceFromGrid[3D] (physics.cpp:91-205 / physics3D.cpp:131-253):
   accelerations of every particle from the current tree */
int ge_compute_forces(ge_ctx *ctx);
/* Physics::integrateEnd (physics.cpp:1114-1125) */
int ge_integrate_end(ge_ctx *ctx);
/* enable per-particle interaction counting in ge_compute_forces (stats) */
int ge_set_count_interactions(ge_ctx *ctx, int32_t enable);
/* Test hook for the failure path of the bounded device-side waits (no
   counterpart in the reference, whose GL path only prints shader errors,
   globalLogic.cpp:601-615).  spin_limit caps every look-back wait of the key
   sort at that many polls (0 restores the default, 2^22).  withhold = 1
   makes the first tile of every pass of ge_sort_by_morton_key keep its digit
   counts to itself, so the waits of the tiles after it run out: that call
   returns GE_ERR_TIMEOUT and the particle state is unspecified until the
   next ge_upload (the frame calls, ge_step and ge_frame_host, never
   withhold).  Nothing faults or hangs: every wait is bounded, and the sort's
   scatter and gather stay inside their arrays whatever the waits found.
   withhold = 0 restores normal operation.  Kept across reallocations. */
int ge_set_sort_wait_test(ge_ctx *ctx, uint32_t spin_limit, int32_t withhold);

/* --- trajectory preview ------------------------------------------------
 * ParticlesSpawning::predictTrajectory (particlesSpawning.cpp:443-500, 3D
 * :1000-1060): nprobes probe particles (pos, vel: [nprobes * dims] host
 * arrays; mass [nprobes]) are each stepped `steps` times against the tree of
 * the last step, which is not rebuilt, with the older walk the preview uses
 * (Physics::calculateForceFromGridOld, physics.cpp:4-90 / physics3D.cpp:
 * 49-120: leaves taken whole, a one-particle leaf within 0.001 of the probe
 * skipped).  eps2 is the value that walk adds to r^2: softening^2 in both 2D
 * and 3D.  path [nprobes * steps * dims] receives each step's position.
 * sim: the simulation's handle (0: the context's first simulation).  Needs
 * GE_PREC_EXACT or GE_PREC_FAST (the walk layout holds node sizes). */
int ge_predict_trajectory(ge_ctx *ctx, int32_t sim, int32_t nprobes, const float *pos,
                          const float *vel, const float *mass, float eps2, int32_t steps,
                          float *path);

/* --- gravity field display ----------------------------------------------
 * The reference's field view (include/Physics/field.h: cells of
 * initializeCells :59-80, compute shader fieldGravityCompute :106-160,
 * fragment shader fieldFragmentShader :165-222), run as CUDA on the resident
 * particles of one simulation (2D): each cell's strength
 * sum_j G * (10 m_j) / (|p_j - corner|^2 + softness^2) (minimum image when
 * periodic, terms with distance <= 1e-4 left out) and, when rgba is not NULL,
 * its colour as RGBA8 (one pixel per cell; no window on this library's
 * side).  Cells: size = min(domain) / res, amount_x x amount_y of them,
 * index j + i * amount_y for the cell with corner (i, j) * size.  Arrays
 * hold cap cells; GE_ERR_CAPACITY (with *amount_x, *amount_y set) when
 * they are too small.  sim: handle, 0 = the first simulation. */
typedef struct {
    int32_t res;              /* Field::res (150) */
    float softness;           /* gravityDisplaySoftness (0.85) */
    float threshold;          /* gravityDisplayThreshold (1000) */
    float stretch;            /* gravityStretchFactor (90) */
    float exposure;           /* gravityExposure (3) */
    int32_t two_color;        /* gravityCustomColors (0: HSV ramp) */
    float color_low[3];       /* colorVisuals.pColor / 255 */
    float color_high[3];      /* colorVisuals.sColor / 255 */
    int32_t reserved[4];
} ge_field_params;
void ge_field_params_default(ge_field_params *fp);
int ge_gravity_field(ge_ctx *ctx, int32_t sim, const ge_field_params *fp, int64_t cap,
                     float *strength, uint8_t *rgba, int32_t *amount_x, int32_t *amount_y);

/* --- SPH neighbour grid (2D) -------------------------------------------
 * Replaces SPH::newGridGPU (GalaxyEngine/include/Physics/SPH.h:533-590 with
 * its shaders :101-152, :247-296, :369-400, :455-470).  For one simulation's
 * particles in their current order (sim 0 = the first or only one):
 * cell (cx, cy) = floor(position / cell_size); key = (uint32(cx * 73856093) ^
 * uint32(cy * 19349663)) % table_size with wrapping 32-bit products; the
 * entries {key, particle, cx, cy} sorted by key (stable: a key's particles in
 * increasing order; the reference's bitonic network leaves ties in an order
 * of its own); offsets[key] = the key's first entry, UINT32_MAX for a key no
 * particle has.  keys/index/cell_x/cell_y hold n entries (cap >= n), offsets
 * table_size entries.  The reference uses hashTableSize 16384 and cellSize =
 * radiusMultiplier = 3 (SPH.h:16,28,97).  table_size in [1, 2^24]. */
int ge_sph_grid(ge_ctx *ctx, int32_t sim, float cell_size, uint32_t table_size, int64_t cap,
                uint32_t *keys, uint32_t *index, int32_t *cell_x, int32_t *cell_y,
                uint32_t *offsets);

/* --- scene files -------------------------------------------------------
 * Reader of the reference's save files (SaveSystem, src/UX/saveSystem.cpp:
 * 285-362; include/UX/saveSystem.h:120-290; versions 190 and 180): the YAML
 * parameter block (is3DMode decides the dimension), then per particle the
 * binary ParticlePhysics(3D) / ParticleRendering(3D) members
 * (include/Particles/particle.h).  Host code only; no context or GPU needed.
 * ge_save_read_info gives the header; ge_save_read copies the members the
 * gravity step uses into caller arrays of at least `cap` particles, in the
 * file's order (any pointer may be NULL; z/vz/az ignored in 2D):
 * positions, velocities, accelerations, mass, temperature, id, isPinned.
 * GE_ERR_UNSUPPORTED for other versions, GE_ERR_ARG for a missing,
 * malformed or truncated file, GE_ERR_CAPACITY when cap is too small. */
typedef struct {
    uint32_t version;
    int32_t dims;
    int64_t n;
    uint32_t global_id, global_shape_id, global_wall_id;
    int32_t record_bytes;      /* bytes per particle record (180 in 2D, 208 in 3D) */
} ge_save_info;
int ge_save_read_info(const char *path, ge_save_info *info);
int ge_save_read(const char *path, int64_t cap, float *x, float *y, float *z, float *vx,
                 float *vy, float *vz, float *ax, float *ay, float *az, float *m, float *temp,
                 uint32_t *id, uint8_t *pinned);

/* --- FP64 diagnostics (accuracy reference; not on the step path) ------- */
/* Direct-sum accelerations in FP64 of the particles at indices idx[0..nt) of
   the current order: sum over j != i of G m_j d / (|d|^2 + eps2)^(3/2), j over
   the particle's own sim.
   ax/ay/az (host, nt doubles each; az ignored in 2D). */
int ge_direct_sum_f64(ge_ctx *ctx, int64_t nt, const uint32_t *idx, double *ax, double *ay,
                      double *az);
/* FP64 sums over the state: out = {kinetic energy, p_x, p_y, p_z, total mass} */
int ge_sums_f64(ge_ctx *ctx, double *out);
/* Energy of the current state (no counterpart in the reference):
   out = {kinetic, potential, total}, kinetic summed in FP64 over the
   particles, potential = 1/2 sum_i m_i phi_i with phi_i from the mixed
   mode's group walk (monopole + quadrupole of the softened kernel, the
   particle itself left out) summed in FP64; over all simulations of the
   context.  Needs GE_PREC_MIXED with the group walk (group_size > 0, not
   periodic); builds the tree when the last step's is not current. */
int ge_energy_f64(ge_ctx *ctx, double *out);
/* Timeline of the last tree build: device time (ns, from the first entry) at
   each of its grid-wide barriers, in order (the pending-count phase, one per
   level of the large-node phase, the rebuild and subtree phase, the
   end-count scan), then the start of the layout scatter and the end of the
   build (stamped by the last block to finish).  Profiling aid with no
   counterpart in the reference. */
int ge_build_timeline(ge_ctx *ctx, int32_t cap, uint64_t *ns, int32_t *count);

/* --- 2D Morton sort without device allocation --------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory, such as an application that carves its device
 * memory into a fixed arena up front and accounts for every byte itself, or
 * a frame loop that must not call cudaMalloc / cudaFree because they can
 * synchronise the whole device mid-frame.
 *
 * Same result as ge_compute_morton_keys + ge_sort_by_morton_key on a context
 * (root box, Morton keys, stable radix sort), on caller-owned DEVICE buffers:
 * d_x, d_y (n floats each, read), d_perm (n uint32: the input index that
 * lands in each sorted slot), d_keys (optional, n uint64: the sorted keys).
 * `stream` is a cudaStream_t (NULL: the legacy default stream).
 *
 * All temporaries live in one fixed-size device array inside the library
 * (about 5.1 MB on every GPU that loads it, held until the process exits), so
 * n is limited to GE_NOALLOC_MAX_N; larger n returns GE_ERR_CAPACITY without
 * launching anything.  The first call on each device looks up that array's
 * device address (cudaGetSymbolAddress) for the current device; make that
 * first call before any stream capture.  Every call shares the one array:
 * calls that overlap on the GPU (other streams, other host threads) race and
 * corrupt each other's results, so serialise them.  The call waits for its
 * work to finish and returns GE_ERR_TIMEOUT if a bounded device-side wait gave
 * up.  It calls no allocating routine. */
#define GE_NOALLOC_MAX_N 262144
int ge_morton_sort_2d_noalloc(int64_t n, const float *d_x, const float *d_y, uint32_t *d_perm,
                              uint64_t *d_keys, void *stream);

/* --- batched simulations -----------------------------------------------
 * No counterpart in the reference (one particle system per process).  A
 * context holds any number of independent simulations ("sims") of its dims
 * and parameters; every ge_step / ge_batch_step advances all of them with
 * one launch per stage.  Each sim keeps its own particle range, root box,
 * Morton order and tree; no sim sees another's particles, so every sim's
 * result is the same as stepping it alone in its own context.
 * ge_upload replaces all sims by a single one.  Handles are positive and
 * never reused within a context.  Adding or removing a sim waits for the
 * context's stream and may reallocate (existing state is kept). */
/* same as ge_create / ge_step */
int ge_batch_create(const ge_params *p, ge_ctx **out);
int ge_batch_step(ge_ctx *ctx, int32_t nsteps);
/* appends a sim of n >= 1 particles (host SoA, as ge_upload; id NULL =
   0..n-1); *sim receives its handle */
int ge_batch_add_sim(ge_ctx *ctx, int64_t n, const float *x, const float *y, const float *z,
                     const float *vx, const float *vy, const float *vz, const float *m,
                     const uint32_t *id, int32_t *sim);
/* removes a sim; the others keep their state */
int ge_batch_remove_sim(ge_ctx *ctx, int32_t sim);
/* removes count sims at once (one compaction) */
int ge_batch_remove_sims(ge_ctx *ctx, int32_t count, const int32_t *sims);
/* number of sims and, when sims != NULL, up to cap handles in slot order */
int ge_batch_list(ge_ctx *ctx, int32_t cap, int32_t *sims, int32_t *count);
/* a sim's particle count, first slot in the context's arrays, and steps taken
   since it was added (any pointer may be NULL) */
int ge_batch_query(ge_ctx *ctx, int32_t sim, int64_t *n, int64_t *offset, int64_t *steps);
/* one sim's state (its particles in its Morton order), as ge_download */
int ge_batch_download_sim(ge_ctx *ctx, int32_t sim, float *x, float *y, float *z, float *vx,
                          float *vy, float *vz, float *ax, float *ay, float *az, float *m,
                          uint32_t *id);

/* --- device memory ------------------------------------------------------
 * No counterpart in the reference.  A context's device memory is its
 * particle capacity (state, sort scratch, node arrays sized node_cap_factor
 * times the capacity) plus per-simulation tables.  ge_reserve sizes it up
 * front for n particles in up to `sims` simulations, so that later uploads
 * and additions within those limits never reallocate; ge_memory_bytes
 * reports what the context holds; ge_estimate_bytes reports what a context
 * with these parameters would hold after ge_reserve(n, sims). */
int ge_reserve(ge_ctx *ctx, int64_t n, int64_t sims);
int ge_memory_bytes(ge_ctx *ctx, int64_t *bytes);
int ge_estimate_bytes(const ge_params *p, int64_t n, int64_t sims, int64_t *bytes);

/* --- serving ------------------------------------------------------------
 * No counterpart in the reference.  A server runs requests -- a simulation
 * plus a step count -- with continuous batching under a device-memory
 * budget.  It owns two batch contexts (pools: params[0] for 2D requests,
 * params[1] for 3D), each reserved once at creation from its share of
 * hbm_budget_bytes (frac_2d for 2D, the rest for 3D), so the pools together
 * never hold more than the budget and admission never allocates.  Each
 * pool's loop (its own worker thread after ge_server_start; both pools per
 * ge_server_poll call on the calling thread) admits queued requests first
 * come first served while the pool has room (particles and max_sims), takes
 * one step of all of its admitted simulations (the two pools step at their
 * own rates and their kernels overlap on the device), and retires
 * simulations that reached their step count: their final state is copied to
 * host memory and their room freed.
 * A result equals the same request run alone on a context with the same
 * parameters.  submit / status / wait / take / get_stats may be called from
 * any thread. */
typedef struct ge_server ge_server;

typedef enum {
    GE_REQ_QUEUED = 0,
    GE_REQ_RUNNING = 1,
    GE_REQ_DONE = 2,
    GE_REQ_FAILED = 3
} ge_request_state;

typedef struct {
    int64_t hbm_budget_bytes;  /* device memory of both pools together */
    double frac_2d;            /* share of the budget for the 2D pool */
    int32_t max_sims;          /* simulations per pool at once */
    int32_t reserved[7];
    ge_params params[2];       /* [0]: 2D pool (dims 2), [1]: 3D pool (dims 3) */
} ge_server_config;

typedef struct {
    int64_t submitted, completed, failed, queued, running;
    int64_t iterations;          /* batched steps taken (both pools) */
    int64_t particle_steps;      /* particles stepped, summed over iterations */
    double busy_s;               /* wall time spent in batched steps (both pools) */
    double step_ms_p50, step_ms_p99;      /* wall time of one batched step */
    double latency_s_p50, latency_s_p99;  /* submit -> done, completed requests */
    int64_t pool_bytes[2];       /* device memory held by each pool */
    int64_t pool_capacity[2];    /* particles each pool runs at once */
    int64_t pool_iterations[2];
    double pool_step_ms_p50[2], pool_step_ms_p99[2];
    double pool_busy_s[2];       /* wall time of each pool's batched steps */
    double pool_admit_s[2];      /* ... adding admitted simulations to the pool */
    double pool_retire_s[2];     /* ... copying finished ones out and compacting */
    int64_t pool_particle_steps[2];
    double queue_wait_s_p50, queue_wait_s_p99;   /* submit -> admit, admitted requests */
} ge_server_stats;

int ge_server_create(const ge_server_config *cfg, ge_server **out);
int ge_server_destroy(ge_server *srv);
const char *ge_server_last_error(const ge_server *srv);
/* queues a request (the host arrays are copied); *request receives its id.
   GE_ERR_CAPACITY when n exceeds its pool's capacity. */
int ge_server_submit(ge_server *srv, int32_t dims, int64_t n, const float *x, const float *y,
                     const float *z, const float *vx, const float *vy, const float *vz,
                     const float *m, int32_t steps, int64_t *request);
int ge_server_start(ge_server *srv);
/* stops the worker after its current iteration; returns the loop's error */
int ge_server_stop(ge_server *srv);
/* one loop iteration on the calling thread (server not started);
   *stepped = 1 when a batched step ran */
int ge_server_poll(ge_server *srv, int32_t *stepped);
/* waits (worker running) until the request is done; GE_ERR_TIMEOUT after
   timeout_s seconds */
int ge_server_wait(ge_server *srv, int64_t request, double timeout_s);
/* state (ge_request_state), steps taken, and submit-to-done seconds (-1 until done) */
int ge_server_status(ge_server *srv, int64_t request, int32_t *state, int32_t *steps_done,
                     double *latency_s);
/* copies a finished request's final state (its particles in Morton order,
   id = index in the submitted arrays) and releases it */
int ge_server_take(ge_server *srv, int64_t request, float *x, float *y, float *z, float *vx,
                   float *vy, float *vz, float *ax, float *ay, float *az, float *m,
                   uint32_t *id);
int ge_server_get_stats(ge_server *srv, ge_server_stats *out);

/* --- tree export: the reference's globalNodes in DFS pre-order --------- */
/* Returns the node count in *count (with several sims: every sim's tree, one
   after another in slot order).  Arrays (capacity cap nodes; any may be
   NULL): pos/com [cap*dims], size, mass [cap], start, end, next [cap],
   child [cap * 2^dims] with child[q], q = xbit | ybit<<1 (| zbit<<2), the
   reference's subGrids[x][y]([z]); 0xFFFFFFFF marks an empty slot. */
int ge_export_tree(ge_ctx *ctx, int64_t cap, int64_t *count, float *pos, float *size,
                   float *com, float *mass, uint32_t *start, uint32_t *end, uint32_t *next,
                   uint32_t *child);

#ifdef __cplusplus
}
#endif
#endif
