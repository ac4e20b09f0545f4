/*
 * grains_b200.h -- C ABI of the B200 DEM time-step engine.
 *
 * The engine replaces the per-time-step loop of Grains3D's ComponentManager
 * (Grains/Component/include/ComponentManager.hh:130-182): linked-cell broad
 * phase, GJK narrow phase, contact law, per-particle reduction and time
 * integration, run as sm_100a CUDA kernels on one GPU.  Every entry point
 * uses plain C types (pointers, sizes, PODs) so that a C++ ComponentManager
 * subclass, a ctypes binding or any other FFI can bind it directly.
 *
 * Conventions
 *   - Every call returns GB_OK (0) or a negative GB_E_* status; nothing
 *     exits or aborts.  gb_status_string() names a status.
 *   - A context owns all device memory and one CUDA stream.  Calls on one
 *     context are not thread-safe; different contexts are independent.
 *   - Host buffers are plain row-major double arrays.  A transform is 12
 *     doubles: the 3x3 basis row-major (Mxx Mxy Mxz Myx ... Mzz) followed by
 *     the origin (Ox Oy Oz), the layout of Grains' Transform3 buffer
 *     (Grains/Geometry/src/Transform3.cpp:26-29, :133-137).
 *   - Calls that read state back to the host synchronise the context stream.
 */
#ifndef GRAINS_B200_H
#define GRAINS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GB_ABI_VERSION 1

/* ---- status codes --------------------------------------------------------- */
#define GB_OK 0
#define GB_E_INVALID_ARG (-1)   /* bad pointer, size or enum value            */
#define GB_E_CUDA (-2)          /* a CUDA runtime call failed                  */
#define GB_E_OUT_OF_MEMORY (-3) /* device allocation failed                    */
#define GB_E_NOT_READY (-4)     /* call order: e.g. a step before set_state    */
#define GB_E_OUT_OF_DOMAIN (-5) /* a particle centre left the linked-cell grid */
#define GB_E_NONFINITE (-6)     /* NaN/Inf found in the particle state         */
#define GB_E_NO_DEVICE (-7)     /* no usable CUDA device                       */
#define GB_E_CAPACITY (-8)      /* a fixed-size buffer is too small            */
#define GB_E_UNSUPPORTED (-9)   /* feature/shape combination not available     */

/* ---- convex types: the values of Grains' ConvexType enum
 *      (Grains/Geometry/include/Convex.hh:7-16) -------------------------------
 * p[] holds
 *   GB_SPHERE        r
 *   GB_BOX           half edge lengths ex ey ez   (Box(T x, T y, T z), Box.cpp:6-8)
 *   GB_SUPERQUADRIC  a b c n1 n2                  (Superquadric.cpp:10-17)
 *   GB_POLYHEDRON    (unused) vertices come from the vertex pool
 *   GB_RECTANGLE     half edge lengths LX/2 LY/2  (plane z=0 of its frame)
 *   GB_DRUM          radius, half-length           (obstacles only; see below)
 */
#define GB_SPHERE 0
#define GB_BOX 1
#define GB_CYLINDER 2 /* not provided: GB_E_UNSUPPORTED */
#define GB_CONE 3     /* not provided: GB_E_UNSUPPORTED */
#define GB_SUPERQUADRIC 4
#define GB_POLYHEDRON 5
#define GB_RECTANGLE 6
/* NEW (no reference shape): an obstacle only -- the inner surface of a
 * circular cylinder (a rotating drum's wall) of radius p[0] and half-length
 * p[1] about its frame's z axis, the particles inside it.  A particle meets
 * it at the tangent plane of the wall point nearest its centre, evaluated as
 * closestPointsRectangle evaluates a plane (CollisionDetection.cpp:53-90). */
#define GB_DRUM 7

#define GB_MAX_POLY_VERTICES 64

/* ---- run modes -------------------------------------------------------------- */
#define GB_FP64 0        /* every kernel in double precision, FMA contraction on  */
#define GB_MIXED 1       /* FP32 bulk; FP64 positions and candidate tests, FP64 GJK */
#define GB_FP64_STRICT 2 /* FP64 in the reference's IEEE operation order (no FMA
                            contraction): the parity mode                          */

#define GB_LAW_HOOKE 0         /* HookeContactForceModel (parity)          */
#define GB_LAW_HOOKE_HISTORY 1 /* spring-dashpot + Coulomb-capped tangential
                                  spring with per-pair history               */

#define GB_FIRST_ORDER_EXPLICIT 0 /* FirstOrderExplicit (parity)             */
#define GB_VELOCITY_VERLET 1      /* velocity-Verlet / leapfrog              */

#define GB_GJK_JH 0       /* Johnson sub-algorithm with cached determinants */
#define GB_GJK_SV 1       /* signed-volume sub-algorithm                    */
#define GB_GJK_NESTEROV 2 /* Nesterov-accelerated GJK                       */

/* ---- plain-data descriptors ---------------------------------------------------*/
typedef struct gb_convex {
    int32_t type;         /* GB_SPHERE ... GB_RECTANGLE                          */
    int32_t n_vertices;   /* GB_POLYHEDRON: vertex count (4..GB_MAX_POLY_VERTICES)*/
    int64_t first_vertex; /* GB_POLYHEDRON: first vertex index in the pool        */
    double p[5];
} gb_convex;

/* One Grains RigidBody (Grains/Geometry/src/RigidBody.cpp:19-59):
 * RigidBody(convex, crustThickness, material, density). */
typedef struct gb_rigid_body_desc {
    gb_convex convex;
    double crust_thickness;
    double density; /* 0 for obstacles: mass and inertia are 0 */
    int32_t material;
    int32_t reserved;
} gb_rigid_body_desc;

/* Derived rigid-body properties, as RigidBody computes them. */
typedef struct gb_rigid_body_props {
    double volume;
    double mass;
    double circumscribed_radius;
    double bounding_box[3]; /* half extents of the local bounding box */
    double inertia[6];      /* xx xy xz yy yz zz, times density     */
    double inertia_inv[6];  /* inverse, divided by density           */
} gb_rigid_body_props;

/* Contact-law parameters of one material pair: HookeContactForceModel's
 * kn, en, etat, muc, kr (HookeContactForceModel.cpp:48-57) plus the tangential
 * spring stiffness kt of the history law.  The table is indexed like
 * ContactForceModelBuilderFactory::computeHash: l*(l+1)/2 + s with
 * l = max(matA, matB), s = min(matA, matB). */
typedef struct gb_contact_model {
    double kn, en, etat, muc, kr, kt;
} gb_contact_model;

typedef struct gb_config {
    int32_t n_particles;
    int32_t n_rigid_bodies; /* entries of the rigid-body table               */
    int32_t n_obstacles;
    int32_t n_materials;
    double origin[3];         /* GrainsParameters::m_origin (LinkedCell min)  */
    double max_coordinate[3]; /* GrainsParameters::m_maxCoordinate            */
    double cell_size_factor;  /* LinkedCell CellSizeFactor, clamped to >= 1   */
    int32_t pad_grid;         /* 1: max += one cell size per axis so that the
                                 floored cell count covers the whole box      */
    int32_t precision;        /* GB_FP64 | GB_MIXED                           */
    double dt;
    double gravity[3];
    int32_t contact_law; /* GB_LAW_*          */
    int32_t integrator;  /* GB_FIRST_ORDER_EXPLICIT | GB_VELOCITY_VERLET */
    int32_t gjk_variant; /* GB_GJK_*          */
    int32_t device;      /* CUDA device ordinal */
    int64_t pair_capacity; /* initial candidate-pair capacity, 0 = automatic */
    int32_t flags;         /* GB_FLAG_* */
    int32_t reserved;
} gb_config;

/* gb_config.flags */
#define GB_FLAG_RECORD_CONTACT_INFO 1 /* keep per-pair contact info for dumps   */
#define GB_FLAG_PHASE_TIMING 2        /* CUDA-event timing of each step phase */
/* Bounding tests that include the crust: the circumscribed radius and the
 * bounding box's half-extents of every rigid body grow by its crust thickness
 * in the candidate test, the linked-cell size and the OBB pre-filter.  Off
 * (the reference's rule), those bound the shapes alone while a contact starts
 * once the shapes come within the crusts' sum, so a body whose box is tight
 * (a cube as a box or polyhedron) first reaches the closest-point solver
 * when it already intersects its neighbour, where the contact normal is 0/0
 * (CollisionDetection.cpp:208-245).  The sphere-sphere closed form keeps the
 * radius. */
#define GB_FLAG_CRUST_BOUNDS 4

/* Step phases timed under GB_FLAG_PHASE_TIMING (gb_get_phase_times). */
#define GB_PHASE_HASH 0       /* cell hash per particle                       */
#define GB_PHASE_SORT 1       /* radix sort of (cell, id)                     */
#define GB_PHASE_CELL_START 2 /* cell-start table + sorted positions          */
#define GB_PHASE_PAIR_COUNT 3 /* candidate count + scan                       */
#define GB_PHASE_PAIR_FILL 4  /* candidate pair records                       */
#define GB_PHASE_NARROW 5     /* OBB + GJK + contact law per pair             */
#define GB_PHASE_PARTICLE 6   /* reduction + walls + gravity + integration    */
#define GB_N_PHASES 7

/* Counters of the last completed step (or of the last detect call). */
typedef struct gb_stats {
    int64_t steps_done;
    int64_t candidate_pairs;  /* ordered pairs passing the bounding-sphere test */
    int64_t contacts;         /* ordered particle pairs with overlap < 0         */
    int64_t obstacle_contacts;
    int64_t gjk_calls;        /* particle pairs past the bounding tests and GJK's first
                                 iteration (queued for the GJK pass)           */
    int64_t gjk_iterations;   /* summed over the steps of the last gb_step call */
    int32_t status_flags; /* bit i set: device-side error (1 << -GB_E_x)    */
    int32_t n_cells;
    int32_t cells_per_dir[3];
    int32_t key_bits;
    double cell_size;
    double grid_max[3];      /* linked-cell max corner actually used */
    int64_t kernel_launches; /* kernels launched by this context so far */
    int64_t gjk_fp64_calls;  /* particle pairs solved by the FP64 GJK (GB_MIXED: those its
                                FP32 stage leaves open; otherwise gjk_calls) */
    int64_t fine_grid_cells; /* cells of the finer candidate grid of a polydisperse packing
                                (0: candidates from the linked cells alone) */
    int64_t obstacle_candidates; /* particle-obstacle records of the last detect (the obstacles
                                    past the first 32 come from linked-cell bins) */
} gb_stats;

/* ---- debug dump kinds -------------------------------------------------------- */
#define GB_DUMP_CELL_HASH 0       /* uint32[N]: cell hash per particle id          */
#define GB_DUMP_SORTED_IDS 1      /* uint32[N]: particle ids sorted by (cell, id)  */
#define GB_DUMP_CELL_START 2      /* uint32[C+1]: first sorted index of each cell  */
#define GB_DUMP_CANDIDATE_PAIRS 3 /* uint32[2P]: (A,B) ordered candidate pairs     */
#define GB_DUMP_CONTACT_PAIRS 4   /* uint32[2K]: (A,B) pairs with overlap < 0      */
#define GB_DUMP_CONTACT_INFO 5    /* double[7K]: contact point, vector, overlap    */
#define GB_DUMP_NEIGHBORS 6       /* uint32[27C]: neighbour table (UINT32_MAX out) */
#define GB_DUMP_CONTACT_FORCES 7  /* double[6K]: force, torque on A of each contact
                                     pair, in GB_DUMP_CONTACT_PAIRS order           */

typedef struct gb_ctx gb_ctx;

/* ---- lifetime ------------------------------------------------------------------ */
gb_ctx* gb_create(const gb_config* cfg, int* status);
int gb_destroy(gb_ctx* ctx);
const char* gb_status_string(int status);
int gb_abi_version(void);

/* ---- set-up (Grains::Construction, Grains/Base/src/Grains.cpp:90-300) ----------- */
/* Rigid-body table; `vertices` holds 3 doubles per polyhedron vertex. */
int gb_set_rigid_bodies(gb_ctx* ctx, const gb_rigid_body_desc* rbs,
                        const double* vertices, int64_t n_vertices);
int gb_get_rigid_body_props(gb_ctx* ctx, int32_t rb, gb_rigid_body_props* out);
/* n_materials*(n_materials+1)/2 entries. */
int gb_set_contact_models(gb_ctx* ctx, const gb_contact_model* table);
/* Obstacles: n_obstacles rigid bodies (density 0) and their transforms. */
int gb_set_obstacles(gb_ctx* ctx, const gb_rigid_body_desc* obstacles,
                     const double* transforms);
/* Moving walls (no counterpart in the reference, whose obstacles are at rest,
 * ComponentManagerCPU.cpp:326-336): 6 doubles per obstacle, the velocity of
 * its origin and its angular velocity (world axes).  They enter the contact
 * laws as the wall's velocity at the contact point, v + w x (p - origin);
 * the wall's geometry stays where gb_set_obstacles put it (a surface velocity:
 * a drum turning about its own axis, a conveyor), and a caller that moves a
 * wall calls gb_set_obstacles again between steps.  Zero until set. */
int gb_set_obstacle_velocities(gb_ctx* ctx, const double* kin);

/* ---- particle state (ComponentManager set/get, ComponentManager.hh:37-104) ------ */
int gb_set_rigid_body_ids(gb_ctx* ctx, const uint32_t* ids);
int gb_set_transforms(gb_ctx* ctx, const double* transforms); /* 12 per particle */
int gb_set_velocities(gb_ctx* ctx, const double* kin);        /* v(3) omega(3)   */
int gb_get_transforms(gb_ctx* ctx, double* transforms);
int gb_get_velocities(gb_ctx* ctx, double* kin);
/* Torce per particle: force(3) torque(3), accumulated since the last move. */
int gb_get_torces(gb_ctx* ctx, double* torce);
/* ComponentManager::setTorce (ComponentManager.hh:93): replaces the
 * accumulated torces; the next detect and add_external_forces add to them and
 * the next move consumes and resets them, as in ComponentManagerCPU. */
int gb_set_torces(gb_ctx* ctx, const double* torce);

/* ---- differentiable stepping (no counterpart in the reference) ------------------
 * FP64 modes only.  A state is 18 rows of n doubles on the device: position
 * (3), Transform3 basis (9, row-major), velocity (3), angular velocity (3). */
int gb_save_state(gb_ctx* ctx, double* dst_device);
int gb_load_state(gb_ctx* ctx, const double* src_device);
/* GB_VELOCITY_VERLET: started = 0 makes the next step a trajectory's first
 * (a half kick of the velocities, dt/2), 1 a later one (a full kick, dt).  A
 * context starts at 0 and every step sets 1; a trajectory replayed from a
 * saved state sets the phase it had there. */
int gb_set_integrator_phase(gb_ctx* ctx, int32_t started);
/* Reverse-mode derivative of one step from the current state s, for spheres,
 * GB_LAW_HOOKE with kr = 0, GB_FIRST_ORDER_EXPLICIT or GB_VELOCITY_VERLET (the
 * step's kick as gb_set_integrator_phase left it) and Rectangle walls
 * (GB_E_UNSUPPORTED otherwise).  adj_next = dL/ds' and adj_prev = dL/ds are
 * 9 rows of n doubles on the device (position, velocity, angular velocity);
 * dL/dtheta is added to grad_laws (device, 4 doubles per contact law: kn, en,
 * etat, muc).  The contacts are those found at s; the state and the torces
 * are left as they were. */
int gb_adjoint_step(gb_ctx* ctx, const double* adj_next, double* adj_prev, double* grad_laws);
/* The contact set of the last detect (pair list and contact flags), so that a
 * replayed step's adjoint need not detect again: gb_save_contacts copies it to
 * `buf` (device memory of `capacity` bytes; NULL only queries) and sets *size
 * to the bytes it needs (GB_E_CAPACITY when capacity is short); after
 * gb_load_state of the state that detect was made on, gb_load_contacts puts it
 * back, and the next gb_adjoint_step uses it instead of detecting.  Any step,
 * detect or load_state drops a loaded set. */
int gb_save_contacts(gb_ctx* ctx, void* buf, int64_t capacity, int64_t* size);
int gb_load_contacts(gb_ctx* ctx, const void* buf);

/* ---- the time step: the ComponentManager hot-path calls ---------------------- */
/* ComponentManager::updateLinks (ComponentManagerCPU.cpp:278-296). */
int gb_update_links(gb_ctx* ctx);
/* ComponentManager::detectCollisionAndComputeContactForces
 * (ComponentManagerCPU.cpp:428-443): updateLinks, particle-particle and
 * particle-obstacle contacts, forces added to the torces.  `result` (host,
 * n_particles ints, may be NULL) is incremented per particle by the number of
 * ordered contacts, like the reference's `int* result`. */
int gb_detect_collision_and_compute_contact_forces(gb_ctx* ctx, int32_t* result);
/* ComponentManager::addExternalForces (ComponentManagerCPU.cpp:448-460). */
int gb_add_external_forces(gb_ctx* ctx);
/* ComponentManager::moveParticles (ComponentManagerCPU.cpp:465-500). */
int gb_move_particles(gb_ctx* ctx);
/* n_steps of GrainsCPU::simulate's loop body (GrainsCPU.cpp:55-66), fused. */
int gb_step(gb_ctx* ctx, int32_t n_steps);

/* ---- diagnostics ---------------------------------------------------------------- */
int gb_get_stats(gb_ctx* ctx, gb_stats* out);
/* Copies a dump (GB_DUMP_*) of the last detect step to `out` (host memory of
 * `capacity` elements); *count receives the number of elements available. */
int gb_debug_dump(gb_ctx* ctx, int32_t kind, void* out, int64_t capacity,
                  int64_t* count);
/* Device pointers of the SoA state for zero-copy consumers (torch, CUDA code).
 * names: "pos_x" "pos_y" "pos_z" (double), "vel_x" ... "omega_z" "force_x" ...
 * "torque_z" (double in the FP64 modes, float in GB_MIXED), "rotation" (the
 * FP64 modes: 9 rows of n doubles, the Transform3 basis row-major; GB_MIXED:
 * 8 rows of n floats, the unit quaternion w x y z followed by its FP32
 * remainder, whose sum is the orientation), "rb_id" (uint32). */
int gb_device_pointer(gb_ctx* ctx, const char* name, void** ptr);
/* Synchronises the context stream and returns the device-side status flags. */
int gb_synchronize(gb_ctx* ctx);
/* Runs the context on the caller's CUDA stream (a cudaStream_t; NULL returns
 * to the context's own stream).  The caller keeps ownership of the stream. */
int gb_set_stream(gb_ctx* ctx, void* cuda_stream);
/* Accumulated device time per phase (GB_N_PHASES doubles, milliseconds) and
 * the number of steps they cover, when GB_FLAG_PHASE_TIMING is set; `reset`
 * clears the accumulators after reading. */
int gb_get_phase_times(gb_ctx* ctx, double* ms, int64_t* steps, int32_t reset);

/* ---- linked-cell sort without device allocation -------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory where they need the broad phase (their device memory is wholly
 * reserved by another allocator, or their time loop must not block on a
 * cudaMalloc): the cell hash, stable radix sort of (cell, particle id) and
 * cell-start table of gb_update_links, with all scratch in a static device
 * array of the library sized for at most 262,144 particles (about 6.4 MB held
 * on every GPU that loads the library).  Nothing is allocated.
 *   pos         device, 3*n doubles: x[n], y[n], z[n]
 *   origin      host, the linked-cell min corner; cell_size and dims (host)
 *               describe the grid as gb_get_stats reports it
 *   sorted_ids  device, n uint32: particle ids sorted by (cell, id)
 *   cell_start  device, dims[0]*dims[1]*dims[2]+1 uint32
 *   stream      cudaStream_t (NULL: the legacy default stream)
 * Returns GB_E_CAPACITY when n exceeds 262,144.  Every call synchronises
 * `stream` to report GB_E_OUT_OF_DOMAIN / GB_E_NONFINITE like gb_update_links,
 * so no call may be made while the stream is being captured into a CUDA
 * graph.  All calls share the scratch: calls whose work overlaps on the GPU
 * race and must be serialised by the caller. */
int gb_linked_cell_sort_static(const double* pos, int32_t n, const double origin[3],
                               double cell_size, const int32_t dims[3], uint32_t* sorted_ids,
                               uint32_t* cell_start, void* stream);

/* ---- RawData post-processing output ------------------------------------------------
 * RawDataPostProcessingWriter (PostProcessing/src/RawDataPostProcessingWriter.cpp:
 * PostProcessing_start :63-71, PostProcessing :75-212, PostProcessing_end :218-231),
 * called where Grains drives its writers (Grains.cpp:52, :66, :82).  Files
 * <directory>/<root_name>_{position,translational_velocity,angular_velocity}_{x,y,z}.dat
 * get one line per save: the time, every particle's value, then every obstacle's
 * (origin; zero velocities), each printed as realToString(ios::scientific, 6, v)
 * ("%.6e"; a zero as "0").  _coordinationNumber.dat gets an empty line per save, as
 * the reference writes it, or with GB_RAW_COORDINATION_NUMBER the time and each
 * particle's particle-contact count of the last detect.  _particleType.dat holds one
 * empty line.  gb_rawdata_write snapshots the state on the context's stream after
 * the work launched before it and returns; the files are written by a host thread
 * while later steps run, and the next write or the close waits for it (and returns
 * its status). */
#define GB_RAW_COORDINATION_NUMBER 1
typedef struct gb_rawdata_writer gb_rawdata_writer;
int gb_rawdata_open(gb_ctx* ctx, const char* directory, const char* root_name, int32_t flags,
                    gb_rawdata_writer** out);
int gb_rawdata_write(gb_rawdata_writer* writer, double time);
int gb_rawdata_close(gb_rawdata_writer* writer);

/* ---- host set-up helpers (no context needed) ------------------------------------- */
/* Volume, mass, circumscribed radius, bounding box and inertia of a rigid
 * body as RigidBody::RigidBody computes them; polyhedra use their convex
 * hull.  `vertices` may be NULL unless the convex is a polyhedron. */
int gb_rigid_body_properties(const gb_rigid_body_desc* rb, const double* vertices,
                             gb_rigid_body_props* out);
/* Convex hull of n points (n <= GB_MAX_POLY_VERTICES): writes the hull's
 * centroid to centroid[3] and its volume to *volume. */
int gb_convex_hull_centroid(const double* points, int32_t n, double* centroid,
                            double* volume);

#ifdef __cplusplus
}
#endif

#endif /* GRAINS_B200_H */
