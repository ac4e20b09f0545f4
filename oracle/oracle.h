/*
 * oracle.h -- FP64 CPU restatement of Grains3D's per-time-step DEM loop.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load liboracle.so, and only as the checker or as the timed
 * CPU baseline.  The product (grains3dgpu_b200) never links or calls it.
 *
 * Parity anchor: the restated functions follow the reference's operation
 * order, so on one machine they reproduce the reference's compiled CPU path
 * (oracle/_ref, built by oracle/ref/Makefile from the reference sources)
 * bit for bit.  tests/test_oracle_pinned.py checks that directly and against
 * golden fixtures in tests/golden/ generated from oracle/_ref.
 *
 * The system API (or_*) mirrors include/grains_b200.h one to one, so a test
 * drives the GPU engine and the oracle with the same calls.
 */
#ifndef GRAINS_ORACLE_H
#define GRAINS_ORACLE_H

#include "../include/grains_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Contact information (Grains/Geometry/include/ContactInfo.hh:19-21). */
typedef struct or_contact {
    double pt[3];
    double vec[3];
    double overlap;
} or_contact;

/* ---- per-function entry points (known-answer tests) ----------------------- */
int or_support(const gb_convex* c, const double* vertices, const double v[3],
               double out[3]);
int or_rigid_body_properties(const gb_rigid_body_desc* rb, const double* vertices,
                             gb_rigid_body_props* out);
int or_obb(const double ext_a[3], const double ext_b[3], const double a2w[12],
           const double b2w[12]);
/* GJK distance between two convexes; pa/pb in the local frames. */
double or_gjk(int variant, const gb_convex* a, const double* verts_a,
              const gb_convex* b, const double* verts_b, const double a2w[12],
              const double b2w[12], double pa[3], double pb[3], int* n_iter);
int or_closest_points(const gb_rigid_body_desc* rb_a, const double* verts_a,
                      const gb_rigid_body_desc* rb_b, const double* verts_b,
                      const double a2w[12], const double b2w[12], int gjk_variant,
                      or_contact* out);
/* HookeContactForceModel::computeForces: adds to force[3] and torque[3]. */
int or_hooke(const gb_contact_model* cm, const or_contact* ci,
             const double rel_vel[3], const double rel_ang_vel[3], double m1,
             double m2, const double tr_origin[3], double force[3],
             double torque[3]);
/* One FirstOrderExplicit move of one particle (ComponentManagerCPU.cpp:470-499):
 * tr[12] and kin[6] are updated in place; torce = force(3) torque(3). */
int or_move_first_order(const gb_rigid_body_props* rb, double dt, double tr[12],
                        double kin[6], const double torce[6]);
/* Linked cell (LinkedCell.cpp:16-73): cells per direction and cell hashes. */
int or_linked_cell_dims(const double min[3], const double max[3], double extent,
                        uint32_t dims[3]);
int or_cell_hash(const double min[3], const double max[3], double extent,
                 int64_t n, const double* pos3, uint32_t* hash);

/* ---- system API: mirrors gb_* in include/grains_b200.h --------------------- */
typedef struct or_ctx or_ctx;
or_ctx* or_create(const gb_config* cfg, int* status);
int or_destroy(or_ctx* ctx);
int or_set_threads(or_ctx* ctx, int32_t n_threads);
int or_set_rigid_bodies(or_ctx* ctx, const gb_rigid_body_desc* rbs,
                        const double* vertices, int64_t n_vertices);
int or_get_rigid_body_props(or_ctx* ctx, int32_t rb, gb_rigid_body_props* out);
int or_set_contact_models(or_ctx* ctx, const gb_contact_model* table);
/* Test hook: overrides the derived properties of rigid body `rb`. */
int or_set_rigid_body_props(or_ctx* ctx, int32_t rb, const gb_rigid_body_props* props);
int or_set_obstacles(or_ctx* ctx, const gb_rigid_body_desc* obstacles,
                     const double* transforms);
int or_set_obstacle_velocities(or_ctx* ctx, const double* kin);
int or_set_rigid_body_ids(or_ctx* ctx, const uint32_t* ids);
int or_set_transforms(or_ctx* ctx, const double* transforms);
int or_set_velocities(or_ctx* ctx, const double* kin);
int or_get_transforms(or_ctx* ctx, double* transforms);
int or_get_velocities(or_ctx* ctx, double* kin);
int or_get_torces(or_ctx* ctx, double* torce);
int or_set_torces(or_ctx* ctx, const double* torce);
/* Adjoint of one step from the current state (spheres, Hooke, first order):
   adj_next, adj_prev: 9 x n (position, velocity, angular velocity rows);
   grad_laws: 4 per law (kn, en, etat, muc), accumulated. */
int or_adjoint_step(or_ctx* ctx, const double* adj_next, double* adj_prev, double* grad_laws);
int or_update_links(or_ctx* ctx);
int or_detect_collision_and_compute_contact_forces(or_ctx* ctx, int32_t* result);
int or_add_external_forces(or_ctx* ctx);
int or_move_particles(or_ctx* ctx);
int or_step(or_ctx* ctx, int32_t n_steps);
int or_get_stats(or_ctx* ctx, gb_stats* out);
int or_debug_dump(or_ctx* ctx, int32_t kind, void* out, int64_t capacity,
                  int64_t* count);

#ifdef __cplusplus
}
#endif

#endif
