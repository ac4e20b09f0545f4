// ref_harness.cpp -- exposes the reference's own CPU code (Grains3DGPU, compiled
// from its sources by oracle/ref/Makefile into oracle/_ref/libgrainsref.so)
// behind the oracle's C API with a ref_ prefix.
//
// TEST INFRASTRUCTURE: used to pin the oracle restatement, to generate the
// golden fixtures in tests/golden/, and as the timed CPU baseline.  Everything
// numeric here is done by reference classes; this file only marshals plain
// arrays into them and replays GrainsCPU::simulate's call order
// (Grains/Base/src/GrainsCPU.cpp:55-66).
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ComponentManagerCPU.hh"
#include "Box.hh"
#include "CollisionDetection.hh"
#include "ContactForceModelBuilderFactory.hh"
#include "FirstOrderExplicit.hh"
#include "GJK_AY.hh"
#include "GJK_JH.hh"
#include "HookeContactForceModel.hh"
#include "LinkedCell.hh"
#include "OBB.hh"
#include "RawDataPostProcessingWriter.hh"
#include "Rectangle.hh"
#include "RigidBody.hh"
#include "Sphere.hh"
#include "Superquadric.hh"
#include "VectorMath.hh"

#include "../oracle.h"

using T = double;

namespace
{
Convex<T>* make_convex(const gb_convex* c)
{
    switch(c->type)
    {
        case GB_SPHERE:
            return new Sphere<T>(c->p[0]);
        case GB_BOX:
            return new Box<T>(c->p[0], c->p[1], c->p[2]); // half extents
        case GB_SUPERQUADRIC:
            return new Superquadric<T>(c->p[0], c->p[1], c->p[2], c->p[3], c->p[4]);
        case GB_RECTANGLE:
            return new Rectangle<T>(T(2) * c->p[0], T(2) * c->p[1]); // full lengths
        default:
            return nullptr; // the reference has no polyhedron
    }
}

RigidBody<T, T>* make_rb(const gb_rigid_body_desc* d)
{
    Convex<T>* cv = make_convex(&d->convex);
    if(!cv)
        return nullptr;
    return new RigidBody<T, T>(cv, d->crust_thickness, (uint)d->material, d->density);
}

void props_of(const RigidBody<T, T>& rb, gb_rigid_body_props* o)
{
    o->volume               = rb.getVolume();
    o->mass                 = rb.getMass();
    o->circumscribed_radius = rb.getCircumscribedRadius();
    Vector3<T> e            = rb.getBoundingBox()->getExtent();
    for(int k = 0; k < 3; ++k)
        o->bounding_box[k] = e[k];
    rb.getInertia(o->inertia);
    rb.getInertia_1(o->inertia_inv);
}

void put_contact(const ContactInfo<T>& ci, or_contact* o)
{
    Vector3<T> p = ci.getContactPoint(), v = ci.getContactVector();
    for(int k = 0; k < 3; ++k)
    {
        o->pt[k]  = p[k];
        o->vec[k] = v[k];
    }
    o->overlap = ci.getOverlapDistance();
}

// ComponentManagerCPU with access to its cell lists.  updateLinks clears
// m_cell[0..m_nCells] inclusive (ComponentManagerCPU.cpp:281-282), one past
// the end of the vector; reserving spare capacity keeps that write inside
// this object's own allocation.
class HarnessManager : public ComponentManagerCPU<T>
{
public:
    HarnessManager(uint np, uint no, uint nc)
        : ComponentManagerCPU<T>(np, no, nc)
    {
        this->m_cell.reserve(this->m_cell.size() + 4);
    }
    const std::vector<std::vector<uint>>& cells() const
    {
        return this->m_cell;
    }
    const std::vector<uint>& cellHash() const
    {
        return this->m_particleCellHash;
    }
};
} // namespace

extern "C" {

int ref_support(const gb_convex* c, const double* vertices, const double v[3], double out[3])
{
    (void)vertices;
    Convex<T>* cv = make_convex(c);
    if(!cv)
        return GB_E_UNSUPPORTED;
    Vector3<T> s = cv->support(Vector3<T>(v[0], v[1], v[2]));
    for(int k = 0; k < 3; ++k)
        out[k] = s[k];
    delete cv;
    return GB_OK;
}

int ref_rigid_body_properties(const gb_rigid_body_desc* d, const double* vertices,
                              gb_rigid_body_props* out)
{
    (void)vertices;
    RigidBody<T, T>* rb = make_rb(d);
    if(!rb)
        return GB_E_UNSUPPORTED;
    props_of(*rb, out);
    return GB_OK; // RigidBody owns no destructor for its convex; leak is test-only
}

int ref_obb(const double ext_a[3], const double ext_b[3], const double a2w[12],
            const double b2w[12])
{
    BoundingBox<T> a(ext_a[0], ext_a[1], ext_a[2]), b(ext_b[0], ext_b[1], ext_b[2]);
    return intersectOrientedBoundingBox(a, b, Transform3<T>(a2w), Transform3<T>(b2w)) ? 1 : 0;
}

double ref_gjk(int variant, const gb_convex* a, const double* verts_a, const gb_convex* b,
               const double* verts_b, const double a2w[12], const double b2w[12],
               double pa[3], double pb[3], int* n_iter)
{
    (void)verts_a;
    (void)verts_b;
    Convex<T>* ca = make_convex(a);
    Convex<T>* cb = make_convex(b);
    if(!ca || !cb)
        return -1.0;
    Vector3<T> va, vb;
    int        it = 0;
    T          d;
    if(variant == GB_GJK_SV)
        d = computeClosestPoints_GJK_AY(*ca, *cb, Transform3<T>(a2w), Transform3<T>(b2w), va, vb, it);
    else
        d = computeClosestPoints_GJK_JH(*ca, *cb, Transform3<T>(a2w), Transform3<T>(b2w), va, vb, it);
    for(int k = 0; k < 3; ++k)
    {
        pa[k] = va[k];
        pb[k] = vb[k];
    }
    if(n_iter)
        *n_iter = it;
    delete ca;
    delete cb;
    return d;
}

int ref_closest_points(const gb_rigid_body_desc* rb_a, const double* verts_a,
                       const gb_rigid_body_desc* rb_b, const double* verts_b,
                       const double a2w[12], const double b2w[12], int gjk_variant,
                       or_contact* out)
{
    (void)verts_a;
    (void)verts_b;
    (void)gjk_variant;
    RigidBody<T, T>* A = make_rb(rb_a);
    RigidBody<T, T>* B = make_rb(rb_b);
    if(!A || !B)
        return GB_E_UNSUPPORTED;
    ContactInfo<T> ci = closestPointsRigidBodies(*A, *B, Transform3<T>(a2w), Transform3<T>(b2w));
    put_contact(ci, out);
    return GB_OK;
}

int ref_hooke(const gb_contact_model* cm, const or_contact* c, const double rel_vel[3],
              const double rel_ang_vel[3], double m1, double m2, const double tr_origin[3],
              double force[3], double torque[3])
{
    HookeContactForceModel<T> law(cm->kn, cm->en, cm->etat, cm->muc, cm->kr);
    ContactInfo<T>            ci(Vector3<T>(c->pt[0], c->pt[1], c->pt[2]),
                      Vector3<T>(c->vec[0], c->vec[1], c->vec[2]),
                      c->overlap);
    Torce<T> t(Vector3<T>(torque[0], torque[1], torque[2]),
               Vector3<T>(force[0], force[1], force[2]));
    law.computeForces(ci,
                      Vector3<T>(rel_vel[0], rel_vel[1], rel_vel[2]),
                      Vector3<T>(rel_ang_vel[0], rel_ang_vel[1], rel_ang_vel[2]),
                      m1,
                      m2,
                      Vector3<T>(tr_origin[0], tr_origin[1], tr_origin[2]),
                      t);
    Vector3<T> f = t.getForce(), q = t.getTorque();
    for(int k = 0; k < 3; ++k)
    {
        force[k]  = f[k];
        torque[k] = q[k];
    }
    return GB_OK;
}

int ref_linked_cell_dims(const double min[3], const double max[3], double extent,
                         uint32_t dims[3])
{
    LinkedCell<T> lc(Vector3<T>(min[0], min[1], min[2]), Vector3<T>(max[0], max[1], max[2]),
                     extent);
    // number of cells per direction recovered from the neighbour table extent
    uint32_t n = lc.getNumCells();
    // dims are not exposed by the reference; probe them with computeLinearCellHash
    uint3 one_x = {1, 0, 0}, one_y = {0, 1, 0}, one_z = {0, 0, 1};
    uint32_t sx = lc.computeLinearCellHash(one_x);
    uint32_t sy = lc.computeLinearCellHash(one_y);
    uint32_t sz = lc.computeLinearCellHash(one_z);
    (void)sx;
    dims[0] = sy;
    dims[1] = sy ? sz / sy : 0;
    dims[2] = sz ? n / sz : 0;
    return GB_OK;
}

int ref_cell_hash(const double min[3], const double max[3], double extent, int64_t n,
                  const double* pos3, uint32_t* hash)
{
    LinkedCell<T> lc(Vector3<T>(min[0], min[1], min[2]), Vector3<T>(max[0], max[1], max[2]),
                     extent);
    for(int64_t i = 0; i < n; ++i)
        hash[i] = lc.computeLinearCellHash(
            Vector3<T>(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]));
    return GB_OK;
}

// ---------------------------------------------------------------------------
// The system: ComponentManagerCPU + RigidBody/LinkedCell/ContactForceModel/
// TimeIntegrator objects built as Grains::Construction builds them
// (Grains/Base/src/Grains.cpp:90-300), minus the XML.
struct ref_ctx
{
    gb_config                      cfg;
    std::vector<RigidBody<T, T>*>  prb, orb;
    std::vector<gb_rigid_body_desc> rbd;
    LinkedCell<T>*                 lc = nullptr;
    HarnessManager*                cm = nullptr;
    std::vector<ContactForceModel<T>*> cf;
    TimeIntegrator<T>*             ti = nullptr;
    std::vector<int>               result;
    double                         cell = 0, lc_max[3] = {0, 0, 0};
    uint32_t                       ncells = 0;
    int64_t                        steps  = 0;
    bool                           detected = false;
    // the reference's RawData writer (ref_rawdata_write) and its XML node
    std::unique_ptr<DOMElement>                          raw_node;
    std::unique_ptr<RawDataPostProcessingWriter<T>>      raw;
};

ref_ctx* ref_create(const gb_config* cfg, int* status)
{
    if(!cfg || cfg->n_particles < 0 || cfg->n_rigid_bodies < 1 || cfg->n_materials < 1)
    {
        if(status)
            *status = GB_E_INVALID_ARG;
        return nullptr;
    }
    // the reference's own law, integrator and bounding tests only
    if(cfg->contact_law != GB_LAW_HOOKE || cfg->integrator != GB_FIRST_ORDER_EXPLICIT
       || (cfg->flags & GB_FLAG_CRUST_BOUNDS))
    {
        if(status)
            *status = GB_E_UNSUPPORTED;
        return nullptr;
    }
    ref_ctx* c = new ref_ctx;
    c->cfg     = *cfg;
    c->result.assign(cfg->n_particles, 0);
    c->ti = new FirstOrderExplicit<T>(cfg->dt);
    if(status)
        *status = GB_OK;
    return c;
}

// The reference's RawDataPostProcessingWriter (RawDataPostProcessingWriter.cpp:
// 13-22 from an XML node, PostProcessing_start :63-71, PostProcessing :75-212,
// PostProcessing_end :218-231) on the harness's particles and obstacles.  The
// first call (`first` != 0) builds the writer from <RawData Directory=...
// RootName=...> (through the Xerces-free ReaderXML) and starts it, which
// removes earlier files of that root name in the directory; each call writes
// one save at `time`.
int ref_rawdata_write(ref_ctx* c, const char* directory, const char* root_name, double time,
                      int32_t first)
{
    if(!c || !c->cm || !directory || !root_name)
        return GB_E_INVALID_ARG;
    if(first || !c->raw)
    {
        auto quote = [](std::string v) {
            std::string o;
            for(char ch : v)
                o += ch == '"' ? std::string("&quot;") : ch == '&' ? std::string("&amp;")
                     : ch == '<' ? std::string("&lt;") : std::string(1, ch);
            return o;
        };
        std::string err;
        c->raw.reset();
        c->raw_node = gb::xml::parse("<RawData Directory=\"" + quote(directory) + "\" RootName=\""
                                         + quote(root_name) + "\"/>",
                                     &err);
        if(!c->raw_node)
            return GB_E_INVALID_ARG;
        c->raw.reset(new RawDataPostProcessingWriter<T>(c->raw_node.get()));
        c->raw->PostProcessing_start();
    }
    c->raw->PostProcessing(c->prb.data(), c->orb.data(), c->cm, T(time));
    return GB_OK;
}

int ref_rawdata_close(ref_ctx* c)
{
    if(!c)
        return GB_E_INVALID_ARG;
    if(c->raw)
        c->raw->PostProcessing_end();
    c->raw.reset();
    return GB_OK;
}

int ref_destroy(ref_ctx* c)
{
    if(!c)
        return GB_E_INVALID_ARG;
    c->raw.reset();
    delete c->cm;
    delete c->lc;
    delete c->ti;
    for(auto* f : c->cf)
        delete f;
    delete c;
    return GB_OK;
}

int ref_set_rigid_bodies(ref_ctx* c, const gb_rigid_body_desc* rbs, const double* vertices,
                         int64_t n_vertices)
{
    (void)vertices;
    (void)n_vertices;
    c->prb.clear();
    c->rbd.assign(rbs, rbs + c->cfg.n_rigid_bodies);
    T lcs = 0;
    for(int i = 0; i < c->cfg.n_rigid_bodies; ++i)
    {
        RigidBody<T, T>* rb = make_rb(&rbs[i]);
        if(!rb)
            return GB_E_UNSUPPORTED;
        c->prb.push_back(rb);
        if(rb->getCircumscribedRadius() > lcs) // Grains.cpp:226-231
            lcs = rb->getCircumscribedRadius();
    }
    T coeff = T(c->cfg.cell_size_factor);
    if(coeff < T(1))
        coeff = T(1);
    c->cell = coeff * T(2) * lcs; // Grains.cpp:242
    for(int k = 0; k < 3; ++k)
        c->lc_max[k] = c->cfg.max_coordinate[k] + (c->cfg.pad_grid ? c->cell : 0.0);
    c->lc = new LinkedCell<T>(
        Vector3<T>(c->cfg.origin[0], c->cfg.origin[1], c->cfg.origin[2]),
        Vector3<T>(c->lc_max[0], c->lc_max[1], c->lc_max[2]),
        c->cell);
    c->ncells = c->lc->getNumCells();
    c->cm     = new HarnessManager(c->cfg.n_particles, c->cfg.n_obstacles, c->ncells);
    return GB_OK;
}

int ref_get_rigid_body_props(ref_ctx* c, int32_t rb, gb_rigid_body_props* out)
{
    if(!c || rb < 0 || rb >= (int32_t)c->prb.size())
        return GB_E_INVALID_ARG;
    props_of(*c->prb[rb], out);
    return GB_OK;
}

int ref_set_contact_models(ref_ctx* c, const gb_contact_model* t)
{
    const int n = c->cfg.n_materials * (c->cfg.n_materials + 1) / 2;
    for(auto* f : c->cf)
        delete f;
    c->cf.clear();
    for(int i = 0; i < n; ++i)
        c->cf.push_back(new HookeContactForceModel<T>(t[i].kn, t[i].en, t[i].etat, t[i].muc, t[i].kr));
    return GB_OK;
}

int ref_set_obstacles(ref_ctx* c, const gb_rigid_body_desc* ob, const double* tr)
{
    if(!c->cm)
        return GB_E_NOT_READY;
    c->orb.clear();
    std::vector<uint>          ids;
    std::vector<Transform3<T>> trs;
    for(int i = 0; i < c->cfg.n_obstacles; ++i)
    {
        RigidBody<T, T>* rb = make_rb(&ob[i]);
        if(!rb)
            return GB_E_UNSUPPORTED;
        c->orb.push_back(rb);
        ids.push_back(i);
        trs.push_back(Transform3<T>(tr + 12 * i));
    }
    c->cm->setRigidBodyIdObstacles(ids);
    c->cm->setTransformObstacles(trs);
    return GB_OK;
}

int ref_set_rigid_body_ids(ref_ctx* c, const uint32_t* ids)
{
    if(!c->cm)
        return GB_E_NOT_READY;
    c->cm->setRigidBodyId(std::vector<uint>(ids, ids + c->cfg.n_particles));
    return GB_OK;
}

int ref_set_transforms(ref_ctx* c, const double* t)
{
    if(!c->cm)
        return GB_E_NOT_READY;
    std::vector<Transform3<T>> v;
    for(int i = 0; i < c->cfg.n_particles; ++i)
        v.push_back(Transform3<T>(t + 12 * i));
    c->cm->setTransform(v);
    return GB_OK;
}

int ref_set_velocities(ref_ctx* c, const double* k)
{
    if(!c->cm)
        return GB_E_NOT_READY;
    std::vector<Kinematics<T>> v;
    for(int i = 0; i < c->cfg.n_particles; ++i)
        v.push_back(Kinematics<T>(Vector3<T>(k[6 * i], k[6 * i + 1], k[6 * i + 2]),
                                  Vector3<T>(k[6 * i + 3], k[6 * i + 4], k[6 * i + 5])));
    c->cm->setVelocity(v);
    return GB_OK;
}

int ref_get_transforms(ref_ctx* c, double* t)
{
    std::vector<Transform3<T>> v = c->cm->getTransform();
    for(size_t i = 0; i < v.size(); ++i)
    {
        Matrix3<T> b = v[i].getBasis();
        Vector3<T> o = v[i].getOrigin();
        for(int r = 0; r < 3; ++r)
            for(int s = 0; s < 3; ++s)
                t[12 * i + 3 * r + s] = b[r][s];
        for(int k = 0; k < 3; ++k)
            t[12 * i + 9 + k] = o[k];
    }
    return GB_OK;
}

int ref_get_velocities(ref_ctx* c, double* k)
{
    std::vector<Kinematics<T>> v = c->cm->getVelocity();
    for(size_t i = 0; i < v.size(); ++i)
    {
        Vector3<T> a = v[i].getTranslationalComponent(), w = v[i].getAngularComponent();
        for(int j = 0; j < 3; ++j)
        {
            k[6 * i + j]     = a[j];
            k[6 * i + 3 + j] = w[j];
        }
    }
    return GB_OK;
}

int ref_get_torces(ref_ctx* c, double* t)
{
    std::vector<Torce<T>> v = c->cm->getTorce();
    for(size_t i = 0; i < v.size(); ++i)
    {
        Vector3<T> f = v[i].getForce(), q = v[i].getTorque();
        for(int j = 0; j < 3; ++j)
        {
            t[6 * i + j]     = f[j];
            t[6 * i + 3 + j] = q[j];
        }
    }
    return GB_OK;
}

int ref_set_torces(ref_ctx* c, const double* t)
{
    std::vector<Torce<T>> v(c->cfg.n_particles);
    for(size_t i = 0; i < v.size(); ++i)
        v[i] = Torce<T>(Vector3<T>(t[6 * i + 3], t[6 * i + 4], t[6 * i + 5]),
                        Vector3<T>(t[6 * i], t[6 * i + 1], t[6 * i + 2]));
    c->cm->setTorce(v);
    return GB_OK;
}

int ref_update_links(ref_ctx* c)
{
    LinkedCell<T>* lcp = c->lc;
    c->cm->updateLinks(&lcp);
    c->detected = true;
    return GB_OK;
}

int ref_detect_collision_and_compute_contact_forces(ref_ctx* c, int32_t* result)
{
    LinkedCell<T>*          lcp = c->lc;
    std::vector<int>        res(c->cfg.n_particles, 0);
    c->cm->detectCollisionAndComputeContactForces(
        c->prb.data(), c->orb.data(), &lcp, c->cf.data(), res.data());
    if(result)
        for(int i = 0; i < c->cfg.n_particles; ++i)
            result[i] += res[i];
    c->detected = true;
    return GB_OK;
}

int ref_add_external_forces(ref_ctx* c)
{
    c->cm->addExternalForces(
        c->prb.data(), Vector3<T>(c->cfg.gravity[0], c->cfg.gravity[1], c->cfg.gravity[2]));
    return GB_OK;
}

int ref_move_particles(ref_ctx* c)
{
    c->cm->moveParticles(c->prb.data(), &c->ti);
    ++c->steps;
    return GB_OK;
}

int ref_step(ref_ctx* c, int32_t n)
{
    for(int32_t s = 0; s < n; ++s)
    {
        ref_detect_collision_and_compute_contact_forces(c, nullptr);
        ref_add_external_forces(c);
        ref_move_particles(c);
    }
    return GB_OK;
}

int ref_get_stats(ref_ctx* c, gb_stats* o)
{
    std::memset(o, 0, sizeof(*o));
    o->steps_done = c->steps;
    o->n_cells    = (int32_t)c->ncells;
    o->cell_size  = c->cell;
    for(int k = 0; k < 3; ++k)
        o->grid_max[k] = c->lc_max[k];
    uint32_t d[3];
    ref_linked_cell_dims(c->cfg.origin, c->lc_max, c->cell, d);
    for(int k = 0; k < 3; ++k)
        o->cells_per_dir[k] = (int32_t)d[k];
    return GB_OK;
}

// Dumps of the last updateLinks / detect call: cell hashes and cell lists
// straight from the manager, pair sets by calling closestPointsRigidBodies
// over the manager's own cell lists and the LinkedCell neighbour table, in
// the order of ComponentManagerCPU.cpp:364-421.
int ref_debug_dump(ref_ctx* c, int32_t kind, void* out, int64_t capacity, int64_t* count)
{
    if(!c->detected)
        return GB_E_NOT_READY;
    const auto&  cells = c->cm->cells();
    const auto&  hash  = c->cm->cellHash();
    uint32_t*    o32   = (uint32_t*)out;
    double*      o64   = (double*)out;
    int64_t      w     = 0;
    const int    n     = c->cfg.n_particles;
    switch(kind)
    {
        case GB_DUMP_CELL_HASH:
            for(int i = 0; i < n; ++i)
                if(out && w < capacity)
                    o32[w++] = hash[i];
                else
                    ++w;
            break;
        case GB_DUMP_SORTED_IDS:
            for(uint32_t h = 0; h < c->ncells; ++h)
                for(uint id : cells[h])
                    if(out && w < capacity)
                        o32[w++] = id;
                    else
                        ++w;
            break;
        case GB_DUMP_CELL_START:
        {
            uint32_t acc = 0;
            for(uint32_t h = 0; h <= c->ncells; ++h)
            {
                if(out && w < capacity)
                    o32[w] = acc;
                ++w;
                if(h < c->ncells)
                    acc += (uint32_t)cells[h].size();
            }
            break;
        }
        case GB_DUMP_NEIGHBORS:
            for(uint32_t h = 0; h < c->ncells; ++h)
            {
                const uint* nb = c->lc->getNeighbors(h);
                for(int i = 0; i < 27; ++i)
                {
                    if(out && w < capacity)
                        o32[w] = nb[i];
                    ++w;
                }
            }
            break;
        case GB_DUMP_CANDIDATE_PAIRS:
        case GB_DUMP_CONTACT_PAIRS:
        case GB_DUMP_CONTACT_INFO:
        {
            std::vector<uint>          rbid = c->cm->getRigidBodyId();
            std::vector<Transform3<T>> tr   = c->cm->getTransform();
            int64_t                    k    = 0;
            for(int a = 0; a < n; ++a)
            {
                const RigidBody<T, T>& A  = *c->prb[rbid[a]];
                const uint*            nb = c->lc->getNeighbors(hash[a]);
                for(int i = 0; i < 27; ++i)
                {
                    if(nb[i] == UINT_MAX)
                        continue;
                    for(uint b : cells[nb[i]])
                    {
                        if(b == (uint)a)
                            continue;
                        const RigidBody<T, T>& B = *c->prb[rbid[b]];
                        if(kind == GB_DUMP_CANDIDATE_PAIRS)
                        {
                            T ov = norm(tr[b].getOrigin() - tr[a].getOrigin())
                                   - (A.getCircumscribedRadius() + B.getCircumscribedRadius());
                            if(!(ov < T(0)))
                                continue;
                        }
                        else
                        {
                            ContactInfo<T> ci = closestPointsRigidBodies(A, B, tr[a], tr[b]);
                            if(!(ci.getOverlapDistance() < T(0)))
                                continue;
                            if(kind == GB_DUMP_CONTACT_INFO)
                            {
                                or_contact oc;
                                put_contact(ci, &oc);
                                if(out && 7 * k + 7 <= capacity)
                                {
                                    std::memcpy(o64 + 7 * k, oc.pt, 3 * sizeof(double));
                                    std::memcpy(o64 + 7 * k + 3, oc.vec, 3 * sizeof(double));
                                    o64[7 * k + 6] = oc.overlap;
                                }
                                ++k;
                                continue;
                            }
                        }
                        if(out && 2 * k + 2 <= capacity)
                        {
                            o32[2 * k]     = (uint32_t)a;
                            o32[2 * k + 1] = b;
                        }
                        ++k;
                    }
                }
            }
            w = kind == GB_DUMP_CONTACT_INFO ? 7 * k : 2 * k;
            break;
        }
        default:
            return GB_E_INVALID_ARG;
    }
    *count = w;
    return GB_OK;
}

} // extern "C"
