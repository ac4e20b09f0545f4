// grains_b200_component_manager.hh -- ComponentManagerB200<T>, the drop-in
// for Grains3D's ComponentManager<T> (Grains/Component/include/
// ComponentManager.hh:24-185) that runs the DEM time step on a B200 through
// the C ABI of grains_b200.h.
//
// Header-only.  Include it from code that is compiled together with the
// Grains headers (it uses RigidBody, Convex, Transform3, Kinematics, Torce,
// LinkedCell, HookeContactForceModel and TimeIntegrator as the reference
// declares them) and link libgrains_b200.so.  Where Grains::Construction
// creates `new ComponentManagerCPU<T>(...)` (Grains/Base/src/Grains.cpp), a
// caller creates a ComponentManagerB200<T> instead, or builds the host
// manager as before and copies it over with ComponentManager<T>::copy, as the
// reference's GPU path does.  GrainsCPU::simulate's loop
// (Grains/Base/src/GrainsCPU.cpp:55-66) then runs unchanged.
//
// Differences from ComponentManagerCPU, all deliberate:
//  * errors throw std::runtime_error / std::invalid_argument with the
//    engine's status text instead of printing and continuing;
//  * the construction data that LinkedCell and TimeIntegrator keep protected
//    (grid corners, cell factor, time step) and the gravity vector are given
//    once, in Setup; calls check LinkedCell's cell count and the gravity they
//    are given against it and throw on a mismatch;
//  * detectCollisionAndComputeContactForcesParticles / ...Obstacles on their
//    own are not offered (the engine evaluates both in one pass); the
//    combined detectCollisionAndComputeContactForces is.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "Box.hh"
#include "ComponentManager.hh"
#include "HookeContactForceModel.hh"
#include "Rectangle.hh"
#include "Sphere.hh"
#include "Superquadric.hh"

#include "grains_b200.h"

template <typename T>
class ComponentManagerB200 : public ComponentManager<T>
{
public:
    /** Construction data that Grains::Construction reads from its XML input
        (Grains/Base/src/Grains.cpp:90-300) and keeps in GrainsParameters. */
    struct Setup
    {
        Vector3<T> origin;                 // GrainsParameters::m_origin
        Vector3<T> maxCoordinate;          // GrainsParameters::m_maxCoordinate
        T          cellSizeFactor = T(1);  // LinkedCell CellSizeFactor
        bool       padGrid = true;         // LinkedCell max corner raised by one cell
        T          dt = T(0);              // TimeIntegrator::m_dt
        Vector3<T> gravity;                // GrainsParameters::m_gravity
        int        precision  = GB_FP64_STRICT;
        int        contactLaw = GB_LAW_HOOKE;
        int        integrator = GB_FIRST_ORDER_EXPLICIT;
        T          ktOverKn   = T(0.8);    // tangential spring of GB_LAW_HOOKE_HISTORY
        int        device     = 0;
        int        flags      = 0;
        // material id of each particle / obstacle rigid body; empty: the
        // rigid body's own (RigidBody::getMaterial)
        std::vector<int32_t> particleMaterials;
        std::vector<int32_t> obstacleMaterials;
    };

    /** particleRB[nRigidBodies], obstacleRB[nObstacles] (one rigid body per
        obstacle), obstacleTr[nObstacles], CF[nMaterials*(nMaterials+1)/2]
        (HookeContactForceModel only), nParticles particles. */
    ComponentManagerB200(RigidBody<T, T> const* const*      particleRB,
                         uint                               nRigidBodies,
                         RigidBody<T, T> const* const*      obstacleRB,
                         uint                               nObstacles,
                         std::vector<Transform3<T>> const&  obstacleTr,
                         ContactForceModel<T> const* const* CF,
                         uint                               nMaterials,
                         uint                               nParticles,
                         Setup const&                       setup)
        : m_setup(setup)
        , m_nParticles(nParticles)
        , m_nObstacles(nObstacles)
    {
        gb_config cfg{};
        cfg.n_particles    = (int32_t)nParticles;
        cfg.n_rigid_bodies = (int32_t)nRigidBodies;
        cfg.n_obstacles    = (int32_t)nObstacles;
        cfg.n_materials    = (int32_t)nMaterials;
        for(int k = 0; k < 3; ++k)
        {
            cfg.origin[k]         = (double)setup.origin[k];
            cfg.max_coordinate[k] = (double)setup.maxCoordinate[k];
            cfg.gravity[k]        = (double)setup.gravity[k];
        }
        cfg.cell_size_factor = (double)setup.cellSizeFactor;
        cfg.pad_grid         = setup.padGrid ? 1 : 0;
        cfg.precision        = setup.precision;
        cfg.dt               = (double)setup.dt;
        cfg.contact_law      = setup.contactLaw;
        cfg.integrator       = setup.integrator;
        cfg.gjk_variant      = GB_GJK_JH;
        cfg.device           = setup.device;
        cfg.flags            = setup.flags;
        int st               = GB_OK;
        m_ctx                = gb_create(&cfg, &st);
        if(!m_ctx)
            fail(st, "gb_create");
        try
        {
            std::vector<gb_rigid_body_desc> rbs(nRigidBodies);
            for(uint i = 0; i < nRigidBodies; ++i)
            {
                rbs[i] = describe(*particleRB[i]);
                if(i < setup.particleMaterials.size())
                    rbs[i].material = setup.particleMaterials[i];
            }
            check(gb_set_rigid_bodies(m_ctx, rbs.data(), nullptr, 0), "gb_set_rigid_bodies");
            const uint nLaws = nMaterials * (nMaterials + 1) / 2;
            std::vector<gb_contact_model> laws(nLaws);
            for(uint i = 0; i < nLaws; ++i)
                laws[i] = law(*CF[i]);
            check(gb_set_contact_models(m_ctx, laws.data()), "gb_set_contact_models");
            m_obsRB.resize(nObstacles);
            for(uint i = 0; i < nObstacles; ++i)
            {
                m_obsRB[i] = describe(*obstacleRB[i]);
                if(i < setup.obstacleMaterials.size())
                    m_obsRB[i].material = setup.obstacleMaterials[i];
            }
            m_obsId.resize(nObstacles);
            for(uint i = 0; i < nObstacles; ++i)
                m_obsId[i] = i;
            setTransformObstacles(obstacleTr);
            m_rbId.assign(nParticles, 0u);
            m_particleId.resize(nParticles);
            for(uint i = 0; i < nParticles; ++i)
                m_particleId[i] = i;
        }
        catch(...)
        {
            gb_destroy(m_ctx);
            throw;
        }
    }

    ~ComponentManagerB200() override
    {
        if(m_ctx)
            gb_destroy(m_ctx);
    }

    ComponentManagerB200(ComponentManagerB200 const&)            = delete;
    ComponentManagerB200& operator=(ComponentManagerB200 const&) = delete;

    /** The engine context, for the rest of the C ABI (gb_step, stats, dumps). */
    gb_ctx* context() const { return m_ctx; }

    // ---- get methods (ComponentManager.hh:37-71) ----------------------------
    std::vector<uint> getRigidBodyId() const override { return m_rbId; }
    std::vector<uint> getRigidBodyIdObstacles() const override { return m_obsId; }

    std::vector<Transform3<T>> getTransform() const override
    {
        std::vector<double> buf(12 * (size_t)m_nParticles);
        check(gb_get_transforms(m_ctx, buf.data()), "gb_get_transforms");
        std::vector<Transform3<T>> out;
        out.reserve(m_nParticles);
        T t[12];
        for(uint i = 0; i < m_nParticles; ++i)
        {
            for(int k = 0; k < 12; ++k)
                t[k] = (T)buf[12 * (size_t)i + k];
            out.emplace_back(t);
        }
        return out;
    }

    std::vector<Transform3<T>> getTransformObstacles() const override { return m_obsTr; }

    std::vector<Kinematics<T>> getVelocity() const override
    {
        std::vector<double> buf(6 * (size_t)m_nParticles);
        check(gb_get_velocities(m_ctx, buf.data()), "gb_get_velocities");
        std::vector<Kinematics<T>> out;
        out.reserve(m_nParticles);
        for(uint i = 0; i < m_nParticles; ++i)
        {
            const double* v = buf.data() + 6 * (size_t)i;
            out.emplace_back(Vector3<T>(T(v[0]), T(v[1]), T(v[2])),
                             Vector3<T>(T(v[3]), T(v[4]), T(v[5])));
        }
        return out;
    }

    std::vector<Torce<T>> getTorce() const override
    {
        std::vector<double> buf(6 * (size_t)m_nParticles);
        check(gb_get_torces(m_ctx, buf.data()), "gb_get_torces");
        std::vector<Torce<T>> out;
        out.reserve(m_nParticles);
        for(uint i = 0; i < m_nParticles; ++i)
        {
            const double* f = buf.data() + 6 * (size_t)i; // force(3) torque(3)
            out.emplace_back(Vector3<T>(T(f[3]), T(f[4]), T(f[5])),
                             Vector3<T>(T(f[0]), T(f[1]), T(f[2])));
        }
        return out;
    }

    std::vector<uint> getParticleId() const override { return m_particleId; }
    uint              getNumberOfParticles() const override { return m_nParticles; }
    uint              getNumberOfObstacles() const override { return m_nObstacles; }

    uint getNumberOfCells() const override
    {
        gb_stats s{};
        check(gb_get_stats(m_ctx, &s), "gb_get_stats");
        return (uint)s.n_cells;
    }

    // ---- set methods (ComponentManager.hh:75-99) ----------------------------
    void setRigidBodyId(std::vector<uint> const& id) override
    {
        size_check(id.size(), m_nParticles, "setRigidBodyId");
        std::vector<uint32_t> ids(id.begin(), id.end());
        check(gb_set_rigid_body_ids(m_ctx, ids.data()), "gb_set_rigid_body_ids");
        m_rbId = id;
    }

    void setRigidBodyIdObstacles(std::vector<uint> const& id) override
    {
        size_check(id.size(), m_nObstacles, "setRigidBodyIdObstacles");
        for(uint k : id)
            if(k >= m_obsRB.size())
                throw std::invalid_argument("setRigidBodyIdObstacles: rigid body id out of range");
        m_obsId = id;
        upload_obstacles();
    }

    void setTransform(std::vector<Transform3<T>> const& t) override
    {
        size_check(t.size(), m_nParticles, "setTransform");
        std::vector<double> buf(12 * (size_t)m_nParticles);
        for(uint i = 0; i < m_nParticles; ++i)
            flatten(t[i], buf.data() + 12 * (size_t)i);
        check(gb_set_transforms(m_ctx, buf.data()), "gb_set_transforms");
    }

    void setTransformObstacles(std::vector<Transform3<T>> const& t) override
    {
        size_check(t.size(), m_nObstacles, "setTransformObstacles");
        m_obsTr = t;
        upload_obstacles();
    }

    void setVelocity(std::vector<Kinematics<T>> const& v) override
    {
        size_check(v.size(), m_nParticles, "setVelocity");
        std::vector<double> buf(6 * (size_t)m_nParticles);
        for(uint i = 0; i < m_nParticles; ++i)
        {
            const Vector3<T> a = v[i].getTranslationalComponent(), w = v[i].getAngularComponent();
            for(int k = 0; k < 3; ++k)
            {
                buf[6 * (size_t)i + k]     = (double)a[k];
                buf[6 * (size_t)i + 3 + k] = (double)w[k];
            }
        }
        check(gb_set_velocities(m_ctx, buf.data()), "gb_set_velocities");
    }

    void setTorce(std::vector<Torce<T>> const& t) override
    {
        size_check(t.size(), m_nParticles, "setTorce");
        std::vector<double> buf(6 * (size_t)m_nParticles);
        for(uint i = 0; i < m_nParticles; ++i)
        {
            const Vector3<T> f = t[i].getForce(), q = t[i].getTorque();
            for(int k = 0; k < 3; ++k)
            {
                buf[6 * (size_t)i + k]     = (double)f[k];
                buf[6 * (size_t)i + 3 + k] = (double)q[k];
            }
        }
        check(gb_set_torces(m_ctx, buf.data()), "gb_set_torces");
    }

    void setParticleId(std::vector<uint> const& id) override
    {
        size_check(id.size(), m_nParticles, "setParticleId");
        m_particleId = id;
    }

    // ---- the time-step calls (ComponentManager.hh:130-182) ------------------
    void updateLinks(LinkedCell<T> const* const* LC) override
    {
        check_cells(LC);
        check(gb_update_links(m_ctx), "gb_update_links");
    }

    void detectCollisionAndComputeContactForcesObstacles(RigidBody<T, T> const* const*,
                                                         RigidBody<T, T> const* const*,
                                                         ContactForceModel<T> const* const*) override
    {
        throw std::logic_error("ComponentManagerB200 evaluates particle and obstacle contacts in one "
                               "pass: call detectCollisionAndComputeContactForces");
    }

    void detectCollisionAndComputeContactForcesParticles(RigidBody<T, T> const* const*,
                                                         LinkedCell<T> const* const*,
                                                         ContactForceModel<T> const* const*,
                                                         int*) override
    {
        throw std::logic_error("ComponentManagerB200 evaluates particle and obstacle contacts in one "
                               "pass: call detectCollisionAndComputeContactForces");
    }

    void detectCollisionAndComputeContactForces(RigidBody<T, T> const* const*,
                                                RigidBody<T, T> const* const*,
                                                LinkedCell<T> const* const*        LC,
                                                ContactForceModel<T> const* const*,
                                                int* result) override
    {
        check_cells(LC);
        check(gb_detect_collision_and_compute_contact_forces(m_ctx, result),
              "gb_detect_collision_and_compute_contact_forces");
    }

    void addExternalForces(RigidBody<T, T> const* const*, const Vector3<T>& g) override
    {
        for(int k = 0; k < 3; ++k)
            if(g[k] != m_setup.gravity[k])
                throw std::invalid_argument("addExternalForces: gravity differs from Setup::gravity");
        check(gb_add_external_forces(m_ctx), "gb_add_external_forces");
    }

    void moveParticles(RigidBody<T, T> const* const*, TimeIntegrator<T> const* const*) override
    {
        check(gb_move_particles(m_ctx), "gb_move_particles");
    }

private:
    [[noreturn]] static void fail(int st, const char* what)
    {
        throw std::runtime_error(std::string(what) + ": " + gb_status_string(st));
    }

    static void check(int st, const char* what)
    {
        // GB_E_OUT_OF_DOMAIN reports particles outside the linked-cell grid;
        // the step still ran, as ComponentManagerCPU's does
        if(st != GB_OK && st != GB_E_OUT_OF_DOMAIN)
            fail(st, what);
    }

    static void size_check(size_t got, uint want, const char* what)
    {
        if(got != want)
            throw std::invalid_argument(std::string(what) + ": " + std::to_string(got)
                                        + " entries for " + std::to_string(want));
    }

    // RigidBody(convex, crust, material, density) as a descriptor; the density
    // is recovered as mass / volume (0 for massless obstacles)
    static gb_rigid_body_desc describe(RigidBody<T, T> const& rb)
    {
        gb_rigid_body_desc d{};
        Convex<T> const*   cv = rb.getConvex();
        d.convex.type         = (int32_t)cv->getConvexType();
        switch(cv->getConvexType())
        {
            case SPHERE:
                d.convex.p[0] = (double)static_cast<Sphere<T> const*>(cv)->getRadius();
                break;
            case BOX:
            {
                const Vector3<T> e = static_cast<Box<T> const*>(cv)->getExtent();
                for(int k = 0; k < 3; ++k)
                    d.convex.p[k] = (double)e[k];
                break;
            }
            case SUPERQUADRIC:
            {
                auto const*      sq = static_cast<Superquadric<T> const*>(cv);
                const Vector3<T> e = sq->getExtent(), n = sq->getExponent();
                for(int k = 0; k < 3; ++k)
                    d.convex.p[k] = (double)e[k];
                d.convex.p[3] = (double)n[0];
                d.convex.p[4] = (double)n[1];
                break;
            }
            case RECTANGLE:
            {
                const Vector3<T> e = static_cast<Rectangle<T> const*>(cv)->getExtent();
                d.convex.p[0]      = (double)e[0];
                d.convex.p[1]      = (double)e[1];
                break;
            }
            default:
                throw std::invalid_argument("ComponentManagerB200: convex type "
                                            + std::to_string((int)cv->getConvexType())
                                            + " is not supported");
        }
        d.crust_thickness = (double)rb.getCrustThickness();
        d.density  = rb.getVolume() > T(0) ? (double)rb.getMass() / (double)rb.getVolume() : 0.0;
        d.material = (int32_t)rb.getMaterial();
        return d;
    }

    gb_contact_model law(ContactForceModel<T> const& cf) const
    {
        if(cf.getContactForceModelType() != HOOKE)
            throw std::invalid_argument("ComponentManagerB200: only HookeContactForceModel");
        T kn, en, etat, muc, kr;
        static_cast<HookeContactForceModel<T> const&>(cf).getContactForceModelParameters(
            kn, en, etat, muc, kr);
        gb_contact_model m{};
        m.kn   = (double)kn;
        m.en   = (double)en;
        m.etat = (double)etat;
        m.muc  = (double)muc;
        m.kr   = (double)kr;
        m.kt   = (double)(m_setup.ktOverKn * kn);
        return m;
    }

    static void flatten(Transform3<T> const& t, double* out)
    {
        const Matrix3<T> b = t.getBasis();
        const Vector3<T> o = t.getOrigin();
        for(int r = 0; r < 3; ++r)
            for(int c = 0; c < 3; ++c)
                out[3 * r + c] = (double)b[r][c];
        for(int k = 0; k < 3; ++k)
            out[9 + k] = (double)o[k];
    }

    void upload_obstacles()
    {
        if(m_obsTr.size() != m_nObstacles || m_obsId.size() != m_nObstacles)
            return;
        std::vector<gb_rigid_body_desc> d(m_nObstacles);
        std::vector<double>             tr(12 * (size_t)m_nObstacles);
        for(uint i = 0; i < m_nObstacles; ++i)
        {
            d[i] = m_obsRB[m_obsId[i]];
            flatten(m_obsTr[i], tr.data() + 12 * (size_t)i);
        }
        check(gb_set_obstacles(m_ctx, d.data(), tr.data()), "gb_set_obstacles");
    }

    void check_cells(LinkedCell<T> const* const* LC) const
    {
        if(LC && *LC && (*LC)->getNumCells() != getNumberOfCells())
            throw std::invalid_argument(
                "ComponentManagerB200: the LinkedCell has " + std::to_string((*LC)->getNumCells())
                + " cells, the engine's grid " + std::to_string(getNumberOfCells())
                + " (Setup corners, cell factor or padGrid differ)");
    }

    gb_ctx*                         m_ctx = nullptr;
    Setup                           m_setup;
    uint                            m_nParticles, m_nObstacles;
    std::vector<uint>               m_rbId, m_obsId, m_particleId;
    std::vector<gb_rigid_body_desc> m_obsRB; // per obstacle rigid body
    std::vector<Transform3<T>>      m_obsTr;
};
