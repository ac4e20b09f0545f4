// grains_b200_grains.hh -- GrainsB200<T>, a Grains3D application
// (Grains/Base/include/Grains.hh:21-101) whose time loop runs on a B200
// through ComponentManagerB200<T>.
//
// Header-only, like grains_b200_component_manager.hh: compile it together
// with the Grains sources and the Xerces-free ReaderXML
// (grains3dgpu_b200/xml/ReaderXML.cpp) and link libgrains_b200.so.  It is
// driven exactly as main() drives GrainsCPU (Grains/Main/src/main.cpp):
//
//     ReaderXML::initialize();
//     DOMElement* root = ReaderXML::getRoot(file);
//     GrainsB200<double> grains(options);
//     grains.initialize(root);     // Grains<T>::initialize: Construction,
//     grains.simulate();           //   Forces, AdditionalFeatures
//     grains.finalize();
//
// Grains<T>::Construction reads the XML and builds the rigid bodies, the
// linked cell, the contact force models, the time integrator and a host
// ComponentManagerCPU (Grains.cpp:90-300).  simulate() inserts the particles
// as GrainsCPU::simulate does (GrainsCPU.cpp:41), hands the resulting state
// and every construction object to a ComponentManagerB200, which takes the
// host manager's place, and runs GrainsCPU's loop (GrainsCPU.cpp:46-70):
// detect and contact forces, gravity, move, post-processing writers.
//
// Two defects of the reference's XML construction can be corrected, each
// behind an option (fixMaterialIds on by default, since the uninitialised
// id it replaces is usually outside the contact-law table, which the engine
// rejects; fixInsertionWindow off by default, reproducing the reference):
//   fixMaterialIds      RigidBody(DOMNode*) (RigidBody.cpp:77-90) records a
//                       material the first time it is seen but does not set
//                       the rigid body's id to it, so the first rigid body
//                       of each material indexes the contact laws with an
//                       uninitialised value.  With the option, every particle
//                       and obstacle takes the id that GrainsParameters'
//                       material map holds for its Material attribute.
//   fixInsertionWindow  InsertionWindow(DOMNode*, seed)
//                       (InsertionWindow.cpp:35, :40, :55, :60) declares its
//                       corners as locals that shadow the members, so every
//                       Random insertion draws inside a window collapsed to
//                       the origin.  With the option, simulate() inserts by
//                       its own restatement of Insertion::fetchInsertionData
//                       (Insertion.cpp:187-264) and generateRandomPoint
//                       (InsertionWindow.cpp:92-123), with the corners kept
//                       and the same generator, seeds and draws.
#pragma once

#include <cmath>
#include <ctime>
#include <fstream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "Grains.hh"
#include "GrainsParameters.hh"
#include "ReaderXML.hh"
#include "VectorMath.hh"

#include "grains_b200_component_manager.hh"

template <typename T>
class GrainsB200 : public Grains<T>
{
public:
    struct Options
    {
        // on by default: the engine rejects a material id beyond the
        // contact-law table, which the uninitialised id usually is
        bool fixMaterialIds     = true;
        bool fixInsertionWindow = false;
        // run mode, contact law, device and flags of the engine; the grid,
        // time step and gravity come from the XML
        int  precision  = GB_FP64_STRICT;
        int  contactLaw = GB_LAW_HOOKE;
        int  device     = 0;
        int  flags      = 0;
        // LinkedCell as the reference builds it (floored cell counts) when
        // false; one more cell per axis when true
        bool padGrid = false;
    };

    explicit GrainsB200(Options const& o = Options())
        : m_opt(o)
    {
    }

    ~GrainsB200() override = default;

    void initialize(DOMElement* rootElement) override
    {
        m_root = rootElement;
        Grains<T>::initialize(rootElement);
    }

    /** Material ids of the particles and obstacles, in the order Construction
        creates them, from each Particle / Obstacle node's Material attribute
        and GrainsParameters' material map (fixMaterialIds). */
    static void materialIds(DOMElement* root, std::vector<int32_t>& particles,
                            std::vector<int32_t>& obstacles)
    {
        auto& map = GrainsParameters<T>::m_materialMap;
        particles.clear();
        obstacles.clear();
        DOMNodeList* allParticles = ReaderXML::getNodes(root, "Particle");
        for(XMLSize_t i = 0; i < allParticles->getLength(); ++i)
        {
            DOMNode*  n   = allParticles->item(i);
            const int num = ReaderXML::getNodeAttr_Int(n, "Number");
            const int id  = (int)map.at(ReaderXML::getNodeAttr_String(n, "Material"));
            for(int j = 0; j < num; ++j)
                particles.push_back(id);
        }
        DOMNodeList* allObstacles = ReaderXML::getNodes(root, "Obstacle");
        for(XMLSize_t i = 0; i < allObstacles->getLength(); ++i)
            obstacles.push_back(
                (int)map.at(ReaderXML::getNodeAttr_String(allObstacles->item(i), "Material")));
    }

    /** The initial transforms and velocities that insertion gives the
        particles, starting from `tr` (the transforms Construction read):
        the reference's Insertion through the host manager, or with
        fixInsertionWindow the restatement with the windows' corners kept. */
    void insert(std::vector<Transform3<T>>& tr, std::vector<Kinematics<T>>& kin)
    {
        ComponentManager<T>* host = Grains<T>::m_components;
        if(!m_opt.fixInsertionWindow)
        {
            host->insertParticles(Grains<T>::m_insertion);
            tr  = host->getTransform();
            kin = host->getVelocity();
            return;
        }
        tr = host->getTransform();
        kin.assign(tr.size(), Kinematics<T>());
        DOMNode* sim = ReaderXML::getNode(m_root, "Simulation");
        DOMNode* nIn = sim ? ReaderXML::getNode(sim, "ParticleInsertion") : nullptr;
        Source   pos(nIn, "InitialPosition"), ori(nIn, "InitialOrientation"),
            vel(nIn, "InitialVelocity"), ang(nIn, "InitialAngularVelocity");
        for(size_t i = 0; i < tr.size(); ++i)
        {
            // Insertion::fetchInsertionData and ComponentManagerCPU::insertParticles
            // (Insertion.cpp:240-262, ComponentManagerCPU.cpp:257-273)
            const Vector3<T> p = pos.next(), o = ori.next(), v = vel.next(), w = ang.next();
            Transform3<T>    t;
            t.setBasis(o[X], o[Y], o[Z]);
            t.setOrigin(p);
            tr[i].composeLeftByRotation(t);
            tr[i].setOrigin(t.getOrigin());
            kin[i] = Kinematics<T>(v, w);
        }
        host->setTransform(tr);
        host->setVelocity(kin);
    }

    void simulate() override
    {
        using GP = GrainsParameters<T>;
        std::vector<Transform3<T>> tr;
        std::vector<Kinematics<T>> kin;
        insert(tr, kin);
        ComponentManager<T>* host = Grains<T>::m_components;
        const uint           np = GP::m_numParticles, no = GP::m_numObstacles;

        typename ComponentManagerB200<T>::Setup s;
        s.origin        = GP::m_origin;
        s.maxCoordinate = GP::m_maxCoordinate;
        s.cellSizeFactor = cellSizeFactor();
        s.padGrid       = m_opt.padGrid;
        s.dt            = GP::m_dt;
        s.gravity       = GP::m_gravity;
        s.precision     = m_opt.precision;
        s.contactLaw    = m_opt.contactLaw;
        s.integrator    = GB_FIRST_ORDER_EXPLICIT;
        s.device        = m_opt.device;
        s.flags         = m_opt.flags;
        if(m_opt.fixMaterialIds)
            materialIds(m_root, s.particleMaterials, s.obstacleMaterials);
        auto* b200 = new ComponentManagerB200<T>(
            Grains<T>::m_particleRigidBodyList, np, Grains<T>::m_obstacleRigidBodyList, no,
            host->getTransformObstacles(), Grains<T>::m_contactForce,
            (uint)GP::m_materialMap.size(), np, s);
        b200->setRigidBodyId(host->getRigidBodyId());
        b200->setTransform(tr);
        b200->setVelocity(kin);
        delete host;
        Grains<T>::m_components = b200;

        // GrainsCPU::simulate's loop (GrainsCPU.cpp:46-70), counting the
        // ordered contacts of every step in `result` as it does
        std::vector<int> result(np, 0);
        for(GP::m_time = GP::m_tStart; GP::m_time <= GP::m_tEnd; GP::m_time += GP::m_dt)
        {
            b200->detectCollisionAndComputeContactForces(
                Grains<T>::m_particleRigidBodyList, Grains<T>::m_obstacleRigidBodyList,
                Grains<T>::m_linkedCell, Grains<T>::m_contactForce, result.data());
            b200->addExternalForces(Grains<T>::m_particleRigidBodyList, GP::m_gravity);
            b200->moveParticles(Grains<T>::m_particleRigidBodyList,
                                Grains<T>::m_timeIntegrator);
            // Grains::postProcess reads the next save time even when none is
            // left (Grains.cpp:60-73); it runs only while one is
            if(!GP::m_tSave.empty())
                Grains<T>::postProcess(b200);
        }
        m_contacts = 0;
        for(int r : result)
            m_contacts += r;
    }

    ComponentManager<T>* components() const { return Grains<T>::m_components; }
    long long            contactsCounted() const { return m_contacts; }

private:
    // One quantity of the ParticleInsertion node (InitialPosition, ...), read
    // as Insertion(DOMNode*) reads it (Insertion.cpp:8-97, :141-180), with
    // Random windows that keep their corners.
    struct Source
    {
        enum Kind
        {
            ZERO,
            CONSTANT,
            FILE,
            BOX,
            ANNULUS
        } kind = ZERO;
        Vector3<T>                        c, v1, v2;
        T                                 iRad = T(0), oRad = T(0);
        std::ifstream                     file;
        std::mt19937                      gen;
        std::uniform_real_distribution<T> dist;

        Source(DOMNode* parent, char const* name)
        {
            DOMNode* n = parent ? ReaderXML::getNode(parent, name) : nullptr;
            if(!n)
                return;
            const std::string type = ReaderXML::getNodeAttr_String(n, "Type");
            if(type == "Constant")
            {
                kind = CONSTANT;
                c    = Vector3<T>(T(ReaderXML::getNodeAttr_Double(n, "X")),
                                  T(ReaderXML::getNodeAttr_Double(n, "Y")),
                                  T(ReaderXML::getNodeAttr_Double(n, "Z")));
            }
            else if(type == "File")
            {
                kind = FILE;
                file.open(ReaderXML::getNodeAttr_String(n, "Name"));
                if(!file.good())
                    throw std::runtime_error("GrainsB200: insertion file "
                                             + ReaderXML::getNodeAttr_String(n, "Name")
                                             + " cannot be read");
            }
            else if(type == "Random")
            {
                // the seed as InsertionWindow(DOMNode*, seed) applies it: 0 by
                // default, the clock for "Random", and no seeding for
                // "UserDefined" (the reference passes the kind, not the value)
                const std::string seed = ReaderXML::getNodeAttr_String(n, "Seed");
                if(seed == "Random")
                    gen.seed((unsigned)time(NULL));
                else if(seed != "UserDefined")
                    gen.seed(0);
                DOMNode* nWindows = ReaderXML::getNode(n, "Windows");
                DOMNodeList* all  = nWindows ? ReaderXML::getNodes(nWindows) : nullptr;
                if(!all || all->getLength() == 0)
                    throw std::runtime_error(std::string("GrainsB200: ") + name
                                             + " is Random without a window");
                DOMNode*          w     = all->item(0); // the first window, as the reference
                const std::string wtype = ReaderXML::getNodeAttr_String(w, "Type");
                auto point = [&](char const* tag) {
                    DOMNode* p = ReaderXML::getNode(w, tag);
                    return Vector3<T>(T(ReaderXML::getNodeAttr_Double(p, "X")),
                                      T(ReaderXML::getNodeAttr_Double(p, "Y")),
                                      T(ReaderXML::getNodeAttr_Double(p, "Z")));
                };
                if(wtype == "Box")
                {
                    kind = BOX;
                    v1   = point("MinPoint");
                    v2   = point("MaxPoint");
                }
                else if(wtype == "Annulus")
                {
                    kind        = ANNULUS;
                    v1          = point("BottomPoint");
                    v2          = point("TopPoint");
                    DOMNode* nR = ReaderXML::getNode(w, "Radius");
                    iRad        = T(ReaderXML::getNodeAttr_Double(nR, "Inner"));
                    oRad        = T(ReaderXML::getNodeAttr_Double(nR, "Outter"));
                }
                else
                    throw std::runtime_error("GrainsB200: insertion window type " + wtype);
            }
            else if(type != "Zero")
                throw std::runtime_error("GrainsB200: insertion type " + type);
        }

        Vector3<T> next()
        {
            switch(kind)
            {
                case CONSTANT:
                    return c;
                case FILE:
                {
                    Vector3<T> out;
                    file >> out;
                    return out;
                }
                case BOX:
                    // InsertionWindow::generateRandomPoint's expression, so
                    // that the draws are taken in the same order
                    return Vector3<T>(v1[X] + dist(gen) * (v2[X] - v1[X]),
                                      v1[Y] + dist(gen) * (v2[Y] - v1[Y]),
                                      v1[Z] + dist(gen) * (v2[Z] - v1[Z]));
                case ANNULUS:
                {
                    T          theta = dist(gen) * TWO_PI<T>;
                    T          u     = dist(gen);
                    T          r = sqrt((T(1) - u) * iRad * iRad + u * oRad * oRad);
                    Vector3<T> h = v1 + dist(gen) * (v2 - v1);
                    return Vector3<T>(h + Vector3<T>(r * cos(theta), r * sin(theta), T(0)));
                }
                default:
                    return Vector3<T>();
            }
        }
    };

    T cellSizeFactor() const
    {
        DOMNode* root = ReaderXML::getNode(m_root, "Construction");
        DOMNode* nLC  = root ? ReaderXML::getNode(root, "LinkedCell") : nullptr;
        T        f    = T(1);
        if(nLC && ReaderXML::hasNodeAttr(nLC, "CellSizeFactor"))
            f = T(ReaderXML::getNodeAttr_Double(nLC, "CellSizeFactor"));
        return f < T(1) ? T(1) : f;
    }

    Options     m_opt;
    DOMElement* m_root     = nullptr;
    long long   m_contacts = 0;
};
