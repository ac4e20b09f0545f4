// adapter_drive.cpp -- drop-in check of ComponentManagerB200
// (include/grains_b200_component_manager.hh) against the reference's own
// ComponentManagerCPU.
//
// TEST INFRASTRUCTURE: built by oracle/Makefile into oracle/_ref/ from the
// reference sources where they lie; run by tests/test_gpu_dropin.py.  Both
// managers sit behind one ComponentManager<double>* and are driven with the
// reference's RigidBody, LinkedCell, HookeContactForceModel and
// FirstOrderExplicit objects in GrainsCPU::simulate's call order
// (Grains/Base/src/GrainsCPU.cpp:55-66): detect -> gravity -> move.
//
// Scene: 392 superquadrics (a=b=c=1 mm, n1=n2=4, crust 50 um) on a 2.05 mm
// jittered lattice with random orientations, in a closed 16x16x20 mm box of
// six Rectangle walls, dt = 2e-6 s.
//
// Usage: adapter_drive [steps]   (default 40).  Prints one JSON line and
// exits 0 when the contact counts agree and the transforms differ by less
// than 1e-12 and the velocities by at most 1e-7 of the largest; 1 on a
// mismatch; 2 when the engine cannot run (no GPU).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <random>
#include <vector>

#include "ComponentManagerCPU.hh"
#include "FirstOrderExplicit.hh"
#include "LinkedCell.hh"
#include "grains_b200_component_manager.hh"

using T = double;

namespace
{
// updateLinks clears m_cell[0..m_nCells] inclusive (ComponentManagerCPU.cpp:
// 281-282), one past the end; spare capacity keeps that write in bounds.
class CpuManager : public ComponentManagerCPU<T>
{
public:
    CpuManager(uint np, uint no, uint nc)
        : ComponentManagerCPU<T>(np, no, nc)
    {
        this->m_cell.reserve(this->m_cell.size() + 4);
    }
};

Transform3<T> frame(const double b[9], double x, double y, double z)
{
    double buf[12];
    for(int k = 0; k < 9; ++k)
        buf[k] = b[k];
    buf[9]  = x;
    buf[10] = y;
    buf[11] = z;
    return Transform3<T>(buf);
}

void rotation(std::mt19937_64& rng, double m[9])
{
    std::normal_distribution<double> g;
    double q[4], s = 0;
    for(double& v : q)
        s += (v = g(rng)) * v;
    s = std::sqrt(s);
    const double w = q[0] / s, x = q[1] / s, y = q[2] / s, z = q[3] / s;
    const double r[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),
                         2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                         2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y)};
    for(int k = 0; k < 9; ++k)
        m[k] = r[k];
}
} // namespace

int main(int argc, char** argv)
{
    const int    steps = argc > 1 ? std::atoi(argv[1]) : 40;
    const double L[3]  = {0.016, 0.016, 0.020};
    const double pitch = 2.05e-3, margin = 1.3e-3, dt = 2e-6;
    const int    nx = 7, ny = 7, nz = 8, n = nx * ny * nz;
    const int    nmat = 2; // 0: particles, 1: walls

    RigidBody<T, T>* prb[1] = {
        new RigidBody<T, T>(new Superquadric<T>(1e-3, 1e-3, 1e-3, 4.0, 4.0), 5e-5, 0, 2500.0)};
    // six Rectangle walls (full side lengths), local z = inward normal
    const double frames[6][9] = {{0, 0, 1, 0, 1, 0, -1, 0, 0},  {0, 0, -1, 0, 1, 0, 1, 0, 0},
                                 {1, 0, 0, 0, 0, 1, 0, -1, 0},  {1, 0, 0, 0, 0, -1, 0, 1, 0},
                                 {1, 0, 0, 0, 1, 0, 0, 0, 1},   {1, 0, 0, 0, -1, 0, 0, 0, -1}};
    const double sides[6][2]   = {{L[2], L[1]}, {L[2], L[1]}, {L[0], L[2]},
                                  {L[0], L[2]}, {L[0], L[1]}, {L[0], L[1]}};
    const double centres[6][3] = {{0, L[1] / 2, L[2] / 2},    {L[0], L[1] / 2, L[2] / 2},
                                  {L[0] / 2, 0, L[2] / 2},    {L[0] / 2, L[1], L[2] / 2},
                                  {L[0] / 2, L[1] / 2, 0},    {L[0] / 2, L[1] / 2, L[2]}};
    RigidBody<T, T>*           orb[6];
    std::vector<Transform3<T>> otr;
    std::vector<uint>          oid;
    for(int i = 0; i < 6; ++i)
    {
        orb[i] = new RigidBody<T, T>(new Rectangle<T>(sides[i][0], sides[i][1]), 0.0, 1, 0.0);
        otr.push_back(frame(frames[i], centres[i][0], centres[i][1], centres[i][2]));
        oid.push_back(i);
    }
    ContactForceModel<T>* cf[3];
    for(int i = 0; i < 3; ++i)
        cf[i] = new HookeContactForceModel<T>(1e4, 0.7, 0.0, 0.5, 0.0);
    const Vector3<T> g(0.0, 0.0, -9.81);

    // LinkedCell as Grains builds it (cell = 2 x the largest circumscribed
    // radius), max corner raised by one cell so that the floored cell count
    // covers the box
    const T    cell = T(2) * prb[0]->getCircumscribedRadius();
    LinkedCell<T>  lc(Vector3<T>(0, 0, 0), Vector3<T>(L[0] + cell, L[1] + cell, L[2] + cell), cell);
    LinkedCell<T>* lcp = &lc;
    TimeIntegrator<T>* ti = new FirstOrderExplicit<T>(dt);

    std::mt19937_64                        rng(12345);
    std::uniform_real_distribution<double> jit(-0.15e-3, 0.15e-3);
    std::vector<Transform3<T>>             tr;
    for(int k = 0; k < n; ++k)
    {
        double b[9];
        rotation(rng, b);
        const int ix = k % nx, iy = (k / nx) % ny, iz = k / (nx * ny);
        tr.push_back(frame(b, margin + ix * pitch + jit(rng), margin + iy * pitch + jit(rng),
                           margin + iz * pitch + jit(rng)));
    }
    std::vector<Kinematics<T>> kin(n, Kinematics<T>(Vector3<T>(0, 0, 0), Vector3<T>(0, 0, 0)));

    ComponentManager<T>* cm[2] = {nullptr, nullptr};
    cm[0]                      = new CpuManager(n, 6, lc.getNumCells());
    try
    {
        ComponentManagerB200<T>::Setup s;
        s.origin        = Vector3<T>(0, 0, 0);
        s.maxCoordinate = Vector3<T>(L[0], L[1], L[2]);
        s.dt            = dt;
        s.gravity       = g;
        s.precision     = GB_FP64_STRICT;
        cm[1] = new ComponentManagerB200<T>(prb, 1, orb, 6, otr, cf, nmat, n, s);
    }
    catch(const std::exception& e)
    {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
    long contacts[2] = {0, 0};
    try
    {
        for(ComponentManager<T>* m : cm)
        {
            m->setRigidBodyId(std::vector<uint>(n, 0u));
            m->setTransform(tr);
            m->setVelocity(kin);
            m->setRigidBodyIdObstacles(oid);
            m->setTransformObstacles(otr);
        }
        for(int it = 0; it < steps; ++it)
            for(int k = 0; k < 2; ++k)
            {
                std::vector<int> result(n, 0);
                cm[k]->detectCollisionAndComputeContactForces(prb, orb, &lcp, cf, result.data());
                cm[k]->addExternalForces(prb, g);
                cm[k]->moveParticles(prb, &ti);
                for(int r : result)
                    contacts[k] += r;
            }
    }
    catch(const std::exception& e)
    {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
    const std::vector<Transform3<T>> ta = cm[0]->getTransform(), tb = cm[1]->getTransform();
    const std::vector<Kinematics<T>> va = cm[0]->getVelocity(), vb = cm[1]->getVelocity();
    double dx = 0, dv = 0, vmax = 0;
    for(int i = 0; i < n; ++i)
    {
        const Matrix3<T> ba = ta[i].getBasis(), bb = tb[i].getBasis();
        for(int r = 0; r < 3; ++r)
        {
            dx = std::fmax(dx, std::fabs(ta[i].getOrigin()[r] - tb[i].getOrigin()[r]));
            for(int c = 0; c < 3; ++c)
                dx = std::fmax(dx, std::fabs(ba[r][c] - bb[r][c]));
            const T a1 = va[i].getTranslationalComponent()[r], b1 = vb[i].getTranslationalComponent()[r];
            const T a2 = va[i].getAngularComponent()[r], b2 = vb[i].getAngularComponent()[r];
            dv   = std::fmax(dv, std::fmax(std::fabs(a1 - b1), std::fabs(a2 - b2)));
            vmax = std::fmax(vmax, std::fmax(std::fabs(a1), std::fabs(a2)));
        }
    }
    const bool ok = contacts[0] == contacts[1] && contacts[0] > 0 && dx < 1e-12 && dv <= 1e-7 * vmax;
    std::printf("{\"steps\": %d, \"particles\": %d, \"contacts_cpu\": %ld, \"contacts_gpu\": %ld, "
                "\"max_transform_diff\": %.3e, \"max_velocity_diff\": %.3e, \"max_velocity\": %.3e, "
                "\"ok\": %s}\n",
                steps, n, contacts[0], contacts[1], dx, dv, vmax, ok ? "true" : "false");
    delete cm[1];
    delete cm[0];
    return ok ? 0 : 1;
}
