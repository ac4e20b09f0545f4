// gb_dem.cuh -- contact detection between two rigid bodies, the contact laws,
// and the time integrators, as device functions over a scalar policy S.
//
// Coordinates.  In the FP64 modes (S = double, dstrict) points are absolute
// world coordinates exactly as in the reference.  In the mixed mode (S = float)
// every point is relative to particle A's centre: the centres stay FP64 and
// only their difference enters FP32 arithmetic.
#pragma once

#include "gb_geom.cuh"

namespace gb
{

template <typename S>
struct Contact
{
    V3<S> pt;  // contact point: absolute (FP64 modes) or relative to A (mixed)
    V3<S> vec; // overlap vector, from B to A when in contact
    S     overlap;
};

template <typename S>
GB_D Contact<S> no_contact()
{
    Contact<S> c;
    c.pt      = zero3<S>();
    c.vec     = zero3<S>();
    c.overlap = S(0.0);
    return c;
}

// closestPointsRigidBodies for two particles (CollisionDetection.cpp:182-284)
// plus closestPointsSpheres (:26-48).  oA/oB are the frame origins in the
// working coordinates (xA, xB absolute; or 0, xB-xA relative); d = xB - xA.
// VAR selects the GJK (GB_GJK_JH, the reference's choice, or GB_GJK_SV /
// GB_GJK_NESTEROV).
// closestPointsSpheres (CollisionDetection.cpp:26-48); a sphere's radius is
// its circumscribed radius, p[0] (the table's rcirc may include the crust)
template <typename S>
GB_D Contact<S> closest_spheres(const Body<S>& A, const Body<S>& B, const V3<S>& oA,
                                const V3<S>& oB)
{
    V3<S>   vba     = oB - oA;
    const S overlap = norm(vba) - A.p[0] - B.p[0];
    vba             = vba / norm(vba);
    if(overlap < S(0.0))
    {
        Contact<S> c;
        c.pt      = oA + (A.p[0] + S(0.5) * overlap) * vba;
        c.vec     = overlap * vba;
        c.overlap = overlap;
        return c;
    }
    return no_contact<S>();
}

template <int VAR = GB_GJK_JH, typename S>
GB_D Contact<S> closest_points(const Body<S>& A, const Body<S>& B, const M3<S>& RA,
                               const M3<S>& RB, const V3<S>& oA, const V3<S>& oB,
                               const V3<S>& d, int* gjk_iters)
{
    if(A.type == GB_SPHERE && B.type == GB_SPHERE)
        return closest_spheres(A, B, oA, oB);
    const S overlap = norm(d) - (A.rcirc + B.rcirc);
    if(!(overlap < S(0.0)))
        return no_contact<S>();
    if(!obb_overlap(A.bb, B.bb, RA, RB, d))
        return no_contact<S>();
    // b2a = Transform3(a2w, b2w) (Transform3.cpp:34-39, :313-318)
    Tr<S> b2a;
    const M3<S> RAt = transpose(RA);
    b2a.R           = mul(RAt, RB);
    b2a.o           = mul(RAt, d);
    GjkResult<S> g  = gjk<VAR>(A, B, b2a);
    *gjk_iters += g.iters;
    S distance = g.dist - (A.crust + B.crust);
    if(distance > S(0.0))
        return no_contact<S>();
    const V3<S> ptA = mul(RA, g.pa) + oA;
    const V3<S> ptB = mul(RB, g.pb) + oB;
    Contact<S>  c;
    c.pt       = (ptA + ptB) / S(2.0);
    V3<S> vec  = ptA - ptB;
    vec        = vec / norm(vec);
    vec        = round3(vec, k_eps<S>());
    c.vec      = (-distance) * vec;
    c.overlap  = distance;
    return c;
}

// closestPointsRectangle (CollisionDetection.cpp:53-90), the obstacle second.
// rpt is the rectangle centre and rn its frame's z axis, in working coordinates.
template <typename S>
GB_D Contact<S> closest_rectangle(const Body<S>& A, const M3<S>& RA, const V3<S>& oA,
                                  const V3<S>& rpt, V3<S> rn)
{
    rn               = s_copysign(S(1.0), dot(rn, oA - rpt)) * rn;
    const V3<S> pA   = mul(RA, support(A, mul_t(RA, -rn))) + oA;
    if(dot(rn, pA - rpt) < S(0.0))
    {
        const V3<S> pB = dot(rpt - pA, rn) * rn + pA;
        Contact<S>  c;
        c.pt      = S(0.5) * (pA + pB);
        c.vec     = pB - pA;
        c.overlap = -norm(c.vec);
        return c;
    }
    return no_contact<S>();
}

// NEW (no reference shape): the inner wall of a drum of radius R about the
// axis `ax` through oO.  The wall point nearest A's centre, w = oO + t + R e
// (t the axial part of oA - oO, e the unit radial direction), and the inward
// normal -e give the tangent plane that closest_rectangle meets.  A centre on
// the axis has no nearest point: no contact.
template <typename S>
GB_D Contact<S> closest_drum(const Body<S>& A, const M3<S>& RA, const V3<S>& oA, const V3<S>& oO,
                             const V3<S>& ax, S R)
{
    const V3<S> d  = oA - oO;
    const V3<S> t  = dot(ax, d) * ax;
    const V3<S> r  = d - t;
    const S     nr = norm(r);
    if(!(nr > S(1e-12) * R))
        return no_contact<S>();
    const V3<S> e = (S(1.0) / nr) * r;
    V3<S>       w = oO + t;
    w             = w + R * e;
    return closest_rectangle(A, RA, oA, w, -e);
}

// ---------------------------------------------------------------------------
// Contact laws.  Output: force on A, its torque about A's centre, and the
// rolling moment (kr != 0).
template <typename S>
struct Law
{
    S kn, muen, etat, muc, kr, kt;
};

template <typename S>
struct Force
{
    V3<S> f, t, m;
};

// HookeContactForceModel::performForcesCalculus + computeForces
// (HookeContactForceModel.cpp:91-186).  rel_vel uses the reference's lever
// arm (the contact point itself, Kinematics.cpp:87-90 as called at
// ComponentManagerCPU.cpp:404-407); `arm` = contact point - A's centre.
template <typename S>
GB_D Force<S> hooke(const Law<S>& L, const Contact<S>& ci, const V3<S>& rel_vel,
                    const V3<S>& rel_ang_vel, S m1, S m2, const V3<S>& arm)
{
    V3<S>   pen   = ci.vec;
    V3<S>   delFN = L.kn * pen;
    pen           = pen / norm(pen);
    pen           = round3(pen, k_eps<S>());
    const V3<S> v_n     = dot(rel_vel, pen) * pen;
    const V3<S> v_t     = rel_vel - v_n;
    const S     normv_t = norm(v_t);
    V3<S>       tangent = zero3<S>();
    if(normv_t > k_eps<S>())
        tangent = v_t / normv_t;
    S avmass = m1 * m2 / (m1 + m2);
    S omega0 = s_sqrt(L.kn / avmass);
    if(avmass == S(0.0))
    {
        avmass = m2 == S(0.0) ? S(0.5) * m1 : S(0.5) * m2;
        omega0 = S(2.0) * s_sqrt(L.kn / avmass);
    }
    const S muen = -omega0 * L.muen;
    delFN        = delFN + (-S(2.0) * muen * avmass) * v_n;
    const S normFN = norm(delFN);
    V3<S>   delFT  = (-L.etat * S(2.0) * avmass) * v_t;
    const S fn     = L.muc * normFN;
    const S ft     = norm(delFT);
    if(fn < ft)
        delFT = (-fn) * tangent;
    Force<S> out;
    out.m = zero3<S>();
    if(L.kr != S(0.0))
    {
        const V3<S> wn     = dot(rel_ang_vel, pen) * pen;
        const V3<S> wt     = rel_ang_vel - wn;
        const S     normwt = norm(wt);
        out.m              = (-L.kr * normFN * S(0.001)) * wn;
        if(normwt > k_eps<S>())
            out.m = out.m - (L.kr * normFN) * wt;
    }
    out.f = delFN + delFT;
    out.t = cross(arm, out.f);
    return out;
}

// NEW: spring-dashpot normal force (the Hooke normal part) plus a tangential
// spring kt with per-pair history xi (world frame) capped by Coulomb
// friction.  xi is projected on the current tangent plane, advanced by
// v_t dt, and rescaled to the Coulomb limit while sliding.  rel_vel uses each
// body's own lever arm; m2 == 0 (an obstacle) gives m* = m1.
template <typename S>
GB_D Force<S> hooke_history(const Law<S>& L, const Contact<S>& ci, const V3<S>& rel_vel,
                            S m1, S m2, S dt, const V3<S>& xi_prev, V3<S>& xi_new,
                            const V3<S>& arm)
{
    const V3<S> n     = ci.vec / norm(ci.vec);
    const S     mstar = m2 == S(0.0) ? m1 : m1 * m2 / (m1 + m2);
    const S     gn    = -S(2.0) * L.muen * s_sqrt(L.kn * mstar);
    const S     vn    = dot(rel_vel, n);
    const V3<S> v_t   = rel_vel - vn * n;
    const V3<S> fn    = L.kn * ci.vec + (-gn * vn) * n;
    const S     fnorm = norm(fn);
    V3<S>       xi    = xi_prev - dot(xi_prev, n) * n;
    xi                = xi + dt * v_t;
    const S gt        = S(2.0) * L.etat * mstar;
    V3<S>   ft        = (-L.kt) * xi - gt * v_t;
    const S ftn       = norm(ft);
    const S cap       = L.muc * fnorm;
    if(ftn > cap)
    {
        ft = (cap / ftn) * ft;
        xi = L.kt > S(0.0) ? (S(-1.0) / L.kt) * (ft + gt * v_t) : zero3<S>();
    }
    xi_new = xi;
    Force<S> out;
    out.f = fn + ft;
    out.t = cross(arm, out.f);
    out.m = zero3<S>();
    return out;
}

// ---------------------------------------------------------------------------
// Quaternions (w, v) and the rigid-body equations of motion.
template <typename S>
struct Quat
{
    S     w;
    V3<S> v;
};

// operator*(Vector3, Quaternion) = [0, v] x q (QuaternionMath.hh:130-137)
template <typename S>
GB_D Quat<S> vec_times_quat(const V3<S>& v, const Quat<S>& q)
{
    Quat<S> r;
    r.w = dot(-v, q.v);
    r.v = cross(v, q.v) + q.w * v;
    return r;
}
// Quaternion::multToVector3 (Quaternion.cpp:252-258)
template <typename S>
GB_D V3<S> mult_to_vec(const Quat<S>& q, const Quat<S>& r)
{
    return (cross(q.v, r.v) + q.w * r.v) + r.w * q.v;
}
// q1 x q2 (QuaternionMath.hh:98-109)
template <typename S>
GB_D Quat<S> qmul(const Quat<S>& a, const Quat<S>& b)
{
    Quat<S> r;
    r.w = a.w * b.w - dot(a.v, b.v);
    r.v = (cross(a.v, b.v) + a.w * b.v) + b.w * a.v;
    return r;
}

// RigidBody::computeMomentum (Grains/Geometry/src/RigidBody.cpp:267-307):
// angular acceleration in world axes from the Euler equations in body axes.
template <typename S>
GB_D V3<S> angular_acceleration(const S I[6], const S I1[6], const V3<S>& omega,
                                const V3<S>& torque, const Quat<S>& q)
{
    Quat<S> qc;
    qc.w          = q.w;
    qc.v          = -q.v;
    const V3<S> wb = mult_to_vec(qc, vec_times_quat(omega, q));
    V3<S>       am = mult_to_vec(qc, vec_times_quat(torque, q));
    V3<S>       t  = mk<S>(I[0] * wb.x + I[1] * wb.y + I[2] * wb.z,
                    I[1] * wb.x + I[3] * wb.y + I[4] * wb.z,
                    I[2] * wb.x + I[4] * wb.y + I[5] * wb.z);
    am = am + cross(t, wb);
    t  = mk<S>(I1[0] * am.x + I1[1] * am.y + I1[2] * am.z,
              I1[1] * am.x + I1[3] * am.y + I1[4] * am.z,
              I1[2] * am.x + I1[4] * am.y + I1[5] * am.z);
    return mult_to_vec(q, vec_times_quat(t, qc));
}

// Quaternion::setQuaternion(Matrix3) (Grains/Geometry/src/Quaternion.cpp:125-169)
template <typename S>
GB_D Quat<S> quat_from_basis(const M3<S>& R)
{
    const S* b = R.m;
    enum
    {
        XX,
        XY,
        XZ,
        YX,
        YY,
        YZ,
        ZX,
        ZY,
        ZZ
    };
    const S one = S(1.0), half = S(0.5);
    Quat<S> q;
    if(b[YY] > -b[ZZ] && b[XX] > -b[YY] && b[XX] > -b[ZZ])
    {
        const S den = s_pow(one + b[XX] + b[YY] + b[ZZ], half);
        q.w         = half * den;
        q.v         = mk<S>(half * (b[ZY] - b[YZ]) / den, half * (b[XZ] - b[ZX]) / den,
                    half * (b[YX] - b[XY]) / den);
    }
    else if(b[YY] < -b[ZZ] && b[XX] > b[YY] && b[XX] > b[ZZ])
    {
        const S den = s_pow(one + b[XX] - b[YY] - b[ZZ], half);
        q.w         = half * (b[ZY] - b[YZ]) / den;
        q.v         = mk<S>(half * den, half * (b[XY] + b[YX]) / den, half * (b[ZX] + b[XZ]) / den);
    }
    else if(b[YY] > b[ZZ] && b[XX] < b[YY] && b[XX] < -b[ZZ])
    {
        const S den = s_pow(one - b[XX] + b[YY] - b[ZZ], half);
        q.w         = half * (b[XZ] - b[ZX]) / den;
        q.v         = mk<S>(half * (b[XY] + b[YX]) / den, half * den, half * (b[YZ] + b[ZY]) / den);
    }
    else if(b[YY] < b[ZZ] && b[XX] < -b[YY] && b[XX] < b[ZZ])
    {
        const S den = s_pow(one - b[XX] - b[YY] + b[ZZ], half);
        q.w         = half * (b[YX] - b[XY]) / den;
        q.v         = mk<S>(half * (b[ZX] + b[XZ]) / den, half * (b[YZ] + b[ZY]) / den, half * den);
    }
    else
    {
        // a case the reference leaves undefined; identity keeps the step finite
        q.w = one;
        q.v = zero3<S>();
    }
    return q;
}

// Transform3::composeLeftByRotation(Quaternion) (Transform3.cpp:229-246):
// basis <- M_rot(q) basis, column by column.
template <typename S>
GB_D void compose_left_by_rotation(M3<S>& M, const Quat<S>& q)
{
    const S qx = q.v.x, qy = q.v.y, qz = q.v.z, qw = q.w;
    S*      m  = M.m;
#pragma unroll
    for(int i = 0; i < 3; ++i)
    {
        const S px = qy * m[6 + i] - qz * m[3 + i] + qw * m[i];
        const S py = qz * m[i] - qx * m[6 + i] + qw * m[3 + i];
        const S pz = qx * m[3 + i] - qy * m[i] + qw * m[6 + i];
        const S pw = -qx * m[i] - qy * m[3 + i] - qz * m[6 + i];
        m[i]       = qy * pz - qz * py - pw * qx + qw * px;
        m[3 + i]   = qz * px - qx * pz - pw * qy + qw * py;
        m[6 + i]   = qx * py - qy * px - pw * qz + qw * pz;
    }
}

// TimeIntegrator::computeQuaternionChange (TimeIntegrator.cpp:28-44)
template <typename S>
GB_D Quat<S> quaternion_change(const V3<S>& w, S dt)
{
    const S n = norm(w);
    Quat<S> r;
    if(n > k_higheps<S>())
    {
        const S h = n * dt / S(2.0);
        S       c = S(1.0), s = S(0.0);
        bool    small = false;
        if constexpr(std::is_same<S, float>::value)
            if(h < 0.05f)
            {
                // FP32: the rotation of a step is small; Taylor to x^5 and
                // x^4 (the next terms are below 2e-11 of the leading one)
                const float h2 = h * h;
                s              = h * (1.0f - h2 * (1.0f / 6.0f) * (1.0f - h2 * 0.05f));
                c              = 1.0f - h2 * 0.5f * (1.0f - h2 * (1.0f / 12.0f));
                small          = true;
            }
        if(!small)
        {
            c = s_cos(h);
            s = s_sin(h);
        }
        r.v       = (s / n) * w;
        r.w       = c;
    }
    else
    {
        r.v = zero3<S>();
        r.w = S(1.0);
    }
    return r;
}

} // namespace gb
