// gb_host_geometry.cpp -- rigid-body set-up on the host: volume, mass,
// inertia, bounding box and circumscribed radius of each convex, computed as
// RigidBody::RigidBody(convex, ct, material, density) does
// (Grains/Geometry/src/RigidBody.cpp:19-59), and the convex hull used for the
// mass properties of polyhedra.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/grains_b200.h"

namespace
{

constexpr double kPi = 3.1415926535897932385; // Basic.hh:103-104

double beta_fn(double x, double y)
{
    return std::beta(x, y); // grainsBeta on the host (MiscMath.hh:82-90)
}

// ---- convex hull of <= GB_MAX_POLY_VERTICES points (incremental) ----------------
struct Face
{
    int    v[3];
    double n[3], d; // outward unit normal, plane offset
    bool   alive;
};

void face_plane(const double* p, Face& f)
{
    const double* a = p + 3 * f.v[0];
    const double* b = p + 3 * f.v[1];
    const double* c = p + 3 * f.v[2];
    const double  e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double  e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double        n[3]  = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                   e1[0] * e2[1] - e1[1] * e2[0]};
    const double  l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for(int k = 0; k < 3; ++k)
        f.n[k] = l > 0 ? n[k] / l : 0.0;
    f.d = f.n[0] * a[0] + f.n[1] * a[1] + f.n[2] * a[2];
}

double dist_to(const Face& f, const double* q)
{
    return f.n[0] * q[0] + f.n[1] * q[1] + f.n[2] * q[2] - f.d;
}

// Returns outward-oriented triangles of the hull, or an empty list when the
// points are (nearly) coplanar.
std::vector<Face> convex_hull(const double* p, int n)
{
    std::vector<Face> faces;
    if(n < 4)
        return faces;
    double scale = 0;
    for(int i = 0; i < 3 * n; ++i)
        scale = std::max(scale, std::fabs(p[i]));
    const double eps = 1e-10 * std::max(scale, 1e-300);
    // initial tetrahedron: two far points, the point farthest from their
    // line, the point farthest from their plane
    int i0 = 0, i1 = -1, i2 = -1, i3 = -1;
    double best = -1;
    for(int i = 1; i < n; ++i)
    {
        double d2 = 0;
        for(int k = 0; k < 3; ++k)
            d2 += (p[3 * i + k] - p[k]) * (p[3 * i + k] - p[k]);
        if(d2 > best)
            best = d2, i1 = i;
    }
    best = -1;
    for(int i = 0; i < n; ++i)
    {
        const double* a = p + 3 * i0;
        const double* b = p + 3 * i1;
        const double* c = p + 3 * i;
        const double  e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const double  e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        const double  x = e1[1] * e2[2] - e1[2] * e2[1], y = e1[2] * e2[0] - e1[0] * e2[2],
                     z = e1[0] * e2[1] - e1[1] * e2[0];
        const double area = x * x + y * y + z * z;
        if(area > best)
            best = area, i2 = i;
    }
    Face base{{i0, i1, i2}, {0, 0, 0}, 0, true};
    face_plane(p, base);
    best = -1;
    for(int i = 0; i < n; ++i)
    {
        const double dd = std::fabs(dist_to(base, p + 3 * i));
        if(dd > best)
            best = dd, i3 = i;
    }
    if(best <= eps || i1 < 0 || i2 < 0)
        return faces;
    // orient the four faces outward
    const int tet[4][3] = {{i0, i1, i2}, {i0, i3, i1}, {i1, i3, i2}, {i2, i3, i0}};
    double    ctr[3]    = {0, 0, 0};
    for(int k = 0; k < 3; ++k)
        ctr[k] = 0.25 * (p[3 * i0 + k] + p[3 * i1 + k] + p[3 * i2 + k] + p[3 * i3 + k]);
    for(auto& t : tet)
    {
        Face f{{t[0], t[1], t[2]}, {0, 0, 0}, 0, true};
        face_plane(p, f);
        if(dist_to(f, ctr) > 0)
        {
            std::swap(f.v[1], f.v[2]);
            face_plane(p, f);
        }
        faces.push_back(f);
    }
    std::vector<char> used(n, 0);
    used[i0] = used[i1] = used[i2] = used[i3] = 1;
    for(int q = 0; q < n; ++q)
    {
        if(used[q])
            continue;
        const double* pt = p + 3 * q;
        std::vector<int> vis;
        for(int f = 0; f < (int)faces.size(); ++f)
            if(faces[f].alive && dist_to(faces[f], pt) > eps)
                vis.push_back(f);
        if(vis.empty())
            continue; // inside (or on) the current hull
        // horizon: directed edges of visible faces whose twin is not visible
        std::vector<std::pair<int, int>> edges;
        for(int f : vis)
            for(int e = 0; e < 3; ++e)
                edges.push_back({faces[f].v[e], faces[f].v[(e + 1) % 3]});
        std::vector<std::pair<int, int>> horizon;
        for(auto& e : edges)
        {
            bool twin = false;
            for(auto& o : edges)
                if(o.first == e.second && o.second == e.first)
                {
                    twin = true;
                    break;
                }
            if(!twin)
                horizon.push_back(e);
        }
        for(int f : vis)
            faces[f].alive = false;
        for(auto& e : horizon)
        {
            Face nf{{e.first, e.second, q}, {0, 0, 0}, 0, true};
            face_plane(p, nf);
            faces.push_back(nf);
        }
    }
    std::vector<Face> out;
    for(auto& f : faces)
        if(f.alive)
            out.push_back(f);
    return out;
}

// Volume, first and second moments of the solid bounded by outward
// triangles (divergence theorem over tetrahedra from the origin).
void polyhedron_moments(const double* p, const std::vector<Face>& faces, double& vol,
                        double c[3], double sq[3], double pr[3])
{
    vol = 0;
    for(int k = 0; k < 3; ++k)
        c[k] = sq[k] = pr[k] = 0;
    for(const Face& f : faces)
    {
        const double* a = p + 3 * f.v[0];
        const double* b = p + 3 * f.v[1];
        const double* d = p + 3 * f.v[2];
        const double  det = a[0] * (b[1] * d[2] - b[2] * d[1]) - a[1] * (b[0] * d[2] - b[2] * d[0])
                           + a[2] * (b[0] * d[1] - b[1] * d[0]);
        vol += det / 6.0;
        for(int k = 0; k < 3; ++k)
        {
            c[k] += det / 24.0 * (a[k] + b[k] + d[k]);
            sq[k] += det / 60.0
                     * (a[k] * a[k] + b[k] * b[k] + d[k] * d[k] + a[k] * b[k] + a[k] * d[k]
                        + b[k] * d[k]);
        }
        const int ij[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for(int t = 0; t < 3; ++t)
        {
            const int i = ij[t][0], j = ij[t][1];
            pr[t] += det / 120.0
                     * (2.0 * (a[i] * a[j] + b[i] * b[j] + d[i] * d[j]) + a[i] * b[j] + a[j] * b[i]
                        + a[i] * d[j] + a[j] * d[i] + b[i] * d[j] + b[j] * d[i]);
        }
    }
}

int inv_sym3(const double I[6], double o[6])
{
    const double c00 = I[3] * I[5] - I[4] * I[4];
    const double c01 = I[2] * I[4] - I[1] * I[5];
    const double c02 = I[1] * I[4] - I[2] * I[3];
    const double det = I[0] * c00 + I[1] * c01 + I[2] * c02;
    if(!(std::fabs(det) > 0))
        return -1;
    o[0] = c00 / det;
    o[1] = c01 / det;
    o[2] = c02 / det;
    o[3] = (I[0] * I[5] - I[2] * I[2]) / det;
    o[4] = (I[1] * I[2] - I[0] * I[4]) / det;
    o[5] = (I[0] * I[3] - I[1] * I[1]) / det;
    return 0;
}

// Convex::computeVolume / computeInertia / computeCircumscribedRadius /
// computeBoundingBox at unit density.
int convex_props(const gb_convex& cv, const double* verts, double& volume, double I[6],
                 double I1[6], double& rc, double bb[3])
{
    const double* p = cv.p;
    for(int i = 0; i < 6; ++i)
        I[i] = I1[i] = 0.0;
    switch(cv.type)
    {
        case GB_SPHERE:
        {
            const double r = p[0]; // Sphere.cpp:68-101
            if(!(r > 0))
                return GB_E_INVALID_ARG;
            volume          = 4.0 * kPi * r * r * r / 3.0;
            const double r5 = r * r * r * r * r;
            I[5] = I[3] = I[0] = 8.0 * kPi / 15.0 * r5;
            I1[5] = I1[3] = I1[0] = 1.0 / I[0];
            rc                    = r;
            bb[0] = bb[1] = bb[2] = r;
            return GB_OK;
        }
        case GB_BOX:
        {
            const double ex = p[0], ey = p[1], ez = p[2]; // Box.cpp:79-123
            if(!(ex > 0 && ey > 0 && ez > 0))
                return GB_E_INVALID_ARG;
            volume = 8.0 * ex * ey * ez;
            I[0]   = 8.0 * ex * ey * ez * (ey * ey + ez * ez) / 3.0;
            I[3]   = 8.0 * ex * ey * ez * (ex * ex + ez * ez) / 3.0;
            I[5]   = 8.0 * ex * ey * ez * (ey * ey + ex * ex) / 3.0;
            I1[0]  = 1.0 / I[0];
            I1[3]  = 1.0 / I[3];
            I1[5]  = 1.0 / I[5];
            rc     = std::sqrt(ex * ex + ey * ey + ez * ez);
            bb[0] = ex, bb[1] = ey, bb[2] = ez;
            return GB_OK;
        }
        case GB_SUPERQUADRIC:
        {
            const double a = p[0], b = p[1], c = p[2], n1 = p[3], n2 = p[4];
            if(!(a > 0 && b > 0 && c > 0 && n1 >= 2 && n2 >= 2))
                return GB_E_INVALID_ARG;
            { // Superquadric::computeVolume (Superquadric.cpp:81-90)
                const double C    = 2.0 / 3.0 * a * b * c;
                const double eps1 = 2.0 / n1, eps2 = 2.0 / n2;
                volume = C * eps1 * eps2 * beta_fn(eps1, 0.5 * eps1) * beta_fn(0.5 * eps2, 0.5 * eps2);
            }
            { // Superquadric::computeInertia (Superquadric.cpp:95-117)
                const double eps1 = 2.0 / n1, eps2 = 2.0 / n2;
                const double C    = 0.4 * a * b * c * eps1 * eps2;
                const double prod1
                    = beta_fn(1.5 * eps2, 0.5 * eps2) * beta_fn(2.0 * eps1, 0.5 * eps1);
                const double prod2
                    = c * c * beta_fn(0.5 * eps2, 0.5 * eps2) * beta_fn(1.5 * eps1, eps1);
                I[0]  = C * (b * b * prod1 + prod2);
                I[3]  = C * (a * a * prod1 + prod2);
                I[5]  = C * (a * a + b * b) * prod1;
                I1[0] = 1.0 / I[0];
                I1[3] = 1.0 / I[3];
                I1[5] = 1.0 / I[5];
            }
            // Superquadric::computeCircumscribedRadius (Superquadric.cpp:122-155)
            if((n1 == 2.0) && (n2 == 2.0))
                rc = std::max(a, std::max(b, c));
            else if(n1 == 2.0)
            {
                const double alpha = std::pow(b / a, 2.0 / (n2 - 2.0));
                const double xt    = 1.0 / std::pow(1.0 + std::pow(alpha, n2), 1.0 / n2);
                rc = std::max(c, std::sqrt(a * xt * a * xt + alpha * b * xt * alpha * b * xt));
            }
            else if(n2 == 2.0)
            {
                const double m    = std::max(a, b);
                const double beta = std::pow(c * c / (m * m), 1.0 / (n1 - 2.0));
                const double xt   = 1.0 / std::pow(1.0 + std::pow(beta, n1), 1.0 / n1);
                rc                = std::sqrt(m * xt * m * xt + beta * c * xt * beta * c * xt);
            }
            else
            {
                const double alpha = std::pow(b / a, 2.0 / (n2 - 2.0));
                const double gamma = std::pow(1.0 + std::pow(alpha, n2), n1 / n2 - 1.0);
                const double beta  = std::pow(gamma * c * c / (a * a), 1.0 / (n1 - 1.0));
                const double xt
                    = 1.0
                      / std::pow(std::pow(1.0 + std::pow(alpha, n2), n1 / n2) + std::pow(beta, n1),
                                 1.0 / n1);
                rc = std::sqrt(a * xt * a * xt + alpha * b * xt * alpha * b * xt
                               + beta * c * xt * beta * c * xt);
            }
            bb[0] = a, bb[1] = b, bb[2] = c;
            return GB_OK;
        }
        case GB_RECTANGLE:
        {
            const double lx = p[0], ly = p[1]; // Rectangle.cpp:68-109
            volume          = 4.0 * lx * ly;
            I[0]            = 4.0 / 3.0 * lx * ly * ly * ly;
            I[3]            = 4.0 / 3.0 * lx * lx * lx * ly;
            I[5]            = 2.0 / 3.0 * lx * ly * (lx * lx + ly * ly);
            I1[0]           = 1.0 / I[0];
            I1[3]           = 1.0 / I[3];
            I1[5]           = 1.0 / I[5];
            rc              = std::sqrt(lx * lx + ly * ly);
            bb[0] = lx, bb[1] = ly, bb[2] = 0.0;
            return GB_OK;
        }
        case GB_DRUM:
        {
            // NEW: a wall (surface) only -- no volume, mass or inertia; the
            // bounding sphere and box of the cylinder R, half-length L
            const double R = p[0], L = p[1];
            if(!(R > 0.0) || L < 0.0)
                return GB_E_INVALID_ARG;
            volume = 0.0;
            rc     = std::sqrt(R * R + L * L);
            bb[0] = R, bb[1] = R, bb[2] = L;
            return GB_OK;
        }
        case GB_POLYHEDRON:
        {
            if(!verts || cv.n_vertices < 4 || cv.n_vertices > GB_MAX_POLY_VERTICES)
                return GB_E_INVALID_ARG;
            const double*     pv    = verts + 3 * cv.first_vertex;
            std::vector<Face> faces = convex_hull(pv, cv.n_vertices);
            if(faces.size() < 4)
                return GB_E_INVALID_ARG;
            double vol, c[3], sq[3], pr[3];
            polyhedron_moments(pv, faces, vol, c, sq, pr);
            if(!(vol > 0))
                return GB_E_INVALID_ARG;
            volume = vol;
            // inertia about the local origin: I = int (r.r 1 - r r^T) dV
            I[0] = sq[1] + sq[2];
            I[3] = sq[0] + sq[2];
            I[5] = sq[0] + sq[1];
            I[1] = -pr[0];
            I[2] = -pr[1];
            I[4] = -pr[2];
            if(inv_sym3(I, I1))
                return GB_E_INVALID_ARG;
            double r2 = 0;
            bb[0] = bb[1] = bb[2] = 0;
            for(int i = 0; i < cv.n_vertices; ++i)
            {
                const double* q = pv + 3 * i;
                r2              = std::max(r2, q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
                for(int k = 0; k < 3; ++k)
                    bb[k] = std::max(bb[k], std::fabs(q[k]));
            }
            rc = std::sqrt(r2);
            return GB_OK;
        }
        default:
            return GB_E_UNSUPPORTED;
    }
}

} // namespace

extern "C" int gb_rigid_body_properties(const gb_rigid_body_desc* rb, const double* vertices,
                                        gb_rigid_body_props* out)
{
    if(!rb || !out)
        return GB_E_INVALID_ARG;
    double I[6], I1[6], vol = 0, rc = 0, bb[3] = {0, 0, 0};
    int    st = convex_props(rb->convex, vertices, vol, I, I1, rc, bb);
    if(st)
        return st;
    // RigidBody.cpp:32-58: mass = density * volume; inertia *= density,
    // inverse /= density; all zero for density 0
    out->volume = vol;
    out->mass   = rb->density * vol;
    for(int i = 0; i < 6; ++i)
    {
        out->inertia[i]     = rb->density == 0 ? 0.0 : I[i] * rb->density;
        out->inertia_inv[i] = rb->density == 0 ? 0.0 : I1[i] / rb->density;
    }
    for(int k = 0; k < 3; ++k)
        out->bounding_box[k] = bb[k];
    out->circumscribed_radius = rc;
    return GB_OK;
}

extern "C" int gb_convex_hull_centroid(const double* points, int32_t n, double* centroid,
                                       double* volume)
{
    if(!points || n < 4 || n > GB_MAX_POLY_VERTICES || !centroid)
        return GB_E_INVALID_ARG;
    std::vector<Face> faces = convex_hull(points, n);
    if(faces.size() < 4)
        return GB_E_INVALID_ARG;
    double vol, c[3], sq[3], pr[3];
    polyhedron_moments(points, faces, vol, c, sq, pr);
    if(!(vol > 0))
        return GB_E_INVALID_ARG;
    for(int k = 0; k < 3; ++k)
        centroid[k] = c[k] / vol;
    if(volume)
        *volume = vol;
    return GB_OK;
}
