/*
 * oracle.c -- FP64 CPU restatement of Grains3D's per-time-step DEM loop.
 *
 * TEST INFRASTRUCTURE (see oracle.h): loaded only by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.
 *
 * Floating-point discipline: every restated function keeps the reference's
 * operation order and association (a + b + c is (a + b) + c, Vector3 dot
 * products start from 0, ...).  Built with -ffp-contract=off like the
 * reference harness, the restatement reproduces the reference bit for bit on
 * the same machine, except where a function is marked NEW (no reference
 * counterpart) or where noted (the Beta function of the superquadric mass
 * properties uses tgamma, as the reference's device path does).
 *
 * Reference paths are relative to the Grains3DGPU project root.
 */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Grains/Base/include/Basic.hh:103-128 (double values) */
#define OR_PI 3.1415926535897932385
#define OR_HIGHEPS 1.e-15
#define OR_EPS 1.e-10
#define OR_LOWEPS 1.e-05

/* ===========================================================================
 * Vector helpers: Grains/Base/include/VectorMath.hh, Vector3.cpp
 * ======================================================================== */
static inline double dot3(const double a[3], const double b[3])
{
    /* operator*(Vector3, Vector3): out = 0; out += a_i b_i (VectorMath.hh:116-126) */
    double o = 0.0;
    o += a[0] * b[0];
    o += a[1] * b[1];
    o += a[2] * b[2];
    return o;
}
static inline double norm3(const double a[3])
{
    return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); /* VectorMath.hh:20-25 */
}
static inline double norm2_3(const double a[3])
{
    return a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
}
static inline void cross3(const double a[3], const double b[3], double o[3])
{
    /* operator^ (VectorMath.hh:132-143) */
    double t0 = a[1] * b[2] - a[2] * b[1];
    double t1 = a[2] * b[0] - a[0] * b[2];
    double t2 = a[0] * b[1] - a[1] * b[0];
    o[0] = t0;
    o[1] = t1;
    o[2] = t2;
}
static inline void add3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[0] + b[0];
    o[1] = a[1] + b[1];
    o[2] = a[2] + b[2];
}
static inline void sub3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[0] - b[0];
    o[1] = a[1] - b[1];
    o[2] = a[2] - b[2];
}
static inline void scal3(double d, const double a[3], double o[3])
{
    o[0] = d * a[0];
    o[1] = d * a[1];
    o[2] = d * a[2];
}
static inline void copy3(const double a[3], double o[3])
{
    o[0] = a[0];
    o[1] = a[1];
    o[2] = a[2];
}
static inline void zero3(double o[3])
{
    o[0] = o[1] = o[2] = 0.0;
}
static inline void round3(double o[3], double tol)
{
    /* Vector3::round (Vector3.cpp:121-126) */
    for(int i = 0; i < 3; ++i)
        o[i] = fabs(o[i]) < tol ? 0.0 : o[i];
}
static inline int sgn(double x)
{
    return (0.0 < x) - (x < 0.0); /* MiscMath.hh:68-72 */
}

/* Matrix3 (row-major m[9]); MatrixMath.hh */
static inline void mat_vec(const double m[9], const double v[3], double o[3])
{
    /* operator*(Matrix3, Vector3) (MatrixMath.hh:127-138) */
    double t[3];
    for(int i = 0; i < 3; ++i)
        t[i] = m[3 * i] * v[0] + m[3 * i + 1] * v[1] + m[3 * i + 2] * v[2];
    copy3(t, o);
}
static inline void vec_mat(const double v[3], const double m[9], double o[3])
{
    /* operator*(Vector3, Matrix3) = M^T v (MatrixMath.hh:144-155) */
    double t[3];
    for(int i = 0; i < 3; ++i)
        t[i] = m[i] * v[0] + m[i + 3] * v[1] + m[i + 6] * v[2];
    copy3(t, o);
}
static inline void mat_mat(const double a[9], const double b[9], double o[9])
{
    /* operator*(Matrix3, Matrix3) (MatrixMath.hh:160-175); identical order to
       Matrix3::operator*=(Matrix3) (Matrix3.cpp:236-249) */
    double t[9];
    for(int r = 0; r < 3; ++r)
        for(int c = 0; c < 3; ++c)
            t[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c]
                           + a[3 * r + 2] * b[6 + c];
    memcpy(o, t, sizeof(t));
}
static inline void transpose9(const double m[9], double o[9])
{
    double t[9] = {m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]};
    memcpy(o, t, sizeof(t));
}

/* Transform3: tr[0..8] basis, tr[9..11] origin */
static inline void tr_apply(const double tr[12], const double v[3], double o[3])
{
    /* Transform3::operator() (Transform3.cpp:334-337): basis * v + origin */
    double t[3];
    mat_vec(tr, v, t);
    add3(t, tr + 9, o);
}
static void tr_relative(const double a2w[12], const double b2w[12], double b2a[12])
{
    /* Transform3(a2w, b2w) -> b2w.relativeToTransform(a2w)
       (Transform3.cpp:34-39, :313-318) */
    double inv[9], d[3];
    transpose9(a2w, inv);
    mat_mat(inv, b2w, b2a);
    sub3(b2w + 9, a2w + 9, d);
    mat_vec(inv, d, b2a + 9);
}

/* ===========================================================================
 * Convex shapes: support functions and mass properties
 * ======================================================================== */
static void sq_support(const double* p, const double v[3], double o[3])
{
    /* Superquadric::support (Grains/Geometry/src/Superquadric.cpp:169-205) */
    const double a = p[0], b = p[1], c = p[2], n1 = p[3], n2 = p[4];
    const double abvx = fabs(v[0]), abvy = fabs(v[1]), abvz = fabs(v[2]);
    const double signx = sgn(v[0]), signy = sgn(v[1]), signz = sgn(v[2]);
    if(abvx == 0.0)
    {
        if(abvy == 0.0)
        {
            o[0] = 0.0;
            o[1] = 0.0;
            o[2] = signz * c;
        }
        else
        {
            const double alpha = pow(c / b * abvz / abvy, 1.0 / (n1 - 1.0));
            const double yt    = 1.0 / pow(1.0 + pow(alpha, n1), 1.0 / n1);
            o[0]               = 0.0;
            o[1]               = signy * b * yt;
            o[2]               = signz * alpha * c * yt;
        }
    }
    else
    {
        const double alpha = pow(b / a * abvy / abvx, 1.0 / (n2 - 1.0));
        const double temp  = 1.0 + pow(alpha, n2);
        const double gamma = pow(temp, (n1 - n2) / (n2 * (n1 - 1.0)));
        const double beta  = gamma * pow(c / a * abvz / abvx, 1.0 / (n1 - 1.0));
        const double xt = 1.0 / pow(pow(temp, n1 / n2) + pow(beta, n1), 1.0 / n1);
        o[0]            = signx * a * xt;
        o[1]            = signy * alpha * b * xt;
        o[2]            = signz * beta * c * xt;
    }
}

static void convex_support(const gb_convex* cv, const double* verts,
                           const double v[3], double o[3])
{
    switch(cv->type)
    {
        case GB_SPHERE:
        {
            /* Sphere::support = r * v.normalized() (Sphere.cpp:111) */
            const double n = norm3(v);
            double       u[3] = {v[0] / n, v[1] / n, v[2] / n};
            scal3(cv->p[0], u, o);
            break;
        }
        case GB_BOX:
            /* Box::support (Box.cpp:129-134) */
            o[0] = v[0] < 0.0 ? -cv->p[0] : cv->p[0];
            o[1] = v[1] < 0.0 ? -cv->p[1] : cv->p[1];
            o[2] = v[2] < 0.0 ? -cv->p[2] : cv->p[2];
            break;
        case GB_SUPERQUADRIC:
            sq_support(cv->p, v, o);
            break;
        case GB_RECTANGLE:
            /* Rectangle::support (Rectangle.cpp:115-121) */
            o[0] = v[0] < 0.0 ? -cv->p[0] : cv->p[0];
            o[1] = v[1] < 0.0 ? -cv->p[1] : cv->p[1];
            o[2] = 0.0;
            break;
        case GB_POLYHEDRON:
        {
            /* NEW: argmax_i <p_i, v>, first index on ties. */
            const double* pv   = verts + 3 * cv->first_vertex;
            int           best = 0;
            double        bd   = dot3(pv, v);
            for(int i = 1; i < cv->n_vertices; ++i)
            {
                const double d = dot3(pv + 3 * i, v);
                if(d > bd)
                {
                    bd   = d;
                    best = i;
                }
            }
            copy3(pv + 3 * best, o);
            break;
        }
        default:
            o[0] = o[1] = o[2] = NAN;
    }
}

static double beta_fn(double x, double y)
{
    /* grainsBeta (Grains/Base/include/MiscMath.hh:82-90), device form */
    return tgamma(x) * tgamma(y) / tgamma(x + y);
}

/* NEW: convex hull faces of a small point set by exhaustive plane search,
   with coplanar points merged into one polygon (fan-triangulated).  Calls
   fn(a, b, c, user) once per outward-oriented triangle. */
typedef void (*tri_fn)(const double* a, const double* b, const double* c, void* u);
static int hull_triangles(const double* p, int n, tri_fn fn, void* user)
{
    if(n < 4 || n > GB_MAX_POLY_VERTICES)
        return -1;
    double scale = 0.0;
    for(int i = 0; i < 3 * n; ++i)
        scale = fmax(scale, fabs(p[i]));
    const double tol = 1e-12 * scale * scale * scale + 1e-300;
    /* planes already emitted: (normal, offset) */
    double planes[4 * 4 * GB_MAX_POLY_VERTICES * GB_MAX_POLY_VERTICES];
    int    nplanes = 0, ntri = 0;
    for(int i = 0; i < n; ++i)
        for(int j = i + 1; j < n; ++j)
            for(int k = j + 1; k < n; ++k)
            {
                double e1[3], e2[3], nr[3];
                sub3(p + 3 * j, p + 3 * i, e1);
                sub3(p + 3 * k, p + 3 * i, e2);
                cross3(e1, e2, nr);
                const double nn = norm3(nr);
                if(nn <= tol / (scale + 1e-300))
                    continue;
                int pos = 0, neg = 0;
                for(int m = 0; m < n; ++m)
                {
                    double d[3];
                    sub3(p + 3 * m, p + 3 * i, d);
                    const double s = dot3(d, nr);
                    if(s > tol)
                        ++pos;
                    else if(s < -tol)
                        ++neg;
                }
                if(pos && neg)
                    continue;
                double un[3] = {nr[0] / nn, nr[1] / nn, nr[2] / nn};
                if(pos)
                    scal3(-1.0, un, un); /* outward: all points behind */
                const double off = dot3(un, p + 3 * i);
                int          dup = 0;
                for(int q = 0; q < nplanes; ++q)
                    if(fabs(planes[4 * q] - un[0]) < 1e-9
                       && fabs(planes[4 * q + 1] - un[1]) < 1e-9
                       && fabs(planes[4 * q + 2] - un[2]) < 1e-9
                       && fabs(planes[4 * q + 3] - off) < 1e-9 * scale)
                        dup = 1;
                if(dup)
                    continue;
                planes[4 * nplanes]     = un[0];
                planes[4 * nplanes + 1] = un[1];
                planes[4 * nplanes + 2] = un[2];
                planes[4 * nplanes + 3] = off;
                ++nplanes;
                /* collect coplanar points, order them around their mean */
                int    idx[GB_MAX_POLY_VERTICES], cnt = 0;
                double ctr[3] = {0, 0, 0};
                for(int m = 0; m < n; ++m)
                {
                    double d[3];
                    sub3(p + 3 * m, p + 3 * i, d);
                    if(fabs(dot3(d, nr)) <= tol)
                    {
                        idx[cnt++] = m;
                        add3(ctr, p + 3 * m, ctr);
                    }
                }
                scal3(1.0 / cnt, ctr, ctr);
                double ax[3], ay[3];
                sub3(p + 3 * idx[0], ctr, ax);
                const double na = norm3(ax);
                scal3(1.0 / na, ax, ax);
                cross3(un, ax, ay);
                double ang[GB_MAX_POLY_VERTICES];
                for(int m = 0; m < cnt; ++m)
                {
                    double d[3];
                    sub3(p + 3 * idx[m], ctr, d);
                    ang[m] = atan2(dot3(d, ay), dot3(d, ax));
                }
                for(int a = 1; a < cnt; ++a) /* insertion sort by angle */
                    for(int b = a; b > 0 && ang[b] < ang[b - 1]; --b)
                    {
                        double ta  = ang[b];
                        ang[b]     = ang[b - 1];
                        ang[b - 1] = ta;
                        int ti     = idx[b];
                        idx[b]     = idx[b - 1];
                        idx[b - 1] = ti;
                    }
                /* counter-clockwise about the outward normal: fan */
                for(int m = 1; m + 1 < cnt; ++m)
                {
                    fn(p + 3 * idx[0], p + 3 * idx[m], p + 3 * idx[m + 1], user);
                    ++ntri;
                }
            }
    return ntri;
}

typedef struct
{
    double vol, c[3], xx, yy, zz, xy, xz, yz;
} poly_acc;
static void poly_tri(const double* a, const double* b, const double* c, void* u)
{
    /* NEW: mass properties by signed tetrahedra (origin, a, b, c). */
    poly_acc* s = (poly_acc*)u;
    double    bc[3];
    cross3(b, c, bc);
    const double det = dot3(a, bc);
    s->vol += det / 6.0;
    for(int i = 0; i < 3; ++i)
        s->c[i] += det / 24.0 * (a[i] + b[i] + c[i]);
#define SQ(i) (a[i] * a[i] + b[i] * b[i] + c[i] * c[i] + a[i] * b[i] + a[i] * c[i] + b[i] * c[i])
#define PR(i, j)                                                                 \
    (2.0 * (a[i] * a[j] + b[i] * b[j] + c[i] * c[j]) + a[i] * b[j] + a[j] * b[i] \
     + a[i] * c[j] + a[j] * c[i] + b[i] * c[j] + b[j] * c[i])
    s->xx += det / 60.0 * SQ(0);
    s->yy += det / 60.0 * SQ(1);
    s->zz += det / 60.0 * SQ(2);
    s->xy += det / 120.0 * PR(0, 1);
    s->xz += det / 120.0 * PR(0, 2);
    s->yz += det / 120.0 * PR(1, 2);
#undef SQ
#undef PR
}

static int inv_sym3(const double I[6], double o[6])
{
    /* inverse of the symmetric matrix [[0,1,2],[1,3,4],[2,4,5]] */
    const double c00 = I[3] * I[5] - I[4] * I[4];
    const double c01 = I[2] * I[4] - I[1] * I[5];
    const double c02 = I[1] * I[4] - I[2] * I[3];
    const double det = I[0] * c00 + I[1] * c01 + I[2] * c02;
    if(det == 0.0)
        return -1;
    o[0] = c00 / det;
    o[1] = c01 / det;
    o[2] = c02 / det;
    o[3] = (I[0] * I[5] - I[2] * I[2]) / det;
    o[4] = (I[1] * I[2] - I[0] * I[4]) / det;
    o[5] = (I[0] * I[3] - I[1] * I[1]) / det;
    return 0;
}

/* Convex::computeVolume / computeInertia / computeCircumscribedRadius /
   computeBoundingBox per shape, at unit density. */
static int convex_props(const gb_convex* cv, const double* verts, double* volume,
                        double I[6], double I1[6], double* rc, double bb[3])
{
    const double* p = cv->p;
    for(int i = 0; i < 6; ++i)
        I[i] = I1[i] = 0.0;
    switch(cv->type)
    {
        case GB_SPHERE:
        {
            /* Sphere.cpp:68-101 */
            const double r = p[0];
            *volume        = 4.0 * OR_PI * r * r * r / 3.0;
            const double r5 = r * r * r * r * r;
            I[5] = I[3] = I[0] = 8.0 * OR_PI / 15.0 * r5;
            I1[5] = I1[3] = I1[0] = 1.0 / I[0];
            *rc                   = r;
            bb[0] = bb[1] = bb[2] = r;
            return 0;
        }
        case GB_BOX:
        {
            /* Box.cpp:79-123 */
            const double ex = p[0], ey = p[1], ez = p[2];
            *volume         = 8.0 * ex * ey * ez;
            I[0]            = 8.0 * ex * ey * ez * (ey * ey + ez * ez) / 3.0;
            I[3]            = 8.0 * ex * ey * ez * (ex * ex + ez * ez) / 3.0;
            I[5]            = 8.0 * ex * ey * ez * (ey * ey + ex * ex) / 3.0;
            I1[0]           = 1.0 / I[0];
            I1[3]           = 1.0 / I[3];
            I1[5]           = 1.0 / I[5];
            *rc             = norm3(p);
            copy3(p, bb);
            return 0;
        }
        case GB_SUPERQUADRIC:
        {
            /* Superquadric.cpp:81-163 */
            const double a = p[0], b = p[1], c = p[2], n1 = p[3], n2 = p[4];
            {
                const double C    = 2.0 / 3.0 * a * b * c;
                const double eps1 = 2.0 / n1, eps2 = 2.0 / n2;
                *volume = C * eps1 * eps2 * beta_fn(eps1, 0.5 * eps1)
                          * beta_fn(0.5 * eps2, 0.5 * eps2);
            }
            {
                const double eps1 = 2.0 / n1, eps2 = 2.0 / n2;
                const double C    = 0.4 * a * b * c * eps1 * eps2;
                const double prod1
                    = beta_fn(1.5 * eps2, 0.5 * eps2) * beta_fn(2.0 * eps1, 0.5 * eps1);
                const double prod2 = c * c * beta_fn(0.5 * eps2, 0.5 * eps2)
                                     * beta_fn(1.5 * eps1, eps1);
                I[0]  = C * (b * b * prod1 + prod2);
                I[3]  = C * (a * a * prod1 + prod2);
                I[5]  = C * (a * a + b * b) * prod1;
                I1[0] = 1.0 / I[0];
                I1[3] = 1.0 / I[3];
                I1[5] = 1.0 / I[5];
            }
            if((n1 == 2.0) && (n2 == 2.0))
                *rc = fmax(a, fmax(b, c));
            else if(n1 == 2.0)
            {
                const double alpha = pow(b / a, 2.0 / (n2 - 2.0));
                const double xt    = 1.0 / pow(1.0 + pow(alpha, n2), 1.0 / n2);
                *rc = fmax(c, sqrt(a * xt * a * xt + alpha * b * xt * alpha * b * xt));
            }
            else if(n2 == 2.0)
            {
                const double m    = fmax(a, b);
                const double beta = pow(c * c / (m * m), 1.0 / (n1 - 2.0));
                const double xt   = 1.0 / pow(1.0 + pow(beta, n1), 1.0 / n1);
                *rc = sqrt(m * xt * m * xt + beta * c * xt * beta * c * xt);
            }
            else
            {
                const double alpha = pow(b / a, 2.0 / (n2 - 2.0));
                const double gamma = pow(1.0 + pow(alpha, n2), n1 / n2 - 1.0);
                const double beta  = pow(gamma * c * c / (a * a), 1.0 / (n1 - 1.0));
                const double xt
                    = 1.0
                      / pow(pow(1.0 + pow(alpha, n2), n1 / n2) + pow(beta, n1), 1.0 / n1);
                *rc = sqrt(a * xt * a * xt + alpha * b * xt * alpha * b * xt
                           + beta * c * xt * beta * c * xt);
            }
            bb[0] = a;
            bb[1] = b;
            bb[2] = c;
            return 0;
        }
        case GB_DRUM:
        {
            /* NEW: a wall only (no volume, mass or inertia); bounding sphere and
               box of the cylinder of radius p[0] and half-length p[1] */
            if(!(p[0] > 0.0) || p[1] < 0.0)
                return GB_E_INVALID_ARG;
            *volume = 0.0;
            *rc     = sqrt(p[0] * p[0] + p[1] * p[1]);
            bb[0]   = p[0];
            bb[1]   = p[0];
            bb[2]   = p[1];
            return 0;
        }
        case GB_RECTANGLE:
        {
            /* Rectangle.cpp:68-109 */
            const double lx = p[0], ly = p[1];
            *volume         = 4.0 * lx * ly;
            I[0]            = 4.0 / 3.0 * lx * ly * ly * ly;
            I[3]            = 4.0 / 3.0 * lx * lx * lx * ly;
            I[5]            = 2.0 / 3.0 * lx * ly * (lx * lx + ly * ly);
            I1[0]           = 1.0 / I[0];
            I1[3]           = 1.0 / I[3];
            I1[5]           = 1.0 / I[5];
            *rc             = sqrt(lx * lx + ly * ly);
            bb[0]           = lx;
            bb[1]           = ly;
            bb[2]           = 0.0;
            return 0;
        }
        case GB_POLYHEDRON:
        {
            /* NEW: hull volume and inertia about the local origin; bounding box
               and circumscribed radius from the vertices. */
            if(!verts || cv->n_vertices < 4 || cv->n_vertices > GB_MAX_POLY_VERTICES)
                return GB_E_INVALID_ARG;
            const double* pv = verts + 3 * cv->first_vertex;
            poly_acc      s;
            memset(&s, 0, sizeof(s));
            if(hull_triangles(pv, cv->n_vertices, poly_tri, &s) < 4)
                return GB_E_INVALID_ARG;
            *volume = s.vol;
            I[0]    = s.yy + s.zz;
            I[3]    = s.xx + s.zz;
            I[5]    = s.xx + s.yy;
            I[1]    = -s.xy;
            I[2]    = -s.xz;
            I[4]    = -s.yz;
            if(inv_sym3(I, I1))
                return GB_E_INVALID_ARG;
            double r2 = 0.0;
            bb[0] = bb[1] = bb[2] = 0.0;
            for(int i = 0; i < cv->n_vertices; ++i)
            {
                r2 = fmax(r2, norm2_3(pv + 3 * i));
                for(int k = 0; k < 3; ++k)
                    bb[k] = fmax(bb[k], fabs(pv[3 * i + k]));
            }
            *rc = sqrt(r2);
            return 0;
        }
        default:
            return GB_E_UNSUPPORTED;
    }
}

int or_rigid_body_properties(const gb_rigid_body_desc* rb, const double* vertices,
                             gb_rigid_body_props* out)
{
    /* RigidBody::RigidBody(convex, ct, material, density) (RigidBody.cpp:19-59) */
    if(!rb || !out)
        return GB_E_INVALID_ARG;
    double I[6], I1[6], vol, rc, bb[3];
    int    st = convex_props(&rb->convex, vertices, &vol, I, I1, &rc, bb);
    if(st)
        return st;
    out->volume = vol;
    out->mass   = rb->density * vol;
    for(int i = 0; i < 6; ++i)
    {
        out->inertia[i]     = rb->density == 0.0 ? 0.0 : I[i] * rb->density;
        out->inertia_inv[i] = rb->density == 0.0 ? 0.0 : I1[i] / rb->density;
    }
    copy3(bb, out->bounding_box);
    out->circumscribed_radius = rc;
    return GB_OK;
}

int or_support(const gb_convex* c, const double* vertices, const double v[3],
               double out[3])
{
    if(!c || !v || !out)
        return GB_E_INVALID_ARG;
    convex_support(c, vertices, v, out);
    return GB_OK;
}

/* ===========================================================================
 * OBB test: intersectOrientedBoundingBox (Grains/CollisionDetection/src/OBB.cpp:32-94)
 * ======================================================================== */
static int obb_test(const double a[3], const double b[3], const double trA[12],
                    const double trB[12])
{
    double ori[9], cen[3], d[3];
    transpose9(trA, ori);
    sub3(trB + 9, trA + 9, d);
    mat_vec(ori, d, cen);
    mat_mat(ori, trB, ori);
    double oa[9];
    for(int i = 0; i < 9; ++i)
        oa[i] = fabs(ori[i]) + OR_LOWEPS;
#define O(i, j) ori[3 * (i) + (j)]
#define OA(i, j) oa[3 * (i) + (j)]
    for(int i = 0; i < 3; ++i) /* TESTCASE1 */
        if(fabs(cen[i]) > (a[i] + b[0] * OA(i, 0) + b[1] * OA(i, 1) + b[2] * OA(i, 2)))
            return 0;
    for(int i = 0; i < 3; ++i) /* TESTCASE2 */
        if(fabs(cen[0] * O(0, i) + cen[1] * O(1, i) + cen[2] * O(2, i))
           > (b[i] + a[0] * OA(0, i) + a[1] * OA(1, i) + a[2] * OA(2, i)))
            return 0;
    static const int order[9][2]
        = {{0, 0}, {1, 0}, {2, 0}, {0, 1}, {1, 1}, {2, 1}, {0, 2}, {1, 2}, {2, 2}};
    for(int t = 0; t < 9; ++t) /* TESTCASE3(i, j) in the reference's order */
    {
        const int i = order[t][0], j = order[t][1];
        if(fabs(cen[(i + 2) % 3] * O((i + 1) % 3, j) - cen[(i + 1) % 3] * O((i + 2) % 3, j))
           > (a[(i + 1) % 3] * OA((i + 2) % 3, j) + a[(i + 2) % 3] * OA((i + 1) % 3, j)
              + b[(j + 1) % 3] * OA(i, (j + 2) % 3) + b[(j + 2) % 3] * OA(i, (j + 1) % 3)))
            return 0;
    }
#undef O
#undef OA
    return 1;
}

int or_obb(const double ext_a[3], const double ext_b[3], const double a2w[12],
           const double b2w[12])
{
    return obb_test(ext_a, ext_b, a2w, b2w);
}

/* ===========================================================================
 * GJK with Johnson's sub-algorithm (Grains/CollisionDetection/src/GJK_JH.cpp)
 * ======================================================================== */
static void jh_compute_det(unsigned bits, unsigned last, unsigned last_bit,
                           unsigned all_bits, double y[4][3], double dp[4][4],
                           double det[16][4])
{
    /* computeDet (GJK_JH.cpp:9-63) */
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
        if(bits & bit)
            dp[i][last] = dp[last][i] = dot3(y[i], y[last]);
    dp[last][last] = dot3(y[last], y[last]);

    det[last_bit][last] = 1.0;
    for(unsigned j = 0, sj = 1; j < 4; ++j, sj <<= 1)
    {
        if(bits & sj)
        {
            unsigned s2   = sj | last_bit;
            det[s2][j]    = dp[last][last] - dp[last][j];
            det[s2][last] = dp[j][j] - dp[j][last];
            for(unsigned k = 0, sk = 1; k < j; ++k, sk <<= 1)
            {
                if(bits & sk)
                {
                    unsigned s3 = sk | s2;
                    det[s3][k]  = det[s2][j] * (dp[j][j] - dp[j][k])
                                 + det[s2][last] * (dp[last][j] - dp[last][k]);
                    det[s3][j] = det[sk | last_bit][k] * (dp[k][k] - dp[k][j])
                                 + det[sk | last_bit][last] * (dp[last][k] - dp[last][j]);
                    det[s3][last] = det[sk | sj][k] * (dp[k][k] - dp[k][last])
                                    + det[sk | sj][j] * (dp[j][k] - dp[j][last]);
                }
            }
        }
    }
    if(all_bits == 15)
    {
        det[15][0] = det[14][1] * (dp[1][1] - dp[1][0]) + det[14][2] * (dp[2][1] - dp[2][0])
                     + det[14][3] * (dp[3][1] - dp[3][0]);
        det[15][1] = det[13][0] * (dp[0][0] - dp[0][1]) + det[13][2] * (dp[2][0] - dp[2][1])
                     + det[13][3] * (dp[3][0] - dp[3][1]);
        det[15][2] = det[11][0] * (dp[0][0] - dp[0][2]) + det[11][1] * (dp[1][0] - dp[1][2])
                     + det[11][3] * (dp[3][0] - dp[3][2]);
        det[15][3] = det[7][0] * (dp[0][0] - dp[0][3]) + det[7][1] * (dp[1][0] - dp[1][3])
                     + det[7][2] * (dp[2][0] - dp[2][3]);
    }
}

static int jh_valid(unsigned s, unsigned all_bits, double det[16][4])
{
    /* valid (GJK_JH.cpp:67-84) */
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    {
        if(all_bits & bit)
        {
            if(s & bit)
            {
                if(det[s][i] <= OR_EPS)
                    return 0;
            }
            else if(det[s | bit][i] > 0.0)
                return 0;
        }
    }
    return 1;
}

static void jh_compute_vector(unsigned bits, double y[4][3], double det[16][4],
                              double v[3])
{
    /* computeVector (GJK_JH.cpp:88-104) */
    double sum = 0.0;
    zero3(v);
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    {
        if(bits & bit)
        {
            sum += det[bits][i];
            double t[3];
            scal3(det[bits][i], y[i], t);
            add3(v, t, v);
        }
    }
    scal3(1.0 / sum, v, v);
}

static void jh_compute_points(unsigned bits, double det[16][4], double p[4][3],
                              double q[4][3], double p1[3], double p2[3])
{
    /* computePoints (GJK_JH.cpp:108-130) */
    double sum = 0.0;
    zero3(p1);
    zero3(p2);
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
    {
        if(bits & bit)
        {
            sum += det[bits][i];
            double t[3];
            scal3(det[bits][i], p[i], t);
            add3(p1, t, p1);
            scal3(det[bits][i], q[i], t);
            add3(p2, t, p2);
        }
    }
    const double s = 1.0 / sum;
    scal3(s, p1, p1);
    scal3(s, p2, p2);
}

static int jh_proper(unsigned s, double det[16][4])
{
    /* proper (GJK_JH.cpp:134-140) */
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
        if((s & bit) && det[s][i] <= OR_EPS)
            return 0;
    return 1;
}

static int jh_closest(unsigned* bits, unsigned last, unsigned last_bit,
                      unsigned all_bits, double y[4][3], double dp[4][4],
                      double det[16][4], double v[3])
{
    /* closest (GJK_JH.cpp:144-194), with the backup procedure */
    unsigned s;
    jh_compute_det(*bits, last, last_bit, all_bits, y, dp, det);
    for(s = *bits; s; --s)
    {
        if((s & *bits) == s)
        {
            if(jh_valid(s | last_bit, all_bits, det))
            {
                *bits = s | last_bit;
                jh_compute_vector(*bits, y, det, v);
                return 1;
            }
        }
    }
    if(jh_valid(last_bit, all_bits, det))
    {
        *bits = last_bit;
        copy3(y[last], v);
        return 1;
    }
    double min_dist2 = INFINITY;
    for(s = all_bits; s; --s)
    {
        if((s & all_bits) == s)
        {
            if(jh_proper(s, det))
            {
                double u[3];
                jh_compute_vector(s, y, det, u);
                const double dist2 = norm2_3(u);
                if(dist2 < min_dist2)
                {
                    min_dist2 = dist2;
                    *bits     = s;
                    copy3(u, v);
                }
            }
        }
    }
    return 0;
}

static int jh_degenerate(unsigned all_bits, double y[4][3], const double w[3])
{
    /* degenerate (GJK_JH.cpp:200-207) */
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
        if((all_bits & bit) && y[i][0] == w[0] && y[i][1] == w[1] && y[i][2] == w[2])
            return 1;
    return 0;
}

static double gjk_jh(const gb_convex* a, const double* va, const gb_convex* b,
                     const double* vb, const double a2w[12], const double b2w[12],
                     double pa[3], double pb[3], int* nb_iter)
{
    /* computeClosestPoints_GJK_JH (GJK_JH.cpp:310-391) */
    unsigned     bits = 0, last = 0, last_bit = 0, all_bits = 0;
    double       p[4][3], q[4][3], y[4][3];
    double       mu = 0.0;
    int          num_iterations = 0;
    double       det[16][4], dp[4][4];
    const double rel_error = OR_LOWEPS;
    const double abs_error = 1.e-4 * rel_error;
    memset(p, 0, sizeof(p));
    memset(q, 0, sizeof(q));
    memset(y, 0, sizeof(y));
    memset(det, 0, sizeof(det));
    memset(dp, 0, sizeof(dp));

    double b2a[12];
    tr_relative(a2w, b2w, b2a);

    double z[3] = {0.0, 0.0, 0.0}, sa[3], sb[3], tb[3], v[3], w[3];
    convex_support(a, va, z, sa);
    convex_support(b, vb, z, sb);
    tr_apply(b2a, sb, tb);
    sub3(sa, tb, v);
    double dist = norm3(v);

    while(bits < 15 && dist > OR_HIGHEPS && num_iterations < 1000)
    {
        last     = 0;
        last_bit = 1;
        while(bits & last_bit)
        {
            ++last;
            last_bit <<= 1;
        }
        double nv[3] = {-v[0], -v[1], -v[2]}, dir[3];
        convex_support(a, va, nv, p[last]);
        vec_mat(v, b2a, dir);
        convex_support(b, vb, dir, q[last]);
        tr_apply(b2a, q[last], tb);
        sub3(p[last], tb, w);

        const double g = dot3(v, w) / dist; /* set_max(mu, v * w / dist) */
        if(mu < g)
            mu = g;
        if(dist - mu <= dist * rel_error || mu < abs_error)
            break;
        if(jh_degenerate(all_bits, y, w))
            break;

        copy3(w, y[last]);
        all_bits = bits | last_bit;
        ++num_iterations;
        if(!jh_closest(&bits, last, last_bit, all_bits, y, dp, det, v))
            break;
        dist = norm3(v);
    }
    jh_compute_points(bits, det, p, q, pa, pb);
    if(nb_iter)
        *nb_iter = num_iterations;
    return dist;
}

/* ===========================================================================
 * GJK with the signed-volume sub-algorithm
 * (Grains/CollisionDetection/src/GJK_AY.cpp, Montanari et al. 2017)
 * ======================================================================== */
static unsigned sv_same_sign(double a, double b)
{
    /* compareSigns (GJK_AY.cpp:8-12) */
    return (unsigned)(!((a > 0) ^ (b > 0)));
}

static void sv_s1d(double y[4][3], unsigned* bits, double lambdas[4])
{
    /* s1d (GJK_AY.cpp:15-84) */
    int      s1_set = 0;
    unsigned i1 = 0, i2 = 0;
    for(unsigned i = 0; i < 4; ++i)
        if(*bits & (1u << i))
        {
            if(s1_set)
            {
                i2 = i;
                break;
            }
            i1     = i;
            s1_set = 1;
        }
    double t[3];
    sub3(y[i2], y[i1], t);
    unsigned I      = 0;
    double   neg_tI = -t[0];
    if(fabs(t[1]) > fabs(neg_tI))
    {
        I      = 1;
        neg_tI = -t[1];
    }
    if(fabs(t[2]) > fabs(neg_tI))
    {
        I      = 2;
        neg_tI = -t[2];
    }
    const double pI   = dot3(y[i2], t) / norm2_3(t) * neg_tI + y[i2][I];
    const double C[2] = {-y[i2][I] + pI, y[i1][I] - pI};
    const unsigned sc0 = sv_same_sign(neg_tI, C[0]), sc1 = sv_same_sign(neg_tI, C[1]);
    if(sc0 + sc1 == 2)
    {
        lambdas[i1] = C[0] / neg_tI;
        lambdas[i2] = C[1] / neg_tI;
    }
    else if(sc0)
    {
        *bits &= ~(1u << i2);
        lambdas[i1] = 1.0;
    }
    else
    {
        *bits &= ~(1u << i1);
        lambdas[i2] = 1.0;
    }
}

/* new_point = sum over the used points of lambda_i y_i, and its squared norm */
static double sv_point(double y[4][3], unsigned used, const double lambdas[4], double o[3])
{
    zero3(o);
    for(unsigned i = 0; i < 4; ++i)
        if(used & (1u << i))
        {
            double t[3];
            scal3(lambdas[i], y[i], t);
            add3(o, t, o);
        }
    return dot3(o, o);
}

static void sv_s2d(double y[4][3], unsigned* bits, double lambdas[4])
{
    /* s2d (GJK_AY.cpp:87-212) */
    unsigned counter = 0, i0 = 0, i1 = 0, i2 = 0;
    for(unsigned i = 0; i < 4; ++i)
        if(*bits & (1u << i))
        {
            if(counter == 0)
                i0 = i;
            else if(counter == 1)
                i1 = i;
            else
                i2 = i;
            counter += 1;
        }
    double e1[3], e2[3], n[3], p0[3];
    sub3(y[i1], y[i0], e1);
    sub3(y[i2], y[i0], e2);
    cross3(e1, e2, n);
    scal3(dot3(y[i0], n) / norm2_3(n), n, p0);
    double* Y0 = y[i0];
    double* Y1 = y[i1];
    double* Y2 = y[i2];
    unsigned ix = 1, iy = 2;
    double   mu_max = (Y1[1] * Y2[2] + Y0[1] * Y1[2] + Y2[1] * Y0[2] - Y1[1] * Y0[2]
                     - Y2[1] * Y1[2] - Y0[1] * Y2[2]);
    double mu = (Y1[2] * Y0[0] + Y2[2] * Y1[0] + Y0[2] * Y2[0] - Y1[2] * Y2[0]
                 - Y0[2] * Y1[0] - Y2[2] * Y0[0]);
    if(fabs(mu) > fabs(mu_max))
    {
        mu_max = mu;
        ix     = 0;
    }
    mu = (Y1[0] * Y2[1] + Y0[0] * Y1[1] + Y2[0] * Y0[1] - Y1[0] * Y0[1] - Y2[0] * Y1[1]
          - Y0[0] * Y2[1]);
    if(fabs(mu) > fabs(mu_max))
    {
        mu_max = mu;
        ix     = 0;
        iy     = 1;
    }
    double   C[3];
    unsigned sc[3];
    C[0] = (p0[ix] * Y1[iy] + p0[iy] * Y2[ix] + Y1[ix] * Y2[iy] - p0[ix] * Y2[iy]
            - p0[iy] * Y1[ix] - Y2[ix] * Y1[iy]);
    sc[0] = sv_same_sign(mu_max, C[0]);
    C[1] = (p0[ix] * Y2[iy] + p0[iy] * Y0[ix] + Y2[ix] * Y0[iy] - p0[ix] * Y0[iy]
            - p0[iy] * Y2[ix] - Y0[ix] * Y2[iy]);
    sc[1] = sv_same_sign(mu_max, C[1]);
    C[2] = (p0[ix] * Y0[iy] + p0[iy] * Y1[ix] + Y0[ix] * Y1[iy] - p0[ix] * Y1[iy]
            - p0[iy] * Y0[ix] - Y1[ix] * Y0[iy]);
    sc[2] = sv_same_sign(mu_max, C[2]);
    if(sc[0] + sc[1] + sc[2] == 3)
    {
        lambdas[i0] = C[0] / mu_max;
        lambdas[i1] = C[1] / mu_max;
        lambdas[i2] = C[2] / mu_max;
        return;
    }
    double   d        = 100000.0;
    unsigned new_bits = 0;
    const unsigned idx[3] = {i0, i1, i2};
    for(unsigned j = 0; j < 3; ++j)
        if(!sc[j])
        {
            unsigned new_used       = *bits & ~(1u << idx[j]);
            double   new_lambdas[4] = {0.0, 0.0, 0.0, 0.0};
            sv_s1d(y, &new_used, new_lambdas);
            double       np[3];
            const double d_star = sv_point(y, new_used, new_lambdas, np);
            if(d_star < d)
            {
                new_bits = new_used;
                d        = d_star;
                for(unsigned i = 0; i < 4; ++i)
                    lambdas[i] = new_lambdas[i];
            }
        }
    *bits = new_bits;
}

static void sv_s3d(double y[4][3], unsigned* bits, double lambdas[4])
{
    /* s3d (GJK_AY.cpp:215-301) */
    double C[4];
    C[0] = y[3][0] * y[2][1] * y[1][2] + y[2][0] * y[1][1] * y[3][2] + y[1][0] * y[3][1] * y[2][2]
           - y[1][0] * y[2][1] * y[3][2] - y[2][0] * y[3][1] * y[1][2]
           - y[3][0] * y[1][1] * y[2][2];
    C[1] = y[0][0] * y[2][1] * y[3][2] + y[2][0] * y[3][1] * y[0][2] + y[3][0] * y[0][1] * y[2][2]
           - y[3][0] * y[2][1] * y[0][2] - y[2][0] * y[0][1] * y[3][2]
           - y[0][0] * y[3][1] * y[2][2];
    C[2] = y[3][0] * y[1][1] * y[0][2] + y[1][0] * y[0][1] * y[3][2] + y[0][0] * y[3][1] * y[1][2]
           - y[0][0] * y[1][1] * y[3][2] - y[1][0] * y[3][1] * y[0][2]
           - y[3][0] * y[0][1] * y[1][2];
    C[3] = y[0][0] * y[1][1] * y[2][2] + y[1][0] * y[2][1] * y[0][2] + y[2][0] * y[0][1] * y[1][2]
           - y[2][0] * y[1][1] * y[0][2] - y[1][0] * y[0][1] * y[2][2]
           - y[0][0] * y[2][1] * y[1][2];
    const double dM = C[0] + C[1] + C[2] + C[3];
    unsigned     sc[4];
    for(int i = 0; i < 4; ++i)
        sc[i] = sv_same_sign(dM, C[i]);
    if(sc[0] + sc[1] + sc[2] + sc[3] == 4)
    {
        for(int i = 0; i < 4; ++i)
            lambdas[i] = C[i] / dM;
        return;
    }
    double   d        = 100000.0;
    unsigned new_bits = 0;
    for(unsigned j = 0; j < 4; ++j)
        if(!sc[j])
        {
            unsigned new_used       = *bits & ~(1u << j);
            double   new_lambdas[4] = {0.0, 0.0, 0.0, 0.0};
            sv_s2d(y, &new_used, new_lambdas);
            double       np[3];
            const double d_star = sv_point(y, new_used, new_lambdas, np);
            if(d_star < d)
            {
                new_bits = new_used;
                d        = d_star;
                for(unsigned i = 0; i < 4; ++i)
                    lambdas[i] = new_lambdas[i];
            }
        }
    *bits = new_bits;
}

static void sv_subalgorithm(double y[4][3], unsigned* bits, double lambdas[4], double v[3])
{
    /* sv_subalgorithm (GJK_AY.cpp:340-368) */
    unsigned num_used = 0;
    for(unsigned i = 0; i < 4; ++i)
        num_used += (*bits >> i) & 1u;
    if(num_used == 1)
    {
        for(unsigned i = 0; i < 4; ++i)
            if(*bits & (1u << i))
                lambdas[i] = 1.0;
    }
    else if(num_used == 2)
        sv_s1d(y, bits, lambdas);
    else if(num_used == 3)
        sv_s2d(y, bits, lambdas);
    else
        sv_s3d(y, bits, lambdas);
    sv_point(y, *bits, lambdas, v); /* computeVector (GJK_AY.cpp:304-316) */
}

static double gjk_sv(const gb_convex* a, const double* va, const gb_convex* b,
                     const double* vb, const double a2w[12], const double b2w[12],
                     double pa[3], double pb[3], int* nb_iter)
{
    /* computeClosestPoints_GJK_AY (GJK_AY.cpp:392-469) */
    unsigned     bits = 0, last = 0;
    double       p[4][3], q[4][3], y[4][3], lambdas[4] = {0.0, 0.0, 0.0, 0.0};
    int          num_iterations = 0;
    const double rel_error      = OR_LOWEPS;
    const double abs_error      = 1.e-4 * rel_error;
    memset(p, 0, sizeof(p));
    memset(q, 0, sizeof(q));
    memset(y, 0, sizeof(y));
    double b2a[12];
    tr_relative(a2w, b2w, b2a);
    double z[3] = {0.0, 0.0, 0.0}, sa[3], sb[3], tb[3], v[3], w[3];
    convex_support(a, va, z, sa);
    convex_support(b, vb, z, sb);
    tr_apply(b2a, sb, tb);
    sub3(sa, tb, v);
    double dist = norm3(v);
    while(bits < 15 && dist > OR_HIGHEPS && num_iterations < 1000)
    {
        for(unsigned k = 0; k < 4; ++k)
            if(!(bits & (1u << k)))
            {
                last = k;
                break;
            }
        double nv[3] = {-v[0], -v[1], -v[2]}, dir[3];
        convex_support(a, va, nv, p[last]);
        vec_mat(v, b2a, dir);
        convex_support(b, vb, dir, q[last]);
        tr_apply(b2a, q[last], tb);
        sub3(p[last], tb, w);
        const double mu = dist - dot3(v, w) / dist;
        if(mu < dist * rel_error || mu < abs_error)
            break;
        if(jh_degenerate(bits, y, w)) /* degenerate (GJK_AY.cpp:373-386): the current simplex */
            break;
        copy3(w, y[last]);
        bits |= 1u << last;
        ++num_iterations;
        sv_subalgorithm(y, &bits, lambdas, v);
        dist = norm3(v);
    }
    /* computePoints (GJK_AY.cpp:319-337) */
    zero3(pa);
    zero3(pb);
    for(unsigned i = 0; i < 4; ++i)
        if(bits & (1u << i))
        {
            double t[3];
            scal3(lambdas[i], p[i], t);
            add3(pa, t, pa);
            scal3(lambdas[i], q[i], t);
            add3(pb, t, pb);
        }
    if(nb_iter)
        *nb_iter = num_iterations;
    return dist;
}

/* ===========================================================================
 * Nesterov-accelerated GJK (no counterpart in the reference, whose GJK_JH.cpp
 * and GJK_AY.cpp keep only commented-out momentum variables).  Restated from
 * Montaut, Le Lidec, Petrik, Sivic and Carpentier, "Collision Detection
 * Accelerated: An Optimization Perspective" (RSS 2022), Algorithm 2, on the
 * signed-volume sub-algorithm above (the Johnson one's absolute determinant
 * test stops it early on mm-size grains).  The support direction is the
 * normalised momentum average
 *   y_k = delta_k x_k + (1 - delta_k) s_{k-1},   delta_k = (k + 1) / (k + 3),
 *   d_k = delta_k d_{k-1} / |d_{k-1}| + (1 - delta_k) y_k / |y_k|,
 * of the current closest point x_k (v) and the last support point s_{k-1};
 * x_0 = s_{-1} = d_{-1} is the first point.  The optimality gap of
 * GJK_AY.cpp, |x_k| - x_k . s_k / |x_k|, is no certificate when s_k was taken
 * along d_k rather than x_k (it can only understate the true gap), so when it
 * falls below the tolerance, or s_k repeats a simplex vertex, the iteration is
 * redone along x_k and the method continues as plain GJK, whose gap test then
 * ends it.
 * ======================================================================== */
static double gjk_nesterov(const gb_convex* a, const double* va, const gb_convex* b,
                           const double* vb, const double a2w[12], const double b2w[12],
                           double pa[3], double pb[3], int* nb_iter)
{
    unsigned     bits = 0, last = 0;
    double       p[4][3], q[4][3], y[4][3], lambdas[4] = {0.0, 0.0, 0.0, 0.0};
    int          num_iterations = 0, momentum = 1;
    const double rel_error = OR_LOWEPS;
    const double abs_error = 1.e-4 * rel_error;
    memset(p, 0, sizeof(p));
    memset(q, 0, sizeof(q));
    memset(y, 0, sizeof(y));
    double b2a[12];
    tr_relative(a2w, b2w, b2a);
    double z[3] = {0.0, 0.0, 0.0}, sa[3], sb[3], tb[3], v[3], w[3], d[3], s_prev[3];
    convex_support(a, va, z, sa);
    convex_support(b, vb, z, sb);
    tr_apply(b2a, sb, tb);
    sub3(sa, tb, v);
    copy3(v, d);
    copy3(v, s_prev);
    double dist = norm3(v);
    while(bits < 15 && dist > OR_HIGHEPS && num_iterations < 1000)
    {
        for(unsigned k = 0; k < 4; ++k)
            if(!(bits & (1u << k)))
            {
                last = k;
                break;
            }
        if(momentum)
        {
            const double delta = ((double)num_iterations + 1.0) / ((double)num_iterations + 3.0);
            double       yk[3];
            for(int k = 0; k < 3; ++k)
                yk[k] = delta * v[k] + (1.0 - delta) * s_prev[k];
            const double ny = norm3(yk), nd = norm3(d);
            if(ny > OR_HIGHEPS && nd > OR_HIGHEPS)
                for(int k = 0; k < 3; ++k)
                    d[k] = delta * (d[k] / nd) + (1.0 - delta) * (yk[k] / ny);
            else
            {
                momentum = 0;
                copy3(v, d);
            }
        }
        else
            copy3(v, d);
        double nd_[3] = {-d[0], -d[1], -d[2]}, dir[3];
        convex_support(a, va, nd_, p[last]);
        vec_mat(d, b2a, dir);
        convex_support(b, vb, dir, q[last]);
        tr_apply(b2a, q[last], tb);
        sub3(p[last], tb, w);
        const double mu = dist - dot3(v, w) / dist;
        if(mu < dist * rel_error || mu < abs_error || jh_degenerate(bits, y, w))
        {
            if(!momentum)
                break;
            momentum = 0; /* not a certified gap: redo this iteration along x_k */
            continue;
        }
        copy3(w, y[last]);
        bits |= 1u << last;
        ++num_iterations;
        sv_subalgorithm(y, &bits, lambdas, v);
        dist = norm3(v);
        copy3(w, s_prev);
    }
    zero3(pa);
    zero3(pb);
    for(unsigned i = 0; i < 4; ++i)
        if(bits & (1u << i))
        {
            double t[3];
            scal3(lambdas[i], p[i], t);
            add3(pa, t, pa);
            scal3(lambdas[i], q[i], t);
            add3(pb, t, pb);
        }
    if(nb_iter)
        *nb_iter = num_iterations;
    return dist;
}

double or_gjk(int variant, const gb_convex* a, const double* verts_a,
              const gb_convex* b, const double* verts_b, const double a2w[12],
              const double b2w[12], double pa[3], double pb[3], int* n_iter)
{
    if(variant == GB_GJK_SV)
        return gjk_sv(a, verts_a, b, verts_b, a2w, b2w, pa, pb, n_iter);
    if(variant == GB_GJK_NESTEROV)
        return gjk_nesterov(a, verts_a, b, verts_b, a2w, b2w, pa, pb, n_iter);
    return gjk_jh(a, verts_a, b, verts_b, a2w, b2w, pa, pb, n_iter);
}

/* ===========================================================================
 * Contact detection: Grains/CollisionDetection/src/CollisionDetection.cpp
 * ======================================================================== */
typedef struct
{
    const gb_convex* cv;
    const double*    verts;
    double           crust, rcirc, bb[3];
} body_view;

static void no_contact(or_contact* o)
{
    memset(o, 0, sizeof(*o)); /* noContact (Basic.hh:141) */
}

static void closest_spheres(const body_view* A, const body_view* B,
                            const double a2w[12], const double b2w[12], or_contact* o)
{
    /* closestPointsSpheres (CollisionDetection.cpp:26-48); a sphere's radius
       is its circumscribed radius, p[0] (rcirc may include the crust) */
    const double rA = A->cv->p[0], rB = B->cv->p[0];
    double       cen[3], vba[3];
    copy3(a2w + 9, cen);
    sub3(b2w + 9, cen, vba);
    const double overlap = norm3(vba) - rA - rB;
    const double n       = norm3(vba);
    vba[0] /= n;
    vba[1] /= n;
    vba[2] /= n;
    if(overlap < 0.0)
    {
        double t[3];
        scal3(rA + 0.5 * overlap, vba, t);
        add3(cen, t, o->pt);
        scal3(overlap, vba, o->vec);
        o->overlap = overlap;
    }
    else
        no_contact(o);
}

/* closestPointsRectangle (CollisionDetection.cpp:53-90) against the plane
   through rpt with normal rn_in (turned towards A's centre) */
static void closest_plane(const body_view* A, const double a2w[12], const double rpt[3],
                          const double rn_in[3], or_contact* o)
{
    double rn[3], d[3];
    copy3(rn_in, rn);
    sub3(a2w + 9, rpt, d);
    scal3(copysign(1.0, dot3(rn, d)), rn, rn);
    double nrn[3] = {-rn[0], -rn[1], -rn[2]}, dir[3], sa[3], pA[3];
    vec_mat(nrn, a2w, dir);
    convex_support(A->cv, A->verts, dir, sa);
    tr_apply(a2w, sa, pA);
    sub3(pA, rpt, d);
    if(dot3(rn, d) < 0.0)
    {
        double e[3], t[3], pB[3];
        sub3(rpt, pA, e);
        scal3(dot3(e, rn), rn, t);
        add3(t, pA, pB);
        add3(pA, pB, t);
        scal3(0.5, t, o->pt);
        sub3(pB, pA, o->vec);
        o->overlap = -norm3(o->vec);
    }
    else
        no_contact(o);
}

static void closest_rectangle(const body_view* A, const double a2w[12],
                              const double b2w[12], or_contact* o)
{
    /* the plane of the rectangle's frame: its origin, its z axis */
    const double rn[3] = {b2w[2], b2w[5], b2w[8]};
    closest_plane(A, a2w, b2w + 9, rn, o);
}

static void closest_drum(const body_view* A, const double a2w[12], const double b2w[12],
                         double R, or_contact* o)
{
    /* NEW: the inner wall of a drum of radius R about its frame's z axis.  The
       wall point nearest A's centre, w = origin + t + R e (t the axial part of
       the centre's offset, e the unit radial direction), and the inward normal
       -e give the tangent plane met as closest_plane meets a plane; a centre
       on the axis has no nearest point: no contact. */
    const double ax[3] = {b2w[2], b2w[5], b2w[8]};
    double       d[3], t[3], r[3], e[3], w[3], rn[3];
    sub3(a2w + 9, b2w + 9, d);
    scal3(dot3(ax, d), ax, t);
    sub3(d, t, r);
    const double nr = norm3(r);
    if(!(nr > 1e-12 * R))
    {
        no_contact(o);
        return;
    }
    scal3(1.0 / nr, r, e);
    add3(b2w + 9, t, w);
    scal3(R, e, t);
    add3(w, t, w);
    rn[0] = -e[0];
    rn[1] = -e[1];
    rn[2] = -e[2];
    closest_plane(A, a2w, w, rn, o);
}

static void closest_points(const body_view* A, const body_view* B,
                           const double a2w[12], const double b2w[12], int variant,
                           or_contact* o)
{
    /* closestPointsRigidBodies (CollisionDetection.cpp:182-284) */
    if(A->cv->type == GB_SPHERE && B->cv->type == GB_SPHERE)
    {
        closest_spheres(A, B, a2w, b2w, o);
        return;
    }
    else if(B->cv->type == GB_RECTANGLE)
    {
        closest_rectangle(A, a2w, b2w, o);
        return;
    }
    else if(B->cv->type == GB_DRUM)
    {
        closest_drum(A, a2w, b2w, B->cv->p[0], o);
        return;
    }
    double d[3];
    sub3(b2w + 9, a2w + 9, d);
    const double overlap = norm3(d) - (A->rcirc + B->rcirc);
    if(overlap < 0.0)
    {
        if(obb_test(A->bb, B->bb, a2w, b2w))
        {
            double pa[3], pb[3];
            int    nit = 0;
            double distance
                = or_gjk(variant, A->cv, A->verts, B->cv, B->verts, a2w, b2w, pa, pb, &nit);
            const double ct_sum = A->crust + B->crust;
            distance -= ct_sum;
            if(distance > 0.0)
            {
                no_contact(o);
                return;
            }
            double wa[3], wb[3], t[3];
            tr_apply(a2w, pa, wa);
            tr_apply(b2w, pb, wb);
            add3(wa, wb, t);
            o->pt[0] = t[0] / 2.0;
            o->pt[1] = t[1] / 2.0;
            o->pt[2] = t[2] / 2.0;
            sub3(wa, wb, o->vec);
            const double n = norm3(o->vec);
            o->vec[0] /= n;
            o->vec[1] /= n;
            o->vec[2] /= n;
            round3(o->vec, OR_EPS);
            scal3(-distance, o->vec, o->vec);
            o->overlap = distance;
            return;
        }
    }
    no_contact(o);
}

/* crust_bounds (GB_FLAG_CRUST_BOUNDS): the bounding tests' radius and
   half-extents grow by the crust thickness */
static void view_of(body_view* v, const gb_rigid_body_desc* rb,
                    const gb_rigid_body_props* pr, const double* verts, int crust_bounds)
{
    const double grow = crust_bounds ? rb->crust_thickness : 0.0;
    v->cv    = &rb->convex;
    v->verts = verts;
    v->crust = rb->crust_thickness;
    v->rcirc = pr->circumscribed_radius + grow;
    for(int k = 0; k < 3; ++k)
        v->bb[k] = pr->bounding_box[k] + grow;
}

int or_closest_points(const gb_rigid_body_desc* rb_a, const double* verts_a,
                      const gb_rigid_body_desc* rb_b, const double* verts_b,
                      const double a2w[12], const double b2w[12], int gjk_variant,
                      or_contact* out)
{
    gb_rigid_body_props pa, pb;
    int                 st = or_rigid_body_properties(rb_a, verts_a, &pa);
    if(st)
        return st;
    st = or_rigid_body_properties(rb_b, verts_b, &pb);
    if(st)
        return st;
    body_view A, B;
    view_of(&A, rb_a, &pa, verts_a, 0);
    view_of(&B, rb_b, &pb, verts_b, 0);
    closest_points(&A, &B, a2w, b2w, gjk_variant, out);
    return GB_OK;
}

/* ===========================================================================
 * Contact laws
 * ======================================================================== */
static double hooke_muen(double en)
{
    /* m_muen (HookeContactForceModel.cpp:56) */
    return log(en) / sqrt(OR_PI * OR_PI + log(en) * log(en));
}

static void hooke_forces(const gb_contact_model* cm, const or_contact* ci,
                         const double rel_vel[3], const double rel_ang_vel[3],
                         double m1, double m2, const double tr_origin[3],
                         double force[3], double torque[3])
{
    /* HookeContactForceModel::performForcesCalculus + computeForces
       (HookeContactForceModel.cpp:91-186) */
    const double m_muen = hooke_muen(cm->en);
    double       pen[3], delFN[3], delFT[3], delM[3] = {0, 0, 0};
    copy3(ci->vec, pen);
    scal3(cm->kn, pen, delFN);
    const double np = norm3(pen);
    pen[0] /= np;
    pen[1] /= np;
    pen[2] /= np;
    round3(pen, OR_EPS);

    double v_n[3], v_t[3];
    scal3(dot3(rel_vel, pen), pen, v_n);
    sub3(rel_vel, v_n, v_t);
    const double normv_t = norm3(v_t);
    double       tangent[3] = {0.0, 0.0, 0.0};
    if(normv_t > OR_EPS)
    {
        tangent[0] = v_t[0] / normv_t;
        tangent[1] = v_t[1] / normv_t;
        tangent[2] = v_t[2] / normv_t;
    }
    double avmass = m1 * m2 / (m1 + m2);
    double omega0 = sqrt(cm->kn / avmass);
    if(avmass == 0.0)
    {
        avmass = m2 == 0.0 ? 0.5 * m1 : 0.5 * m2;
        omega0 = 2.0 * sqrt(cm->kn / avmass);
    }
    const double muen = -omega0 * m_muen;
    double       t[3];
    scal3(-2.0 * muen * avmass, v_n, t);
    add3(delFN, t, delFN);
    const double normFN = norm3(delFN);

    scal3(-cm->etat * 2.0 * avmass, v_t, delFT);
    const double fn = cm->muc * normFN;
    const double ft = norm3(delFT);
    if(fn < ft)
        scal3(-fn, tangent, delFT);

    if(cm->kr != 0.0)
    {
        double wn[3], wt[3];
        scal3(dot3(rel_ang_vel, pen), pen, wn);
        sub3(rel_ang_vel, wn, wt);
        const double normwt = norm3(wt);
        scal3(-cm->kr * normFN * 0.001, wn, delM);
        if(normwt > OR_EPS)
        {
            scal3(cm->kr * normFN, wt, t);
            sub3(delM, t, delM);
        }
    }
    /* Torce::addForce(f, p) (Torce.cpp:90-94) */
    double f[3], arm[3], tq[3];
    add3(delFN, delFT, f);
    sub3(ci->pt, tr_origin, arm);
    add3(force, f, force);
    cross3(arm, f, tq);
    add3(torque, tq, torque);
    if(cm->kr != 0.0)
        add3(torque, delM, torque);
}

int or_hooke(const gb_contact_model* cm, const or_contact* ci,
             const double rel_vel[3], const double rel_ang_vel[3], double m1,
             double m2, const double tr_origin[3], double force[3], double torque[3])
{
    if(!cm || !ci || !force || !torque)
        return GB_E_INVALID_ARG;
    hooke_forces(cm, ci, rel_vel, rel_ang_vel, m1, m2, tr_origin, force, torque);
    return GB_OK;
}

/* NEW: linear spring-dashpot normal force (the Hooke normal part) plus a
   tangential spring kt with per-pair history xi, capped by Coulomb friction.
   Lever arms are measured from each body's centre.  xi (world frame) is
   projected on the current tangent plane, advanced by v_t dt, and rescaled to
   the Coulomb limit when sliding.  m2 == 0 (an obstacle) uses m* = m1. */
static void history_forces(const gb_contact_model* cm, const or_contact* ci,
                           const double rel_vel[3], double m1, double m2,
                           double dt, const double xi_prev[3], double xi_new[3],
                           const double tr_origin[3], double force[3],
                           double torque[3])
{
    double n[3];
    const double nv = norm3(ci->vec);
    n[0]            = ci->vec[0] / nv;
    n[1]            = ci->vec[1] / nv;
    n[2]            = ci->vec[2] / nv;
    const double mstar = m2 == 0.0 ? m1 : m1 * m2 / (m1 + m2);
    const double gn = -2.0 * hooke_muen(cm->en) * sqrt(cm->kn * mstar);
    const double vn = dot3(rel_vel, n);
    double       v_t[3], fn[3], t[3];
    scal3(vn, n, t);
    sub3(rel_vel, t, v_t);
    scal3(cm->kn, ci->vec, fn);
    scal3(-gn * vn, n, t);
    add3(fn, t, fn);
    const double fnorm = norm3(fn);

    double xi[3];
    scal3(dot3(xi_prev, n), n, t);
    sub3(xi_prev, t, xi);
    xi[0] += v_t[0] * dt;
    xi[1] += v_t[1] * dt;
    xi[2] += v_t[2] * dt;
    const double gt = 2.0 * cm->etat * mstar;
    double       ftv[3];
    for(int i = 0; i < 3; ++i)
        ftv[i] = -cm->kt * xi[i] - gt * v_t[i];
    const double ftn = norm3(ftv);
    const double cap = cm->muc * fnorm;
    if(ftn > cap)
    {
        const double s = cap / ftn;
        for(int i = 0; i < 3; ++i)
        {
            ftv[i] *= s;
            xi[i] = cm->kt > 0.0 ? -(ftv[i] + gt * v_t[i]) / cm->kt : 0.0;
        }
    }
    copy3(xi, xi_new);
    double f[3], arm[3], tq[3];
    add3(fn, ftv, f);
    sub3(ci->pt, tr_origin, arm);
    add3(force, f, force);
    cross3(arm, f, tq);
    add3(torque, tq, torque);
}

/* ===========================================================================
 * Quaternions and time integration
 * ======================================================================== */
typedef struct
{
    double w, v[3];
} quat;

static int quat_from_matrix(const double b[9], quat* q)
{
    /* Quaternion::setQuaternion(Matrix3) (Grains/Geometry/src/Quaternion.cpp:125-169) */
    enum { XX, XY, XZ, YX, YY, YZ, ZX, ZY, ZZ };
    double den;
    if(b[YY] > -b[ZZ] && b[XX] > -b[YY] && b[XX] > -b[ZZ])
    {
        den     = pow(1.0 + b[XX] + b[YY] + b[ZZ], 0.5);
        q->w    = 0.5 * den;
        q->v[0] = 0.5 * (b[ZY] - b[YZ]) / den;
        q->v[1] = 0.5 * (b[XZ] - b[ZX]) / den;
        q->v[2] = 0.5 * (b[YX] - b[XY]) / den;
    }
    else if(b[YY] < -b[ZZ] && b[XX] > b[YY] && b[XX] > b[ZZ])
    {
        den     = pow(1.0 + b[XX] - b[YY] - b[ZZ], 0.5);
        q->w    = 0.5 * (b[ZY] - b[YZ]) / den;
        q->v[0] = 0.5 * den;
        q->v[1] = 0.5 * (b[XY] + b[YX]) / den;
        q->v[2] = 0.5 * (b[ZX] + b[XZ]) / den;
    }
    else if(b[YY] > b[ZZ] && b[XX] < b[YY] && b[XX] < -b[ZZ])
    {
        den     = pow(1.0 - b[XX] + b[YY] - b[ZZ], 0.5);
        q->w    = 0.5 * (b[XZ] - b[ZX]) / den;
        q->v[0] = 0.5 * (b[XY] + b[YX]) / den;
        q->v[1] = 0.5 * den;
        q->v[2] = 0.5 * (b[YZ] + b[ZY]) / den;
    }
    else if(b[YY] < b[ZZ] && b[XX] < -b[YY] && b[XX] < b[ZZ])
    {
        den     = pow(1.0 - b[XX] - b[YY] + b[ZZ], 0.5);
        q->w    = 0.5 * (b[YX] - b[XY]) / den;
        q->v[0] = 0.5 * (b[ZX] + b[XZ]) / den;
        q->v[1] = 0.5 * (b[YZ] + b[ZY]) / den;
        q->v[2] = 0.5 * den;
    }
    else
    {
        q->w = 1.0;
        zero3(q->v);
        return -1; /* the reference leaves the quaternion undefined here */
    }
    return 0;
}

static void vec_times_quat(const double v[3], const quat* q, quat* o)
{
    /* operator*(Vector3, Quaternion) = [0, v] x q (QuaternionMath.hh:130-137) */
    double nv[3] = {-v[0], -v[1], -v[2]}, c[3], s[3];
    const double tmp = dot3(nv, q->v);
    cross3(v, q->v, c);
    scal3(q->w, v, s);
    add3(c, s, o->v);
    o->w = tmp;
}

static void quat_mult_to_vec(const quat* q, const quat* r, double o[3])
{
    /* Quaternion::multToVector3 (Quaternion.cpp:252-258) */
    double c[3], s1[3], s2[3], t[3];
    cross3(q->v, r->v, c);
    scal3(q->w, r->v, s1);
    scal3(r->w, q->v, s2);
    add3(c, s1, t);
    add3(t, s2, o);
}

static void compute_momentum(const gb_rigid_body_props* rb, const double omega[3],
                             const double torque[3], const double force[3],
                             const quat* q, double acc[3], double alpha[3])
{
    /* RigidBody::computeMomentum (Grains/Geometry/src/RigidBody.cpp:267-307) */
    quat qc = {q->w, {-q->v[0], -q->v[1], -q->v[2]}};
    quat t;
    double wb[3], am[3], tmp[3];
    const double* I  = rb->inertia;
    const double* I1 = rb->inertia_inv;
    vec_times_quat(omega, q, &t);
    quat_mult_to_vec(&qc, &t, wb);
    vec_times_quat(torque, q, &t);
    quat_mult_to_vec(&qc, &t, am);
    tmp[0] = I[0] * wb[0] + I[1] * wb[1] + I[2] * wb[2];
    tmp[1] = I[1] * wb[0] + I[3] * wb[1] + I[4] * wb[2];
    tmp[2] = I[2] * wb[0] + I[4] * wb[1] + I[5] * wb[2];
    double c[3];
    cross3(tmp, wb, c);
    add3(am, c, am);
    tmp[0] = I1[0] * am[0] + I1[1] * am[1] + I1[2] * am[2];
    tmp[1] = I1[1] * am[0] + I1[3] * am[1] + I1[4] * am[2];
    tmp[2] = I1[2] * am[0] + I1[4] * am[1] + I1[5] * am[2];
    vec_times_quat(tmp, &qc, &t);
    quat_mult_to_vec(q, &t, alpha);
    acc[0] = force[0] / rb->mass;
    acc[1] = force[1] / rb->mass;
    acc[2] = force[2] / rb->mass;
}

static void quaternion_change(const double w[3], double dt, quat* o)
{
    /* TimeIntegrator::computeQuaternionChange (TimeIntegrator.cpp:28-44) */
    const double n = norm3(w);
    if(n > OR_HIGHEPS)
    {
        const double c = cos(n * dt / 2.0);
        const double s = sin(n * dt / 2.0);
        scal3(s / n, w, o->v);
        o->w = c;
    }
    else
    {
        zero3(o->v);
        o->w = 1.0;
    }
}

static void compose_left_by_rotation(double m[9], const quat* q)
{
    /* Transform3::composeLeftByRotation(Quaternion) (Transform3.cpp:229-246) */
    const double qx = q->v[0], qy = q->v[1], qz = q->v[2], qw = q->w;
    for(int i = 0; i < 3; ++i)
    {
        const double px = qy * m[6 + i] - qz * m[3 + i] + qw * m[i];
        const double py = qz * m[i] - qx * m[6 + i] + qw * m[3 + i];
        const double pz = qx * m[3 + i] - qy * m[i] + qw * m[6 + i];
        const double pw = -qx * m[i] - qy * m[3 + i] - qz * m[6 + i];
        m[i]            = qy * pz - qz * py - pw * qx + qw * px;
        m[3 + i]        = qz * px - qx * pz - pw * qy + qw * py;
        m[6 + i]        = qx * py - qy * px - pw * qz + qw * pz;
    }
}

static int move_first_order(const gb_rigid_body_props* rb, double dt, double tr[12],
                            double kin[6], const double torce[6])
{
    /* ComponentManagerCPU::moveParticles (ComponentManagerCPU.cpp:470-499) with
       FirstOrderExplicit::Move (FirstOrderExplicit.cpp:46-60) */
    quat   q, dq;
    double acc[3], alpha[3], trans[3];
    int    warn = quat_from_matrix(tr, &q);
    compute_momentum(rb, kin + 3, torce + 3, torce, &q, acc, alpha);
    scal3(dt, kin, trans);
    double t[3];
    scal3(dt, acc, t);
    add3(kin, t, kin);
    quaternion_change(kin + 3, dt, &dq);
    scal3(dt, alpha, t);
    add3(kin + 3, t, kin + 3);
    add3(tr + 9, trans, tr + 9); /* updateTransform (Transform3.cpp:324-329) */
    compose_left_by_rotation(tr, &dq);
    return warn;
}

/* NEW: velocity-Verlet in kick-drift form with the force evaluation between
   the two half kicks of consecutive steps: v += h a, x += dt v, and the
   rotation increment uses the kicked omega.  h = dt/2 on the first step. */
static int move_verlet(const gb_rigid_body_props* rb, double dt, double h,
                       double tr[12], double kin[6], const double torce[6])
{
    quat   q, dq;
    double acc[3], alpha[3], t[3];
    int    warn = quat_from_matrix(tr, &q);
    compute_momentum(rb, kin + 3, torce + 3, torce, &q, acc, alpha);
    scal3(h, acc, t);
    add3(kin, t, kin);
    scal3(h, alpha, t);
    add3(kin + 3, t, kin + 3);
    scal3(dt, kin, t);
    add3(tr + 9, t, tr + 9);
    quaternion_change(kin + 3, dt, &dq);
    compose_left_by_rotation(tr, &dq);
    return warn;
}

int or_move_first_order(const gb_rigid_body_props* rb, double dt, double tr[12],
                        double kin[6], const double torce[6])
{
    move_first_order(rb, dt, tr, kin, torce);
    return GB_OK;
}

/* ===========================================================================
 * Linked cell (Grains/Component/src/LinkedCell.cpp)
 * ======================================================================== */
int or_linked_cell_dims(const double min[3], const double max[3], double extent,
                        uint32_t dims[3])
{
    /* LinkedCell::LinkedCell (LinkedCell.cpp:16-29) */
    for(int i = 0; i < 3; ++i)
    {
        double t = OR_EPS;
        t += max[i] - min[i];
        t /= extent;
        dims[i] = (uint32_t)t;
    }
    return GB_OK;
}

static inline int64_t cell_coord(double p, double mn, double extent)
{
    /* LinkedCell::computeCellId (LinkedCell.cpp:117-130): floor((p-min)/extent) */
    const double f = floor((p - mn) / extent);
    if(!(f >= 0.0))
        return -1;
    if(f > 2147483647.0)
        return 2147483647;
    return (int64_t)f;
}

int or_cell_hash(const double min[3], const double max[3], double extent, int64_t n,
                 const double* pos3, uint32_t* hash)
{
    uint32_t d[3];
    or_linked_cell_dims(min, max, extent, d);
    int st = GB_OK;
    for(int64_t i = 0; i < n; ++i)
    {
        int64_t c[3];
        for(int k = 0; k < 3; ++k)
        {
            c[k] = cell_coord(pos3[3 * i + k], min[k], extent);
            if(c[k] < 0 || c[k] >= (int64_t)d[k])
            {
                st   = GB_E_OUT_OF_DOMAIN;
                c[k] = c[k] < 0 ? 0 : (int64_t)d[k] - 1;
            }
        }
        hash[i] = (uint32_t)((c[2] * d[1] + c[1]) * d[0] + c[0]);
    }
    return st;
}

/* ===========================================================================
 * The system: ComponentManagerCPU driven in GrainsCPU::simulate order
 * ======================================================================== */
struct or_ctx
{
    gb_config           cfg;
    int                 threads;
    int32_t             n, nrb, nob, nmat;
    gb_rigid_body_desc* rbs;
    gb_rigid_body_props* rbp;
    double*             verts;
    int64_t             nverts;
    gb_rigid_body_desc* obs;
    gb_rigid_body_props* obp;
    double*             obs_tr;
    double*             obs_vel; /* 6 per obstacle: velocity, angular velocity */
    gb_contact_model*   cm;
    uint32_t*           rb_id;
    double*             tr;    /* 12 per particle */
    double*             kin;   /* 6 per particle */
    double*             torce; /* force(3) torque(3) */
    /* linked cell */
    double   cell, lc_max[3];
    uint32_t dims[3], ncells;
    uint32_t* nbr; /* 27 per cell */
    uint32_t* hash;
    uint32_t* cell_start; /* ncells + 1 */
    uint32_t* sorted;
    int       links_valid;
    /* per-step pair records (candidates) */
    int64_t   npairs, pair_cap;
    uint32_t* pair_off; /* n + 1 */
    uint32_t* pair_b;
    or_contact* pair_ci;
    unsigned char* pair_contact;
    double*   pair_xi; /* history law: 3 per pair */
    /* history of the previous step */
    int64_t   hist_n;
    uint32_t* hist_off;
    uint32_t* hist_b;
    double*   hist_xi;
    int64_t   steps_done, contacts, obstacle_contacts, gjk_calls, gjk_iters;
    int32_t   status_flags;
    int       verlet_started;
};

static void* xcalloc(size_t n, size_t s)
{
    return calloc(n ? n : 1, s);
}

or_ctx* or_create(const gb_config* cfg, int* status)
{
    int st = GB_OK;
    if(!cfg || cfg->n_particles < 0 || cfg->n_rigid_bodies < 1 || cfg->n_obstacles < 0
       || cfg->n_materials < 1 || !(cfg->dt > 0.0))
        st = GB_E_INVALID_ARG;
    or_ctx* c = NULL;
    if(st == GB_OK)
    {
        c = (or_ctx*)xcalloc(1, sizeof(or_ctx));
        if(!c)
            st = GB_E_OUT_OF_MEMORY;
    }
    if(st == GB_OK)
    {
        c->cfg     = *cfg;
        c->threads = 1;
        c->n       = cfg->n_particles;
        c->nrb     = cfg->n_rigid_bodies;
        c->nob     = cfg->n_obstacles;
        c->nmat    = cfg->n_materials;
        int64_t n  = c->n;
        c->rbs     = xcalloc(c->nrb, sizeof(gb_rigid_body_desc));
        c->rbp     = xcalloc(c->nrb, sizeof(gb_rigid_body_props));
        c->obs     = xcalloc(c->nob, sizeof(gb_rigid_body_desc));
        c->obp     = xcalloc(c->nob, sizeof(gb_rigid_body_props));
        c->obs_tr  = xcalloc((size_t)c->nob * 12, sizeof(double));
        c->obs_vel = xcalloc((size_t)c->nob * 6 + 1, sizeof(double));
        c->cm      = xcalloc((size_t)c->nmat * (c->nmat + 1) / 2, sizeof(gb_contact_model));
        c->rb_id   = xcalloc(n, sizeof(uint32_t));
        c->tr      = xcalloc(n * 12, sizeof(double));
        c->kin     = xcalloc(n * 6, sizeof(double));
        c->torce   = xcalloc(n * 6, sizeof(double));
        c->hash    = xcalloc(n, sizeof(uint32_t));
        c->sorted  = xcalloc(n, sizeof(uint32_t));
        c->pair_off = xcalloc(n + 1, sizeof(uint32_t));
        c->hist_off = xcalloc(n + 1, sizeof(uint32_t));
        for(int64_t i = 0; i < n; ++i)
        {
            double* t = c->tr + 12 * i;
            t[0] = t[4] = t[8] = 1.0;
        }
    }
    if(status)
        *status = st;
    return st == GB_OK ? c : NULL;
}

int or_destroy(or_ctx* c)
{
    if(!c)
        return GB_E_INVALID_ARG;
    free(c->rbs);
    free(c->rbp);
    free(c->verts);
    free(c->obs);
    free(c->obp);
    free(c->obs_tr);
    free(c->obs_vel);
    free(c->cm);
    free(c->rb_id);
    free(c->tr);
    free(c->kin);
    free(c->torce);
    free(c->nbr);
    free(c->hash);
    free(c->cell_start);
    free(c->sorted);
    free(c->pair_off);
    free(c->pair_b);
    free(c->pair_ci);
    free(c->pair_contact);
    free(c->pair_xi);
    free(c->hist_off);
    free(c->hist_b);
    free(c->hist_xi);
    free(c);
    return GB_OK;
}

int or_set_threads(or_ctx* c, int32_t n_threads)
{
    if(!c || n_threads < 1)
        return GB_E_INVALID_ARG;
    c->threads = n_threads;
    return GB_OK;
}

/* the bounding radius of rigid body i in the candidate test and the cell
   size: the circumscribed radius, plus the crust under GB_FLAG_CRUST_BOUNDS */
static double bound_radius(const or_ctx* c, int32_t i)
{
    return c->rbp[i].circumscribed_radius
           + ((c->cfg.flags & GB_FLAG_CRUST_BOUNDS) ? c->rbs[i].crust_thickness : 0.0);
}

static int build_linked_cell(or_ctx* c)
{
    /* Grains::Construction (Grains/Base/src/Grains.cpp:226-246): cell size is
       CellSizeFactor * 2 * max circumscribed radius over particles. */
    double lc = 0.0;
    for(int32_t i = 0; i < c->nrb; ++i)
        if(bound_radius(c, i) > lc)
            lc = bound_radius(c, i);
    double coeff = c->cfg.cell_size_factor;
    if(coeff < 1.0)
        coeff = 1.0;
    c->cell = coeff * 2.0 * lc;
    for(int k = 0; k < 3; ++k)
        c->lc_max[k] = c->cfg.max_coordinate[k] + (c->cfg.pad_grid ? c->cell : 0.0);
    or_linked_cell_dims(c->cfg.origin, c->lc_max, c->cell, c->dims);
    uint64_t nc = (uint64_t)c->dims[0] * c->dims[1] * c->dims[2];
    if(nc == 0 || nc > 0xFFFFFFF0ull)
        return GB_E_INVALID_ARG;
    c->ncells = (uint32_t)nc;
    free(c->nbr);
    free(c->cell_start);
    c->nbr        = xcalloc((size_t)nc * 27, sizeof(uint32_t));
    c->cell_start = xcalloc((size_t)nc + 1, sizeof(uint32_t));
    if(!c->nbr || !c->cell_start)
        return GB_E_OUT_OF_MEMORY;
    const uint32_t nx = c->dims[0], ny = c->dims[1], nz = c->dims[2];
    for(uint32_t h = 0; h < c->ncells; ++h) /* LinkedCell.cpp:35-72 */
    {
        uint32_t off = h * 27;
        int      cx = (int)(h % nx), cy = (int)((h / nx) % ny), cz = (int)(h / (nx * ny));
        for(int k = -1; k < 2; ++k)
            for(int j = -1; j < 2; ++j)
                for(int i = -1; i < 2; ++i)
                {
                    int x = cx + i, y = cy + j, z = cz + k;
                    if(x >= 0 && x < (int)nx && y >= 0 && y < (int)ny && z >= 0 && z < (int)nz)
                        c->nbr[off++] = (uint32_t)x + (uint32_t)y * nx + (uint32_t)z * nx * ny;
                    else
                        c->nbr[off++] = UINT32_MAX;
                }
    }
    return GB_OK;
}

int or_set_rigid_bodies(or_ctx* c, const gb_rigid_body_desc* rbs, const double* vertices,
                        int64_t n_vertices)
{
    if(!c || !rbs || n_vertices < 0 || (n_vertices && !vertices))
        return GB_E_INVALID_ARG;
    free(c->verts);
    c->verts  = xcalloc((size_t)n_vertices * 3, sizeof(double));
    c->nverts = n_vertices;
    if(n_vertices)
        memcpy(c->verts, vertices, (size_t)n_vertices * 3 * sizeof(double));
    for(int32_t i = 0; i < c->nrb; ++i)
    {
        c->rbs[i] = rbs[i];
        if(rbs[i].convex.type == GB_POLYHEDRON
           && (rbs[i].convex.first_vertex < 0
               || rbs[i].convex.first_vertex + rbs[i].convex.n_vertices > n_vertices))
            return GB_E_INVALID_ARG;
        if(rbs[i].material < 0 || rbs[i].material >= c->nmat)
            return GB_E_INVALID_ARG;
        int st = or_rigid_body_properties(&rbs[i], c->verts, &c->rbp[i]);
        if(st)
            return st;
    }
    return build_linked_cell(c);
}

int or_get_rigid_body_props(or_ctx* c, int32_t rb, gb_rigid_body_props* out)
{
    if(!c || !out || rb < 0 || rb >= c->nrb)
        return GB_E_INVALID_ARG;
    *out = c->rbp[rb];
    return GB_OK;
}

int or_set_rigid_body_props(or_ctx* c, int32_t rb, const gb_rigid_body_props* in)
{
    /* test hook: lets a pinning test use the reference's own mass properties
       (std::beta) instead of the tgamma form above */
    if(!c || !in || rb < 0 || rb >= c->nrb)
        return GB_E_INVALID_ARG;
    c->rbp[rb] = *in;
    return GB_OK;
}

int or_set_contact_models(or_ctx* c, const gb_contact_model* table)
{
    if(!c || !table)
        return GB_E_INVALID_ARG;
    memcpy(c->cm, table, (size_t)c->nmat * (c->nmat + 1) / 2 * sizeof(gb_contact_model));
    return GB_OK;
}

int or_set_obstacles(or_ctx* c, const gb_rigid_body_desc* obst, const double* tr)
{
    if(!c || (c->nob && (!obst || !tr)))
        return GB_E_INVALID_ARG;
    for(int32_t i = 0; i < c->nob; ++i)
    {
        c->obs[i] = obst[i];
        if(obst[i].convex.type == GB_POLYHEDRON)
            return GB_E_UNSUPPORTED;
        int st = or_rigid_body_properties(&obst[i], NULL, &c->obp[i]);
        if(st)
            return st;
    }
    memcpy(c->obs_tr, tr, (size_t)c->nob * 12 * sizeof(double));
    return GB_OK;
}

int or_set_obstacle_velocities(or_ctx* c, const double* kin)
{
    /* NEW (gb_set_obstacle_velocities): the walls' surface velocities */
    if(!c || (c->nob && !kin))
        return GB_E_INVALID_ARG;
    memcpy(c->obs_vel, kin, (size_t)c->nob * 6 * sizeof(double));
    return GB_OK;
}

int or_set_rigid_body_ids(or_ctx* c, const uint32_t* ids)
{
    if(!c || !ids)
        return GB_E_INVALID_ARG;
    for(int32_t i = 0; i < c->n; ++i)
        if(ids[i] >= (uint32_t)c->nrb)
            return GB_E_INVALID_ARG;
    memcpy(c->rb_id, ids, (size_t)c->n * sizeof(uint32_t));
    return GB_OK;
}

int or_set_transforms(or_ctx* c, const double* t)
{
    if(!c || !t)
        return GB_E_INVALID_ARG;
    memcpy(c->tr, t, (size_t)c->n * 12 * sizeof(double));
    return GB_OK;
}
int or_set_velocities(or_ctx* c, const double* k)
{
    if(!c || !k)
        return GB_E_INVALID_ARG;
    memcpy(c->kin, k, (size_t)c->n * 6 * sizeof(double));
    return GB_OK;
}
int or_get_transforms(or_ctx* c, double* t)
{
    if(!c || !t)
        return GB_E_INVALID_ARG;
    memcpy(t, c->tr, (size_t)c->n * 12 * sizeof(double));
    return GB_OK;
}
int or_get_velocities(or_ctx* c, double* k)
{
    if(!c || !k)
        return GB_E_INVALID_ARG;
    memcpy(k, c->kin, (size_t)c->n * 6 * sizeof(double));
    return GB_OK;
}
int or_get_torces(or_ctx* c, double* t)
{
    if(!c || !t)
        return GB_E_INVALID_ARG;
    memcpy(t, c->torce, (size_t)c->n * 6 * sizeof(double));
    return GB_OK;
}

/* ComponentManagerCPU::setTorce (ComponentManagerCPU.cpp, m_torce = t). */
int or_set_torces(or_ctx* c, const double* t)
{
    if(!c || !t)
        return GB_E_INVALID_ARG;
    memcpy(c->torce, t, (size_t)c->n * 6 * sizeof(double));
    return GB_OK;
}

int or_update_links(or_ctx* c)
{
    /* ComponentManagerCPU::updateLinks (ComponentManagerCPU.cpp:278-296): cell
       hash per particle, then cell lists filled in particle-id order (so ids
       ascend within a cell). */
    if(!c || !c->nbr)
        return GB_E_NOT_READY;
    const int64_t n  = c->n;
    int           st = GB_OK;
    for(int64_t i = 0; i < n; ++i)
    {
        int64_t cc[3];
        for(int k = 0; k < 3; ++k)
        {
            cc[k] = cell_coord(c->tr[12 * i + 9 + k], c->cfg.origin[k], c->cell);
            if(cc[k] < 0 || cc[k] >= (int64_t)c->dims[k])
            {
                st    = GB_E_OUT_OF_DOMAIN;
                cc[k] = cc[k] < 0 ? 0 : (int64_t)c->dims[k] - 1;
            }
        }
        c->hash[i] = (uint32_t)((cc[2] * c->dims[1] + cc[1]) * c->dims[0] + cc[0]);
    }
    memset(c->cell_start, 0, ((size_t)c->ncells + 1) * sizeof(uint32_t));
    for(int64_t i = 0; i < n; ++i)
        c->cell_start[c->hash[i] + 1]++;
    for(uint32_t h = 0; h < c->ncells; ++h)
        c->cell_start[h + 1] += c->cell_start[h];
    uint32_t* fill = xcalloc(c->ncells, sizeof(uint32_t));
    for(int64_t i = 0; i < n; ++i)
    {
        const uint32_t h = c->hash[i];
        c->sorted[c->cell_start[h] + fill[h]++] = (uint32_t)i;
    }
    free(fill);
    c->links_valid = 1;
    if(st)
        c->status_flags |= 1 << (-st);
    return st;
}

static inline const gb_contact_model* model_for(const or_ctx* c, int ma, int mb)
{
    /* ContactForceModelBuilderFactory::computeHash (ContactForceModelBuilderFactory.cpp:77-83) */
    const unsigned s = ma < mb ? ma : mb, l = ma < mb ? mb : ma;
    return &c->cm[l * (l + 1) / 2 + s];
}

static inline double* hist_lookup(or_ctx* c, uint32_t a, uint32_t b)
{
    if(!c->hist_b)
        return NULL;
    for(uint32_t k = c->hist_off[a]; k < c->hist_off[a + 1]; ++k)
        if(c->hist_b[k] == b)
            return c->hist_xi + 3 * k;
    return NULL;
}

static int ensure_pairs(or_ctx* c, int64_t need)
{
    if(need <= c->pair_cap)
        return GB_OK;
    int64_t cap = need + need / 2 + 16;
    free(c->pair_b);
    free(c->pair_ci);
    free(c->pair_contact);
    free(c->pair_xi);
    c->pair_b       = xcalloc(cap, sizeof(uint32_t));
    c->pair_ci      = xcalloc(cap, sizeof(or_contact));
    c->pair_contact = xcalloc(cap, 1);
    c->pair_xi      = xcalloc(cap * 3, sizeof(double));
    c->pair_cap     = cap;
    return (c->pair_b && c->pair_ci && c->pair_contact && c->pair_xi) ? GB_OK
                                                                      : GB_E_OUT_OF_MEMORY;
}

static inline void kin_at_point(const double kin[6], const double r[3], double o[3])
{
    /* Kinematics::kinematicsAtPoint (Kinematics.cpp:87-90): v + w ^ R */
    double c[3];
    cross3(kin + 3, r, c);
    add3(kin, c, o);
}

int or_detect_collision_and_compute_contact_forces(or_ctx* c, int32_t* result)
{
    /* ComponentManagerCPU::detectCollisionAndComputeContactForces
       (ComponentManagerCPU.cpp:428-443) */
    int st = or_update_links(c);
    if(st && st != GB_E_OUT_OF_DOMAIN)
        return st;
    const int64_t n       = c->n;
    const int     hist    = c->cfg.contact_law == GB_LAW_HOOKE_HISTORY;
    const int     variant = c->cfg.gjk_variant;
    const int     cb      = (c->cfg.flags & GB_FLAG_CRUST_BOUNDS) != 0;

    /* enumeration pass 1: bounding-sphere candidates per particle, in the
       reference's order (27 neighbour cells in k, j, i order; ids ascending) */
    int64_t total = 0;
    for(int64_t a = 0; a < n; ++a)
    {
        c->pair_off[a]        = (uint32_t)total;
        const uint32_t* nbl   = c->nbr + 27 * (size_t)c->hash[a];
        const double    ra    = bound_radius(c, c->rb_id[a]);
        for(int i = 0; i < 27; ++i)
        {
            if(nbl[i] == UINT32_MAX)
                continue;
            for(uint32_t k = c->cell_start[nbl[i]]; k < c->cell_start[nbl[i] + 1]; ++k)
            {
                const uint32_t b = c->sorted[k];
                if(b == (uint32_t)a)
                    continue;
                double d[3];
                sub3(c->tr + 12 * b + 9, c->tr + 12 * a + 9, d);
                if(norm3(d) - (ra + bound_radius(c, c->rb_id[b])) < 0.0)
                    ++total;
            }
        }
    }
    c->pair_off[n] = (uint32_t)total;
    if((st = ensure_pairs(c, total)) != GB_OK)
        return st;
    c->npairs = total;

    int64_t contacts = 0, ocontacts = 0, gcalls = 0, giters = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(c->threads) \
    reduction(+ : contacts, ocontacts, gcalls, giters)
    for(int64_t a = 0; a < n; ++a)
    {
        /* ComponentManagerCPU::detectCollisionAndComputeContactForcesParticles
           (ComponentManagerCPU.cpp:356-423) */
        const gb_rigid_body_desc*  rbA  = &c->rbs[c->rb_id[a]];
        const gb_rigid_body_props* prA  = &c->rbp[c->rb_id[a]];
        const double*              trA  = c->tr + 12 * a;
        double*                    F    = c->torce + 6 * a;
        double*                    Tq   = F + 3;
        body_view                  A;
        view_of(&A, rbA, prA, c->verts, cb);
        const uint32_t* nbl = c->nbr + 27 * (size_t)c->hash[a];
        int64_t         slot = c->pair_off[a];
        for(int i = 0; i < 27; ++i)
        {
            if(nbl[i] == UINT32_MAX)
                continue;
            for(uint32_t k = c->cell_start[nbl[i]]; k < c->cell_start[nbl[i] + 1]; ++k)
            {
                const uint32_t b = c->sorted[k];
                if(b == (uint32_t)a)
                    continue;
                const gb_rigid_body_desc*  rbB = &c->rbs[c->rb_id[b]];
                const gb_rigid_body_props* prB = &c->rbp[c->rb_id[b]];
                const double*              trB = c->tr + 12 * b;
                body_view                  B;
                view_of(&B, rbB, prB, c->verts, cb);
                double d[3];
                sub3(trB + 9, trA + 9, d);
                const int cand = norm3(d) - (A.rcirc + B.rcirc) < 0.0;
                or_contact ci;
                closest_points(&A, &B, trA, trB, variant, &ci);
                if(cand)
                {
                    c->pair_b[slot]       = b;
                    c->pair_ci[slot]      = ci;
                    c->pair_contact[slot] = ci.overlap < 0.0;
                    zero3(c->pair_xi + 3 * slot);
                    if(!(A.cv->type == GB_SPHERE && B.cv->type == GB_SPHERE))
                        ++gcalls;
                }
                if(ci.overlap < 0.0)
                {
                    const gb_contact_model* cm  = model_for(c, rbA->material, rbB->material);
                    const double*           v1  = c->kin + 6 * a;
                    const double*           v2  = c->kin + 6 * b;
                    double                  k1[3], k2[3], rv[3], rw[3];
                    if(!hist)
                    {
                        kin_at_point(v1, ci.pt, k1);
                        kin_at_point(v2, ci.pt, k2);
                        sub3(k1, k2, rv);
                        sub3(v1 + 3, v2 + 3, rw);
                        hooke_forces(cm, &ci, rv, rw, prA->mass, prB->mass, trA + 9, F, Tq);
                    }
                    else
                    {
                        double ra[3], rb[3];
                        sub3(ci.pt, trA + 9, ra);
                        sub3(ci.pt, trB + 9, rb);
                        kin_at_point(v1, ra, k1);
                        kin_at_point(v2, rb, k2);
                        sub3(k1, k2, rv);
                        const double* prev = hist_lookup(c, (uint32_t)a, b);
                        double        z[3] = {0, 0, 0};
                        history_forces(cm, &ci, rv, prA->mass, prB->mass, c->cfg.dt,
                                       prev ? prev : z, c->pair_xi + 3 * slot, trA + 9,
                                       F, Tq);
                    }
                    ++contacts;
                    if(result)
                        result[a] += 1;
                }
                if(cand)
                    ++slot;
            }
        }
        /* ComponentManagerCPU::detectCollisionAndComputeContactForcesObstacles
           (ComponentManagerCPU.cpp:301-351) */
        for(int32_t o = 0; o < c->nob; ++o)
        {
            body_view O;
            view_of(&O, &c->obs[o], &c->obp[o], NULL, cb);
            const double* trO = c->obs_tr + 12 * o;
            or_contact    ci;
            closest_points(&A, &O, trA, trO, variant, &ci);
            if(ci.overlap < 0.0)
            {
                const gb_contact_model* cm = model_for(c, rbA->material, c->obs[o].material);
                const double*           v1 = c->kin + 6 * a;
                const double*           vo = c->obs_vel + 6 * o;
                double                  k1[3], k2[3], rv[3], rw[3], ro[3];
                /* the wall's velocity at the contact point, v + w ^ (p - origin):
                   zero for the reference's walls at rest (ComponentManagerCPU.cpp:
                   326-336; NEW for moving walls) */
                sub3(ci.pt, trO + 9, ro);
                kin_at_point(vo, ro, k2);
                if(!hist)
                {
                    kin_at_point(v1, ci.pt, k1);
                    sub3(k1, k2, rv);
                    sub3(v1 + 3, vo + 3, rw);
                    hooke_forces(cm, &ci, rv, rw, prA->mass, c->obp[o].mass, trA + 9, F, Tq);
                }
                else
                {
                    /* wall history is not kept: walls use a fresh spring each step */
                    double ra[3], z[3] = {0, 0, 0}, xi[3];
                    sub3(ci.pt, trA + 9, ra);
                    kin_at_point(v1, ra, k1);
                    sub3(k1, k2, rv);
                    history_forces(cm, &ci, rv, prA->mass, c->obp[o].mass, c->cfg.dt, z,
                                   xi, trA + 9, F, Tq);
                }
                ++ocontacts;
            }
        }
    }
    if(hist)
    {
        /* the pair records of this step become the next step's history */
        free(c->hist_b);
        free(c->hist_xi);
        c->hist_b  = xcalloc(total, sizeof(uint32_t));
        c->hist_xi = xcalloc(total * 3, sizeof(double));
        memcpy(c->hist_off, c->pair_off, (size_t)(n + 1) * sizeof(uint32_t));
        memcpy(c->hist_b, c->pair_b, (size_t)total * sizeof(uint32_t));
        for(int64_t p = 0; p < total; ++p)
        {
            if(c->pair_contact[p])
                copy3(c->pair_xi + 3 * p, c->hist_xi + 3 * p);
            else
                zero3(c->hist_xi + 3 * p);
        }
        c->hist_n = total;
    }
    c->contacts          = contacts;
    c->obstacle_contacts = ocontacts;
    c->gjk_calls         = gcalls;
    c->gjk_iters         = giters;
    return st;
}

int or_add_external_forces(or_ctx* c)
{
    /* ComponentManagerCPU::addExternalForces (ComponentManagerCPU.cpp:448-460) */
    if(!c)
        return GB_E_INVALID_ARG;
    for(int32_t i = 0; i < c->n; ++i)
    {
        const double m = c->rbp[c->rb_id[i]].mass;
        double       g[3];
        scal3(m, c->cfg.gravity, g);
        add3(c->torce + 6 * i, g, c->torce + 6 * i);
    }
    return GB_OK;
}

int or_move_particles(or_ctx* c)
{
    /* ComponentManagerCPU::moveParticles (ComponentManagerCPU.cpp:465-500) */
    if(!c)
        return GB_E_INVALID_ARG;
    const int verlet = c->cfg.integrator == GB_VELOCITY_VERLET;
    const double h   = verlet && !c->verlet_started ? 0.5 * c->cfg.dt : c->cfg.dt;
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for(int32_t i = 0; i < c->n; ++i)
    {
        const gb_rigid_body_props* rb = &c->rbp[c->rb_id[i]];
        double                     torce[6];
        memcpy(torce, c->torce + 6 * i, sizeof(torce));
        memset(c->torce + 6 * i, 0, sizeof(torce)); /* Torce::reset */
        if(verlet)
            move_verlet(rb, c->cfg.dt, h, c->tr + 12 * i, c->kin + 6 * i, torce);
        else
            move_first_order(rb, c->cfg.dt, c->tr + 12 * i, c->kin + 6 * i, torce);
    }
    c->verlet_started = 1;
    c->steps_done++;
    return GB_OK;
}

int or_step(or_ctx* c, int32_t n_steps)
{
    /* GrainsCPU::simulate loop body (Grains/Base/src/GrainsCPU.cpp:55-66) */
    if(!c || n_steps < 0)
        return GB_E_INVALID_ARG;
    int worst = GB_OK;
    for(int32_t s = 0; s < n_steps; ++s)
    {
        int st = or_detect_collision_and_compute_contact_forces(c, NULL);
        if(st && st != GB_E_OUT_OF_DOMAIN)
            return st;
        if(st)
            worst = st;
        or_add_external_forces(c);
        or_move_particles(c);
    }
    return worst;
}

int or_get_stats(or_ctx* c, gb_stats* o)
{
    if(!c || !o)
        return GB_E_INVALID_ARG;
    memset(o, 0, sizeof(*o));
    o->steps_done        = c->steps_done;
    o->candidate_pairs   = c->npairs;
    o->contacts          = c->contacts;
    o->obstacle_contacts = c->obstacle_contacts;
    o->gjk_calls         = c->gjk_calls;
    o->gjk_iterations    = c->gjk_iters;
    o->status_flags      = c->status_flags;
    o->n_cells           = (int32_t)c->ncells;
    for(int k = 0; k < 3; ++k)
    {
        o->cells_per_dir[k] = (int32_t)c->dims[k];
        o->grid_max[k]      = c->lc_max[k];
    }
    uint32_t bits = 0;
    while(bits < 32 && ((uint64_t)1 << bits) < (uint64_t)c->ncells)
        ++bits;
    o->key_bits  = (int32_t)bits;
    o->cell_size = c->cell;
    return GB_OK;
}

int or_debug_dump(or_ctx* c, int32_t kind, void* out, int64_t capacity, int64_t* count)
{
    if(!c || !count)
        return GB_E_INVALID_ARG;
    if(!c->links_valid)
        return GB_E_NOT_READY;
    int64_t avail = 0;
    switch(kind)
    {
        case GB_DUMP_CELL_HASH:
            avail = c->n;
            if(out)
                memcpy(out, c->hash, (size_t)(avail < capacity ? avail : capacity) * 4);
            break;
        case GB_DUMP_SORTED_IDS:
            avail = c->n;
            if(out)
                memcpy(out, c->sorted, (size_t)(avail < capacity ? avail : capacity) * 4);
            break;
        case GB_DUMP_CELL_START:
            avail = (int64_t)c->ncells + 1;
            if(out)
                memcpy(out, c->cell_start, (size_t)(avail < capacity ? avail : capacity) * 4);
            break;
        case GB_DUMP_NEIGHBORS:
            avail = (int64_t)c->ncells * 27;
            if(out)
                memcpy(out, c->nbr, (size_t)(avail < capacity ? avail : capacity) * 4);
            break;
        case GB_DUMP_CANDIDATE_PAIRS:
        case GB_DUMP_CONTACT_PAIRS:
        case GB_DUMP_CONTACT_INFO:
        {
            uint32_t* o32 = (uint32_t*)out;
            double*   o64 = (double*)out;
            int64_t   w   = 0;
            for(int32_t a = 0; a < c->n; ++a)
                for(uint32_t p = c->pair_off[a]; p < c->pair_off[a + 1]; ++p)
                {
                    if(kind != GB_DUMP_CANDIDATE_PAIRS && !c->pair_contact[p])
                        continue;
                    if(kind == GB_DUMP_CONTACT_INFO)
                    {
                        if(out && 7 * w + 7 <= capacity)
                        {
                            memcpy(o64 + 7 * w, c->pair_ci[p].pt, 3 * sizeof(double));
                            memcpy(o64 + 7 * w + 3, c->pair_ci[p].vec, 3 * sizeof(double));
                            o64[7 * w + 6] = c->pair_ci[p].overlap;
                        }
                    }
                    else if(out && 2 * w + 2 <= capacity)
                    {
                        o32[2 * w]     = (uint32_t)a;
                        o32[2 * w + 1] = c->pair_b[p];
                    }
                    ++w;
                }
            avail = kind == GB_DUMP_CONTACT_INFO ? 7 * w : 2 * w;
            break;
        }
        default:
            return GB_E_INVALID_ARG;
    }
    *count = avail;
    return GB_OK;
}

/* ===========================================================================
 * Adjoint of one time step (NEW: the reference has no differentiation).
 *
 * Scope: spheres, the Hooke law with kr = 0 (normal spring-dashpot,
 * tangential viscous force capped by Coulomb friction), Rectangle walls,
 * gravity, first-order explicit integration, in FP64.  The step maps the
 * state s = (x, v, omega) of every particle to s' = Phi(s, theta), with
 * theta = (kn, en, etat, muc) per material-pair law; the set of contacts is
 * the one found at s (frozen for the step).  For spheres the contact
 * geometry (overlap, normal, point) is a closed-form function of the centres
 * (closest_spheres / closest_rectangle above), so this is the exact
 * derivative of the step wherever the contact set does not change.  The
 * orientation of a sphere does not enter its forces and is not carried.
 *
 * Layout of a state adjoint: 9 rows of n doubles (x, y, z of the position,
 * of the velocity, of the angular velocity).
 * ======================================================================== */
static double hooke_en_coef_grad(double en)
{
    /* d/den of log(en) / sqrt(pi^2 + log(en)^2) */
    const double L = log(en), s = OR_PI * OR_PI + L * L;
    return OR_PI * OR_PI / (s * sqrt(s)) / en;
}

/* Reverse of hooke_forces for one contact: given the gradients lf of the
   force and lt of the torque arm x f, the gradients of vec, the contact
   point, the arm, both bodies' velocities and the law's parameters. */
static void hooke_vjp(const gb_contact_model* cm, double avmass, double omega0,
                      const double vec[3], const double pt[3], const double arm[3],
                      const double vA[3], const double wA[3], const double vB[3],
                      const double wB[3], const double lf[3], const double lt[3],
                      double g_vec[3], double g_pt[3], double g_arm[3], double g_vA[3],
                      double g_wA[3], double g_vB[3], double g_wB[3], double g_law[4])
{
    /* forward (the operations of hooke_forces, in plain FP64) */
    const double np = norm3(vec);
    double       n[3], rel[3], t[3], c1[3], c2[3];
    scal3(1.0 / np, vec, n);
    cross3(wA, pt, c1);
    cross3(wB, pt, c2);
    for(int k = 0; k < 3; ++k)
        rel[k] = vA[k] + c1[k] - vB[k] - c2[k];
    const double rn = dot3(rel, n);
    double       vn[3], vt[3], th[3] = {0, 0, 0};
    scal3(rn, n, vn);
    sub3(rel, vn, vt);
    const double nvt = norm3(vt);
    if(nvt > OR_EPS)
        scal3(1.0 / nvt, vt, th);
    const double c  = hooke_muen(cm->en);
    double       FN[3];
    for(int k = 0; k < 3; ++k)
        FN[k] = cm->kn * vec[k] + 2.0 * omega0 * c * avmass * vn[k];
    const double nFN = norm3(FN);
    double       FT[3];
    scal3(-2.0 * cm->etat * avmass, vt, FT);
    const double fn = cm->muc * nFN, ft = norm3(FT);
    const int    capped = fn < ft;
    if(capped)
        scal3(-fn, th, FT);
    double f[3];
    add3(FN, FT, f);
    /* reverse */
    double gf[3], gFN[3], gvt[3] = {0, 0, 0}, gvn[3], grel[3], gn[3];
    cross3(lt, arm, t);
    add3(lf, t, gf);
    cross3(f, lt, g_arm);
    copy3(gf, gFN);
    double g_nFN = 0.0;
    if(capped)
    {
        const double tg = dot3(th, gf);
        g_law[3] += -nFN * tg;
        g_nFN = -cm->muc * tg;
        if(nvt > OR_EPS)
        {
            double gth[3];
            scal3(-fn, gf, gth);
            const double a = dot3(gth, th);
            for(int k = 0; k < 3; ++k)
                gvt[k] = (gth[k] - a * th[k]) / nvt;
        }
    }
    else
    {
        scal3(-2.0 * cm->etat * avmass, gf, gvt);
        g_law[2] += -2.0 * avmass * dot3(vt, gf);
    }
    if(nFN > 0.0)
        for(int k = 0; k < 3; ++k)
            gFN[k] += g_nFN * FN[k] / nFN;
    g_law[0] += dot3(vec, gFN) + omega0 / (2.0 * cm->kn) * 2.0 * c * avmass * dot3(vn, gFN);
    g_law[1] += 2.0 * omega0 * avmass * dot3(vn, gFN) * hooke_en_coef_grad(cm->en);
    scal3(cm->kn, gFN, g_vec);
    scal3(2.0 * omega0 * c * avmass, gFN, gvn);
    copy3(gvt, grel);
    sub3(gvn, gvt, gvn);
    const double ngvn = dot3(n, gvn);
    for(int k = 0; k < 3; ++k)
    {
        grel[k] += ngvn * n[k];
        gn[k] = rn * gvn[k] + ngvn * rel[k];
    }
    const double ngn = dot3(n, gn);
    for(int k = 0; k < 3; ++k)
        g_vec[k] += (gn[k] - ngn * n[k]) / np;
    copy3(grel, g_vA);
    scal3(-1.0, grel, g_vB);
    cross3(pt, grel, g_wA);
    scal3(-1.0, g_wA, g_wB);
    double dw[3];
    sub3(wA, wB, dw);
    cross3(grel, dw, g_pt);
}

static int adjoint_supported(const or_ctx* c)
{
    if(c->cfg.contact_law != GB_LAW_HOOKE || c->cfg.integrator != GB_FIRST_ORDER_EXPLICIT)
        return 0;
    for(int i = 0; i < c->nrb; ++i)
        if(c->rbs[i].convex.type != GB_SPHERE)
            return 0;
    for(int o = 0; o < c->nob; ++o)
        if(c->obs[o].convex.type != GB_RECTANGLE)
            return 0;
    const int nl = c->nmat * (c->nmat + 1) / 2;
    for(int l = 0; l < nl; ++l)
        if(c->cm[l].kr != 0.0)
            return 0;
    return 1;
}

static int law_index(int ma, int mb)
{
    const int s = ma < mb ? ma : mb, l = ma < mb ? mb : ma;
    return l * (l + 1) / 2 + s;
}

int or_adjoint_step(or_ctx* c, const double* adj_next, double* adj_prev, double* grad_laws)
{
    if(!c || !adj_next || !adj_prev || !grad_laws)
        return GB_E_INVALID_ARG;
    if(!adjoint_supported(c))
        return GB_E_UNSUPPORTED;
    const int    n  = c->n;
    const double dt = c->cfg.dt;
#define ADJ(r, i) adj_prev[(size_t)(r) * n + (i)]
#define NXT(r, i) adj_next[(size_t)(r) * n + (i)]
    /* integration: x' = x + dt v, v' = v + dt F / m, omega' = omega + dt T / I */
    double* lF = xcalloc((size_t)6 * n, sizeof(double));
    for(int i = 0; i < n; ++i)
    {
        const gb_rigid_body_props* rb = c->rbp + c->rb_id[i];
        for(int k = 0; k < 3; ++k)
        {
            ADJ(k, i)         = NXT(k, i);
            ADJ(3 + k, i)     = NXT(3 + k, i) + dt * NXT(k, i);
            ADJ(6 + k, i)     = NXT(6 + k, i);
            lF[6 * i + k]     = dt / rb->mass * NXT(3 + k, i);
            lF[6 * i + 3 + k] = dt * rb->inertia_inv[0] * NXT(6 + k, i);
        }
    }
    /* contacts at s, each on its first particle */
    for(int a = 0; a < n; ++a)
    {
        const gb_rigid_body_props* pa = c->rbp + c->rb_id[a];
        const double               rA = c->rbs[c->rb_id[a]].convex.p[0];
        const int                  ma = c->rbs[c->rb_id[a]].material;
        const double*              xa = c->tr + 12 * a + 9;
        double vA[3], wA[3], gx[3] = {0, 0, 0}, gv[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
        copy3(c->kin + 6 * a, vA);
        copy3(c->kin + 6 * a + 3, wA);
        const double* lf = lF + 6 * a;
        const double* lt = lF + 6 * a + 3;
        for(int b = 0; b < n; ++b)
        {
            if(b == a)
                continue;
            const gb_rigid_body_props* pb = c->rbp + c->rb_id[b];
            const double               rB = c->rbs[c->rb_id[b]].convex.p[0];
            const double*              xb = c->tr + 12 * b + 9;
            double                     d[3];
            sub3(xb, xa, d);
            const double dn = norm3(d), delta = dn - rA - rB;
            if(!(delta < 0.0))
                continue;
            double u[3], vec[3], pt[3], arm[3];
            scal3(1.0 / dn, d, u);
            scal3(delta, u, vec);
            for(int k = 0; k < 3; ++k)
                pt[k] = xa[k] + (rA + 0.5 * delta) * u[k];
            sub3(pt, xa, arm);
            const gb_contact_model* cm = c->cm + law_index(ma, c->rbs[c->rb_id[b]].material);
            const double            avm = pa->mass * pb->mass / (pa->mass + pb->mass);
            const double            w0  = sqrt(cm->kn / avm);
            double gvec[3], gpt[3], garm[3], gvA[3], gwA[3], gvB[3], gwB[3];
            hooke_vjp(cm, avm, w0, vec, pt, arm, vA, wA, c->kin + 6 * b, c->kin + 6 * b + 3, lf, lt,
                      gvec, gpt, garm, gvA, gwA, gvB, gwB,
                      grad_laws + 4 * law_index(ma, c->rbs[c->rb_id[b]].material));
            /* geometry: pt = xa + (rA + delta/2) u, vec = delta u, arm = pt - xa */
            for(int k = 0; k < 3; ++k)
            {
                gpt[k] += garm[k];
                gx[k] -= garm[k];
                gx[k] += gpt[k];
            }
            const double gdelta = 0.5 * dot3(u, gpt) + dot3(u, gvec);
            double       gu[3], gd[3];
            for(int k = 0; k < 3; ++k)
                gu[k] = (rA + 0.5 * delta) * gpt[k] + delta * gvec[k];
            const double ugu = dot3(u, gu);
            for(int k = 0; k < 3; ++k)
                gd[k] = (gu[k] - ugu * u[k]) / dn + gdelta * u[k];
            for(int k = 0; k < 3; ++k)
            {
                gx[k] -= gd[k];
                ADJ(k, b) += gd[k];
                gv[k] += gvA[k];
                gw[k] += gwA[k];
                ADJ(3 + k, b) += gvB[k];
                ADJ(6 + k, b) += gwB[k];
            }
        }
        for(int o = 0; o < c->nob; ++o)
        {
            const double* ot = c->obs_tr + 12 * o;
            double        rn[3] = {ot[2], ot[5], ot[8]}, e[3];
            sub3(xa, ot + 9, e);
            scal3(copysign(1.0, dot3(rn, e)), rn, rn);
            const double h = dot3(rn, e), s = h - rA;
            if(!(s < 0.0))
                continue;
            double vec[3], pt[3], arm[3];
            scal3(-s, rn, vec);
            for(int k = 0; k < 3; ++k)
                pt[k] = xa[k] - rA * rn[k] - 0.5 * s * rn[k];
            sub3(pt, xa, arm);
            const int               mo  = c->obs[o].material;
            const gb_contact_model* cm  = c->cm + law_index(ma, mo);
            const double            avm = 0.5 * pa->mass; /* obstacle mass 0: HookeContactForceModel's rule */
            const double            w0  = 2.0 * sqrt(cm->kn / avm);
            const double            z[3] = {0, 0, 0};
            double gvec[3], gpt[3], garm[3], gvA[3], gwA[3], gvB[3], gwB[3];
            hooke_vjp(cm, avm, w0, vec, pt, arm, vA, wA, z, z, lf, lt, gvec, gpt, garm, gvA, gwA,
                      gvB, gwB, grad_laws + 4 * law_index(ma, mo));
            /* pt = xa - rA rn - s rn / 2, vec = -s rn, s = rn . (xa - o) - rA */
            for(int k = 0; k < 3; ++k)
            {
                gpt[k] += garm[k];
                gx[k] += gpt[k] - garm[k];
            }
            const double gs = -dot3(rn, gvec) - 0.5 * dot3(rn, gpt);
            for(int k = 0; k < 3; ++k)
            {
                gx[k] += gs * rn[k];
                gv[k] += gvA[k];
                gw[k] += gwA[k];
            }
        }
        for(int k = 0; k < 3; ++k)
        {
            ADJ(k, a) += gx[k];
            ADJ(3 + k, a) += gv[k];
            ADJ(6 + k, a) += gw[k];
        }
    }
    free(lF);
#undef ADJ
#undef NXT
    return GB_OK;
}
