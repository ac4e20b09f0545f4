// gb_geom.cuh -- device rigid-body tables, support functions, OBB test and
// GJK with Johnson's sub-algorithm.
#pragma once

#include "gb_math.cuh"
#include "../../include/grains_b200.h"

namespace gb
{

// Shape part of a rigid body, as read by the narrow phase.  k[] caches the
// superquadric ratios and exponents that Superquadric::support recomputes
// on every call (Superquadric.cpp:169-205); each is the same IEEE value the
// reference computes inline.
template <typename St>
struct RBShape
{
    int32_t type;
    int32_t nverts;
    int64_t first_vert;
    St      p[5];
    St      k[8]; // b/a, c/a, c/b, 1/(n1-1), 1/(n2-1), (n1-n2)/(n2 (n1-1)), n1/n2, 1/n1
    St      crust;
    St      rcirc;
    St      bb[3];
    int32_t material;
    int32_t pad;
};

// Inertial part, as read by the per-particle kernel (RigidBody.hh:28-37),
// with the bounding box the obstacle mask needs: 16 values, one aligned
// record (64 B in FP32), so that a particle's body costs two 32-byte sectors.
template <typename St>
struct alignas(16 * sizeof(St)) RBInertia
{
    St mass;
    St I[6];
    St I1[6];
    St bb[3];
};

template <typename St>
struct Vert
{
    St x, y, z, w;
};

template <typename S>
struct Body
{
    int                      type;
    int                      nverts;
    const Vert<store_t<S>>*  verts;
    S                        p[5];
    S                        k[8];
    S                        crust, rcirc;
    V3<S>                    bb;
};

template <typename S>
GB_D Body<S> load_body(const RBShape<store_t<S>>* __restrict__ tab, uint32_t rb,
                       const Vert<store_t<S>>* __restrict__ verts)
{
    const RBShape<store_t<S>>* r = tab + rb;
    Body<S>                    b;
    b.type   = __ldg(&r->type);
    b.nverts = __ldg(&r->nverts);
    b.verts  = verts + __ldg(&r->first_vert);
#pragma unroll
    for(int i = 0; i < 5; ++i)
        b.p[i] = S(__ldg(&r->p[i]));
#pragma unroll
    for(int i = 0; i < 8; ++i)
        b.k[i] = S(__ldg(&r->k[i]));
    b.crust = S(__ldg(&r->crust));
    b.rcirc = S(__ldg(&r->rcirc));
    b.bb    = mk<S>(S(__ldg(&r->bb[0])), S(__ldg(&r->bb[1])), S(__ldg(&r->bb[2])));
    return b;
}

template <typename S>
GB_D S sgn(S x)
{
    // MiscMath.hh:68-72, returned as the scalar type
    return S(double((S(0.0) < x) - (x < S(0.0))));
}

// Superquadric::support for v.x != 0 in plain FP64: the reference's
// expressions with every power x^y written as 2^(y log2 x) and kept in the
// log domain between the steps.  The dependent chain falls from five pow
// calls and a division to three log2/exp2 pairs (pow is the longest-latency
// FP64 function); the values agree with pow's to a few ulps times
// |y log2 x|.  Zero y or z components give log2 0 = -inf and 2^-inf = 0, as
// pow(0, y) does.  Straight-line code, so that two calls interleave.
GB_D V3<double> support_sq_log(const Body<double>& b, const V3<double>& v)
{
    const double abvx = fabs(v.x), abvy = fabs(v.y), abvz = fabs(v.z);
    const double la = b.k[4] * log2(b.k[0] * abvy / abvx);              // log2 alpha
    const double lt = log2(1.0 + exp2(b.p[4] * la));                     // log2 temp
    const double lb = b.k[5] * lt + b.k[3] * log2(b.k[1] * abvz / abvx); // log2 beta
    const double xt = exp2(-b.k[7] * log2(exp2(b.k[6] * lt) + exp2(b.p[3] * lb)));
    return mk<double>(sgn(v.x) * b.p[0] * xt, sgn(v.y) * exp2(la) * b.p[1] * xt,
                      sgn(v.z) * exp2(lb) * b.p[2] * xt);
}

// Superquadric::support (Grains/Geometry/src/Superquadric.cpp:169-205)
template <typename S>
GB_D V3<S> support_sq(const Body<S>& b, const V3<S>& v)
{
    const S abvx = s_fabs(v.x), abvy = s_fabs(v.y), abvz = s_fabs(v.z);
    const S signx = sgn(v.x), signy = sgn(v.y), signz = sgn(v.z);
    const S one = S(1.0);
    if constexpr(std::is_same<S, double>::value)
    {
        if(abvx == 0.0)
        {
            if(abvy == 0.0)
                return mk<S>(0.0, 0.0, signz * b.p[2]);
            const double la = b.k[3] * log2(b.k[2] * abvz / abvy); // log2 alpha
            const double yt = exp2(-b.k[7] * log2(1.0 + exp2(b.p[3] * la)));
            return mk<S>(0.0, signy * b.p[1] * yt, signz * exp2(la) * b.p[2] * yt);
        }
        return support_sq_log(b, v);
    }
    if(abvx == S(0.0))
    {
        if(abvy == S(0.0))
            return mk<S>(S(0.0), S(0.0), signz * b.p[2]);
        const S alpha = s_pow(b.k[2] * abvz / abvy, b.k[3]);
        const S yt    = one / s_pow(one + s_pow(alpha, b.p[3]), b.k[7]);
        return mk<S>(S(0.0), signy * b.p[1] * yt, signz * alpha * b.p[2] * yt);
    }
    const S alpha = s_pow(b.k[0] * abvy / abvx, b.k[4]);
    const S temp  = one + s_pow(alpha, b.p[4]);
    const S gamma = s_pow(temp, b.k[5]);
    const S beta  = gamma * s_pow(b.k[1] * abvz / abvx, b.k[3]);
    const S xt    = one / s_pow(s_pow(temp, b.k[6]) + s_pow(beta, b.p[3]), b.k[7]);
    return mk<S>(signx * b.p[0] * xt, signy * alpha * b.p[1] * xt, signz * beta * b.p[2] * xt);
}

// NEW (no reference shape): argmax over the vertices, first index on ties.
template <typename S>
GB_D V3<S> support_poly(const Body<S>& b, const V3<S>& v)
{
    const Vert<store_t<S>>* __restrict__ pv = b.verts;
    Vert<store_t<S>> q0 = pv[0];
    V3<S>            best = mk<S>(S(q0.x), S(q0.y), S(q0.z));
    S                bd   = dot(best, v);
    for(int i = 1; i < b.nverts; ++i)
    {
        Vert<store_t<S>> q = pv[i];
        V3<S>            c = mk<S>(S(q.x), S(q.y), S(q.z));
        S                d = dot(c, v);
        if(d > bd)
        {
            bd   = d;
            best = c;
        }
    }
    return best;
}

template <typename S>
GB_D V3<S> support(const Body<S>& b, const V3<S>& v)
{
    switch(b.type)
    {
        case GB_SUPERQUADRIC:
            return support_sq(b, v);
        case GB_POLYHEDRON:
            return support_poly(b, v);
        case GB_BOX: // Box::support (Box.cpp:129-134)
            return mk<S>(v.x < S(0.0) ? -b.p[0] : b.p[0], v.y < S(0.0) ? -b.p[1] : b.p[1],
                         v.z < S(0.0) ? -b.p[2] : b.p[2]);
        case GB_SPHERE: // Sphere::support = r v/|v| (Sphere.cpp:111)
        {
            const S n = norm(v);
            return b.p[0] * mk<S>(v.x / n, v.y / n, v.z / n);
        }
        case GB_RECTANGLE: // Rectangle::support (Rectangle.cpp:115-121)
            return mk<S>(v.x < S(0.0) ? -b.p[0] : b.p[0], v.y < S(0.0) ? -b.p[1] : b.p[1],
                         S(0.0));
        default:
            return mk<S>(S(0.0), S(0.0), S(0.0));
    }
}

// Superquadric::support in FP32 in the log domain (the form of
// support_sq_log), for the mixed mode's FP32 stages (the first-iteration test
// and the FP32 GJK), which only certify separation with a margin of 1e-4 of
// the bounding radii.  The hardware approximations of log2 and of the
// quotient (a few ulp; 2^-21.4 absolute for log2 near 1) and exp2f's 2 ulp
// move a support point by ~1e-6 of its size, some 1e-9 m, far inside that
// margin.  FP32
// exponents overflow where FP64 ones do not (2^e for e > 128): a direction
// whose chain would exceed 2^100 at any step, or with v.x = 0, gives NaN,
// which sends the pair to the FP64 solve.
GB_D V3<float> support_sq_log32(const Body<float>& b, const V3<float>& v)
{
    const float abvx = fabsf(v.x), abvy = fabsf(v.y), abvz = fabsf(v.z);
    const float la = b.k[4] * __log2f(__fdividef(b.k[0] * abvy, abvx));
    const float ea = b.p[4] * la;
    const float lt = __log2f(1.0f + exp2f(ea));
    const float lb = b.k[5] * lt + b.k[3] * __log2f(__fdividef(b.k[1] * abvz, abvx));
    const float e1 = b.k[6] * lt, e2 = b.p[3] * lb;
    if(!(abvx > 0.0f) || !(ea <= 100.0f) || !(e1 <= 100.0f) || !(e2 <= 100.0f)
       || !(la <= 100.0f) || !(lb <= 100.0f))
        return mk<float>(NAN, NAN, NAN);
    const float xt = exp2f(-b.k[7] * __log2f(exp2f(e1) + exp2f(e2)));
    return mk<float>(sgn(v.x) * b.p[0] * xt, sgn(v.y) * exp2f(la) * b.p[1] * xt,
                     sgn(v.z) * exp2f(lb) * b.p[2] * xt);
}

// The support used by the first-iteration test of GJK: the log-domain form
// for FP32 superquadrics, support() otherwise.
template <typename S>
GB_D V3<S> support_first(const Body<S>& b, const V3<S>& v)
{
    if constexpr(std::is_same<S, float>::value)
        if(b.type == GB_SUPERQUADRIC)
            return support_sq_log32(b, v);
    return support(b, v);
}

// A GJK variant flag: the solve runs on two adjacent lanes, which compute
// the same iterates; the even lane evaluates A's support and the odd lane B's,
// in parallel, and they exchange them by shuffles.  (A support is the longest
// dependent chain of an iteration: ~2,000 cycles for an FP64 superquadric.)
constexpr int kGjkPaired = 8;

GB_D float lane_shfl(unsigned mask, float v, unsigned src)
{
    return __shfl_sync(mask, v, src);
}
GB_D double lane_shfl(unsigned mask, double v, unsigned src)
{
    return __shfl_sync(mask, v, src);
}
GB_D dstrict lane_shfl(unsigned mask, dstrict v, unsigned src)
{
    return dstrict(__shfl_sync(mask, v.v, src));
}

// The supports of A along va and of B along vb, the results of two support
// calls.  PAIRED: one per lane of a lane pair (kGjkPaired).  Otherwise two
// FP64 superquadrics take the straight-line log-domain form side by side
// (the rare v.x = 0 direction is redone on the general path).
template <bool PAIRED = false, typename S>
GB_D void support2(const Body<S>& A, const V3<S>& va, const Body<S>& B, const V3<S>& vb,
                   V3<S>& pa, V3<S>& pb)
{
    if constexpr(PAIRED)
    {
        const unsigned lane   = threadIdx.x & 31u;
        const unsigned even   = lane & ~1u;
        const unsigned mask   = 3u << even;
        const bool     second = (lane & 1u) != 0u;
        // field by field, so that the two lanes select data, not code paths
        Body<S> X;
        X.type   = second ? B.type : A.type;
        X.nverts = second ? B.nverts : A.nverts;
        X.verts  = second ? B.verts : A.verts;
#pragma unroll
        for(int i = 0; i < 5; ++i)
            X.p[i] = second ? B.p[i] : A.p[i];
#pragma unroll
        for(int i = 0; i < 8; ++i)
            X.k[i] = second ? B.k[i] : A.k[i];
        X.crust = second ? B.crust : A.crust;
        X.rcirc = second ? B.rcirc : A.rcirc;
        X.bb    = second ? B.bb : A.bb;
        const V3<S> r = support(X, second ? vb : va);
        pa = mk<S>(lane_shfl(mask, r.x, even), lane_shfl(mask, r.y, even),
                   lane_shfl(mask, r.z, even));
        pb = mk<S>(lane_shfl(mask, r.x, even + 1u), lane_shfl(mask, r.y, even + 1u),
                   lane_shfl(mask, r.z, even + 1u));
        return;
    }
    if constexpr(std::is_same<S, double>::value)
        if(A.type == GB_SUPERQUADRIC && B.type == GB_SUPERQUADRIC)
        {
            pa = support_sq_log(A, va);
            pb = support_sq_log(B, vb);
            if(va.x == 0.0)
                pa = support_sq(A, va);
            if(vb.x == 0.0)
                pb = support_sq(B, vb);
            return;
        }
    pa = support(A, va);
    pb = support(B, vb);
}

// intersectOrientedBoundingBox (Grains/CollisionDetection/src/OBB.cpp:32-94):
// `cen` is B's origin relative to A's in world axes, RA/RB the bases.
template <typename S>
GB_D bool obb_overlap(const V3<S>& a, const V3<S>& b, const M3<S>& RA, const M3<S>& RB,
                      const V3<S>& d)
{
    const M3<S> oriT = transpose(RA);
    const V3<S> cen  = mul(oriT, d);
    const M3<S> ori  = mul(oriT, RB);
    M3<S>       oa;
#pragma unroll
    for(int i = 0; i < 9; ++i)
        oa.m[i] = s_fabs(ori.m[i]) + k_loweps<S>();
    const S A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, c[3] = {cen.x, cen.y, cen.z};
#define O_(i, j) ori.m[3 * (i) + (j)]
#define OA_(i, j) oa.m[3 * (i) + (j)]
#pragma unroll
    for(int i = 0; i < 3; ++i)
        if(s_fabs(c[i]) > (A[i] + B[0] * OA_(i, 0) + B[1] * OA_(i, 1) + B[2] * OA_(i, 2)))
            return false;
#pragma unroll
    for(int i = 0; i < 3; ++i)
        if(s_fabs(c[0] * O_(0, i) + c[1] * O_(1, i) + c[2] * O_(2, i))
           > (B[i] + A[0] * OA_(0, i) + A[1] * OA_(1, i) + A[2] * OA_(2, i)))
            return false;
#pragma unroll
    for(int j = 0; j < 3; ++j)
#pragma unroll
        for(int i = 0; i < 3; ++i) // TESTCASE3(i, j), j outer as in the reference
            if(s_fabs(c[(i + 2) % 3] * O_((i + 1) % 3, j) - c[(i + 1) % 3] * O_((i + 2) % 3, j))
               > (A[(i + 1) % 3] * OA_((i + 2) % 3, j) + A[(i + 2) % 3] * OA_((i + 1) % 3, j)
                  + B[(j + 1) % 3] * OA_(i, (j + 2) % 3) + B[(j + 2) % 3] * OA_(i, (j + 1) % 3)))
                return false;
#undef O_
#undef OA_
    return true;
}

// ---------------------------------------------------------------------------
// GJK with Johnson's distance sub-algorithm and cached sub-determinants
// (Grains/CollisionDetection/src/GJK_JH.cpp:9-391).  One thread per pair.
template <typename S>
struct JH
{
    S     det[16][4];
    S     dp[4][4];
    V3<S> y[4];

    GB_D void compute_det(unsigned bits, unsigned last, unsigned last_bit, unsigned all_bits)
    {
        // computeDet (GJK_JH.cpp:9-63)
        for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
            if(bits & bit)
                dp[i][last] = dp[last][i] = dot(y[i], y[last]);
        dp[last][last] = dot(y[last], y[last]);
        det[last_bit][last] = S(1.0);
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

    GB_D bool valid(unsigned s, unsigned all_bits) const
    {
        for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
        {
            if(all_bits & bit)
            {
                if(s & bit)
                {
                    if(det[s][i] <= k_eps<S>())
                        return false;
                }
                else if(det[s | bit][i] > S(0.0))
                    return false;
            }
        }
        return true;
    }

    GB_D V3<S> compute_vector(unsigned bits) const
    {
        S     sum = S(0.0);
        V3<S> v   = zero3<S>();
        for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
            if(bits & bit)
            {
                sum = sum + det[bits][i];
                v   = v + det[bits][i] * y[i];
            }
        return (S(1.0) / sum) * v;
    }

    GB_D bool proper(unsigned s) const
    {
        for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
            if((s & bit) && det[s][i] <= k_eps<S>())
                return false;
        return true;
    }

    GB_D bool closest(unsigned& bits, unsigned last, unsigned last_bit, unsigned all_bits,
                      V3<S>& v)
    {
        compute_det(bits, last, last_bit, all_bits);
        for(unsigned s = bits; s; --s)
            if((s & bits) == s && valid(s | last_bit, all_bits))
            {
                bits = s | last_bit;
                v    = compute_vector(bits);
                return true;
            }
        if(valid(last_bit, all_bits))
        {
            bits = last_bit;
            v    = y[last];
            return true;
        }
        // backup procedure (GJK_JH.cpp:173-193)
        S min_dist2 = S(INFINITY);
        for(unsigned s = all_bits; s; --s)
            if((s & all_bits) == s && proper(s))
            {
                V3<S> u     = compute_vector(s);
                S     dist2 = norm2(u);
                if(dist2 < min_dist2)
                {
                    min_dist2 = dist2;
                    bits      = s;
                    v         = u;
                }
            }
        return false;
    }

    GB_D bool degenerate(unsigned all_bits, const V3<S>& w) const
    {
        for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
            if((all_bits & bit) && eq3(y[i], w))
                return true;
        return false;
    }
};

template <typename S>
struct GjkResult
{
    S        dist;
    S        lower;  // the optimality-gap lower bound mu on the distance
    V3<S>    pa, pb; // closest points in A's and B's local frames
    int      iters;
};

// computeClosestPoints_GJK_JH (GJK_JH.cpp:310-391), in A's frame with b2a.
// `max_iter` caps the iterations (the reference's cap is 1000).
template <typename S, bool PAIRED = false>
GB_D GjkResult<S> gjk_jh(const Body<S>& A, const Body<S>& B, const Tr<S>& b2a,
                         int max_iter = 1000)
{
    unsigned bits = 0, last = 0, last_bit = 0, all_bits = 0;
    V3<S>    p[4], q[4];
    JH<S>    jh;
#pragma unroll
    for(int i = 0; i < 16; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j)
            jh.det[i][j] = S(0.0);
#pragma unroll
    for(int i = 0; i < 4; ++i)
    {
#pragma unroll
        for(int j = 0; j < 4; ++j)
            jh.dp[i][j] = S(0.0);
        p[i] = q[i] = jh.y[i] = zero3<S>();
    }
    S       mu = S(0.0);
    int     num_iterations = 0;
    const S rel_error      = k_loweps<S>();
    const S abs_error      = S(1.e-4) * rel_error;

    V3<S> s0A, s0B;
    support2<PAIRED>(A, zero3<S>(), B, zero3<S>(), s0A, s0B);
    V3<S> v    = s0A - apply(b2a, s0B);
    V3<S> w    = v;
    S     dist = norm(v);
    while(bits < 15 && dist > k_higheps<S>() && num_iterations < max_iter)
    {
        last     = 0;
        last_bit = 1;
        while(bits & last_bit)
        {
            ++last;
            last_bit <<= 1;
        }
        support2<PAIRED>(A, -v, B, mul_t(b2a.R, v), p[last], q[last]);
        w       = p[last] - apply(b2a, q[last]);
        const S g = dot(v, w) / dist;
        if(mu < g)
            mu = g;
        if(dist - mu <= dist * rel_error || mu < abs_error)
            break;
        if(jh.degenerate(all_bits, w))
            break;
        jh.y[last] = w;
        all_bits   = bits | last_bit;
        ++num_iterations;
        if(!jh.closest(bits, last, last_bit, all_bits, v))
            break;
        dist = norm(v);
    }
    // computePoints (GJK_JH.cpp:108-130)
    GjkResult<S> r;
    S            sum = S(0.0);
    r.pa             = zero3<S>();
    r.pb             = zero3<S>();
    for(unsigned i = 0, bit = 1; i < 4; ++i, bit <<= 1)
        if(bits & bit)
        {
            sum  = sum + jh.det[bits][i];
            r.pa = r.pa + jh.det[bits][i] * p[i];
            r.pb = r.pb + jh.det[bits][i] * q[i];
        }
    const S s = S(1.0) / sum;
    r.pa      = s * r.pa;
    r.pb      = s * r.pb;
    r.dist    = dist;
    r.lower   = mu;
    r.iters   = num_iterations;
    return r;
}

// ---- signed-volume sub-algorithm (GJK_AY.cpp:15-368, Montanari et al. 2017) --
template <typename S>
GB_D S comp(const V3<S>& v, unsigned i)
{
    return i == 0 ? v.x : (i == 1 ? v.y : v.z);
}

template <typename S>
GB_D unsigned sv_same_sign(S a, S b)
{
    return (unsigned)(!((a > S(0.0)) ^ (b > S(0.0)))); // compareSigns (GJK_AY.cpp:8-12)
}

// sum of lambda_i y_i over the used points (computeVector, GJK_AY.cpp:304-316)
template <typename S>
GB_D V3<S> sv_point(const V3<S> y[4], unsigned used, const S lambdas[4])
{
    V3<S> o = zero3<S>();
#pragma unroll
    for(unsigned i = 0; i < 4; ++i)
        if(used & (1u << i))
            o = o + lambdas[i] * y[i];
    return o;
}

// s1d (GJK_AY.cpp:15-84)
template <typename S>
GB_D void sv_s1d(const V3<S> y[4], unsigned& bits, S lambdas[4])
{
    bool     s1_set = false;
    unsigned i1 = 0, i2 = 0;
    for(unsigned i = 0; i < 4; ++i)
        if(bits & (1u << i))
        {
            if(s1_set)
            {
                i2 = i;
                break;
            }
            i1     = i;
            s1_set = true;
        }
    const V3<S> t      = y[i2] - y[i1];
    unsigned    I      = 0;
    S           neg_tI = -t.x;
    if(s_fabs(t.y) > s_fabs(neg_tI))
    {
        I      = 1;
        neg_tI = -t.y;
    }
    if(s_fabs(t.z) > s_fabs(neg_tI))
    {
        I      = 2;
        neg_tI = -t.z;
    }
    const S pI  = dot(y[i2], t) / norm2(t) * neg_tI + comp(y[i2], I);
    const S C0  = -comp(y[i2], I) + pI, C1 = comp(y[i1], I) - pI;
    const unsigned sc0 = sv_same_sign(neg_tI, C0), sc1 = sv_same_sign(neg_tI, C1);
    if(sc0 + sc1 == 2)
    {
        lambdas[i1] = C0 / neg_tI;
        lambdas[i2] = C1 / neg_tI;
    }
    else if(sc0)
    {
        bits &= ~(1u << i2);
        lambdas[i1] = S(1.0);
    }
    else
    {
        bits &= ~(1u << i1);
        lambdas[i2] = S(1.0);
    }
}

// s2d (GJK_AY.cpp:87-212)
template <typename S>
GB_D void sv_s2d(const V3<S> y[4], unsigned& bits, S lambdas[4])
{
    unsigned counter = 0, i0 = 0, i1 = 0, i2 = 0;
    for(unsigned i = 0; i < 4; ++i)
        if(bits & (1u << i))
        {
            if(counter == 0)
                i0 = i;
            else if(counter == 1)
                i1 = i;
            else
                i2 = i;
            counter += 1;
        }
    const V3<S> n  = cross(y[i1] - y[i0], y[i2] - y[i0]);
    const V3<S> p0 = (dot(y[i0], n) / norm2(n)) * n;
    const V3<S>& Y0 = y[i0];
    const V3<S>& Y1 = y[i1];
    const V3<S>& Y2 = y[i2];
    unsigned     ix = 1, iy = 2;
    S mu_max = (Y1.y * Y2.z + Y0.y * Y1.z + Y2.y * Y0.z - Y1.y * Y0.z - Y2.y * Y1.z - Y0.y * Y2.z);
    S mu     = (Y1.z * Y0.x + Y2.z * Y1.x + Y0.z * Y2.x - Y1.z * Y2.x - Y0.z * Y1.x - Y2.z * Y0.x);
    if(s_fabs(mu) > s_fabs(mu_max))
    {
        mu_max = mu;
        ix     = 0;
    }
    mu = (Y1.x * Y2.y + Y0.x * Y1.y + Y2.x * Y0.y - Y1.x * Y0.y - Y2.x * Y1.y - Y0.x * Y2.y);
    if(s_fabs(mu) > s_fabs(mu_max))
    {
        mu_max = mu;
        ix     = 0;
        iy     = 1;
    }
    const S px = comp(p0, ix), py = comp(p0, iy);
    const S y0x = comp(Y0, ix), y0y = comp(Y0, iy), y1x = comp(Y1, ix), y1y = comp(Y1, iy);
    const S y2x = comp(Y2, ix), y2y = comp(Y2, iy);
    S       C[3];
    C[0] = (px * y1y + py * y2x + y1x * y2y - px * y2y - py * y1x - y2x * y1y);
    C[1] = (px * y2y + py * y0x + y2x * y0y - px * y0y - py * y2x - y0x * y2y);
    C[2] = (px * y0y + py * y1x + y0x * y1y - px * y1y - py * y0x - y1x * y0y);
    const unsigned sc[3] = {sv_same_sign(mu_max, C[0]), sv_same_sign(mu_max, C[1]),
                            sv_same_sign(mu_max, C[2])};
    if(sc[0] + sc[1] + sc[2] == 3)
    {
        lambdas[i0] = C[0] / mu_max;
        lambdas[i1] = C[1] / mu_max;
        lambdas[i2] = C[2] / mu_max;
        return;
    }
    S              d        = S(100000.0);
    unsigned       new_bits = 0;
    const unsigned idx[3]   = {i0, i1, i2};
    for(unsigned j = 0; j < 3; ++j)
        if(!sc[j])
        {
            unsigned new_used       = bits & ~(1u << idx[j]);
            S        new_lambdas[4] = {S(0.0), S(0.0), S(0.0), S(0.0)};
            sv_s1d(y, new_used, new_lambdas);
            const V3<S> np     = sv_point(y, new_used, new_lambdas);
            const S     d_star = dot(np, np);
            if(d_star < d)
            {
                new_bits = new_used;
                d        = d_star;
                for(unsigned i = 0; i < 4; ++i)
                    lambdas[i] = new_lambdas[i];
            }
        }
    bits = new_bits;
}

// s3d (GJK_AY.cpp:215-301)
template <typename S>
GB_D void sv_s3d(const V3<S> y[4], unsigned& bits, S lambdas[4])
{
    S C[4];
    C[0] = y[3].x * y[2].y * y[1].z + y[2].x * y[1].y * y[3].z + y[1].x * y[3].y * y[2].z
           - y[1].x * y[2].y * y[3].z - y[2].x * y[3].y * y[1].z - y[3].x * y[1].y * y[2].z;
    C[1] = y[0].x * y[2].y * y[3].z + y[2].x * y[3].y * y[0].z + y[3].x * y[0].y * y[2].z
           - y[3].x * y[2].y * y[0].z - y[2].x * y[0].y * y[3].z - y[0].x * y[3].y * y[2].z;
    C[2] = y[3].x * y[1].y * y[0].z + y[1].x * y[0].y * y[3].z + y[0].x * y[3].y * y[1].z
           - y[0].x * y[1].y * y[3].z - y[1].x * y[3].y * y[0].z - y[3].x * y[0].y * y[1].z;
    C[3] = y[0].x * y[1].y * y[2].z + y[1].x * y[2].y * y[0].z + y[2].x * y[0].y * y[1].z
           - y[2].x * y[1].y * y[0].z - y[1].x * y[0].y * y[2].z - y[0].x * y[2].y * y[1].z;
    const S  dM = C[0] + C[1] + C[2] + C[3];
    unsigned sc[4];
#pragma unroll
    for(int i = 0; i < 4; ++i)
        sc[i] = sv_same_sign(dM, C[i]);
    if(sc[0] + sc[1] + sc[2] + sc[3] == 4)
    {
#pragma unroll
        for(int i = 0; i < 4; ++i)
            lambdas[i] = C[i] / dM;
        return;
    }
    S        d        = S(100000.0);
    unsigned new_bits = 0;
    for(unsigned j = 0; j < 4; ++j)
        if(!sc[j])
        {
            unsigned new_used       = bits & ~(1u << j);
            S        new_lambdas[4] = {S(0.0), S(0.0), S(0.0), S(0.0)};
            sv_s2d(y, new_used, new_lambdas);
            const V3<S> np     = sv_point(y, new_used, new_lambdas);
            const S     d_star = dot(np, np);
            if(d_star < d)
            {
                new_bits = new_used;
                d        = d_star;
                for(unsigned i = 0; i < 4; ++i)
                    lambdas[i] = new_lambdas[i];
            }
        }
    bits = new_bits;
}

// sv_subalgorithm (GJK_AY.cpp:340-368): new simplex, weights and closest point
template <typename S>
GB_D V3<S> sv_subalgorithm(const V3<S> y[4], unsigned& bits, S lambdas[4])
{
    unsigned num_used = 0;
#pragma unroll
    for(unsigned i = 0; i < 4; ++i)
        num_used += (bits >> i) & 1u;
    if(num_used == 1)
    {
        for(unsigned i = 0; i < 4; ++i)
            if(bits & (1u << i))
                lambdas[i] = S(1.0);
    }
    else if(num_used == 2)
        sv_s1d(y, bits, lambdas);
    else if(num_used == 3)
        sv_s2d(y, bits, lambdas);
    else
        sv_s3d(y, bits, lambdas);
    return sv_point(y, bits, lambdas);
}

// w equal to a vertex of the simplex `bits` (degenerate, GJK_AY.cpp:373-386)
template <typename S>
GB_D bool sv_degenerate(unsigned bits, const V3<S> y[4], const V3<S>& w)
{
    for(unsigned i = 0; i < 4; ++i)
        if((bits & (1u << i)) && y[i].x == w.x && y[i].y == w.y && y[i].z == w.z)
            return true;
    return false;
}

// GJK with the signed-volume sub-algorithm; NESTEROV: the support direction
// follows the momentum average of Montaut et al. (RSS 2022, Algorithm 2),
// with GJK_AY's gap test redone along x_k (see oracle's gjk_nesterov):
//   y_k = delta_k x_k + (1 - delta_k) s_{k-1},   delta_k = (k + 1)/(k + 3),
//   d_k = delta_k d_{k-1}/|d_{k-1}| + (1 - delta_k) y_k/|y_k|.
// Without NESTEROV it is computeClosestPoints_GJK_AY (GJK_AY.cpp:392-469).
template <typename S, bool NESTEROV, bool PAIRED = false>
GB_D GjkResult<S> gjk_sv(const Body<S>& A, const Body<S>& B, const Tr<S>& b2a)
{
    unsigned bits = 0, last = 0;
    V3<S>    p[4], q[4], y[4];
    S        lambdas[4] = {S(0.0), S(0.0), S(0.0), S(0.0)};
#pragma unroll
    for(int i = 0; i < 4; ++i)
        p[i] = q[i] = y[i] = zero3<S>();
    int     num_iterations = 0;
    bool    momentum       = NESTEROV;
    const S rel_error      = k_loweps<S>();
    const S abs_error      = S(1.e-4) * rel_error;
    V3<S>   s0A, s0B;
    support2<PAIRED>(A, zero3<S>(), B, zero3<S>(), s0A, s0B);
    V3<S>   v = s0A - apply(b2a, s0B);
    V3<S>   w = v, d = v, s_prev = v;
    S       dist = norm(v);
    while(bits < 15 && dist > k_higheps<S>() && num_iterations < 1000)
    {
        for(unsigned k = 0; k < 4; ++k)
            if(!(bits & (1u << k)))
            {
                last = k;
                break;
            }
        if constexpr(NESTEROV)
        {
            if(momentum)
            {
                const S     kk    = S((double)num_iterations);
                const S     delta = (kk + S(1.0)) / (kk + S(3.0));
                const S     om    = S(1.0) - delta;
                const V3<S> yk    = mk<S>(delta * v.x + om * s_prev.x, delta * v.y + om * s_prev.y,
                                       delta * v.z + om * s_prev.z);
                const S     ny = norm(yk), nd = norm(d);
                if(ny > k_higheps<S>() && nd > k_higheps<S>())
                    d = mk<S>(delta * (d.x / nd) + om * (yk.x / ny),
                              delta * (d.y / nd) + om * (yk.y / ny),
                              delta * (d.z / nd) + om * (yk.z / ny));
                else
                {
                    momentum = false;
                    d        = v;
                }
            }
            else
                d = v;
        }
        else
            d = v;
        support2<PAIRED>(A, -d, B, mul_t(b2a.R, d), p[last], q[last]);
        w         = p[last] - apply(b2a, q[last]);
        const S mu = dist - dot(v, w) / dist;
        if(mu < dist * rel_error || mu < abs_error || sv_degenerate(bits, y, w))
        {
            if(!momentum)
                break;
            momentum = false; // not a certified gap: redo this iteration along x_k
            continue;
        }
        y[last] = w;
        bits |= 1u << last;
        ++num_iterations;
        v    = sv_subalgorithm(y, bits, lambdas);
        dist = norm(v);
        s_prev = w;
    }
    // computePoints (GJK_AY.cpp:319-337)
    GjkResult<S> r;
    r.pa = zero3<S>();
    r.pb = zero3<S>();
    for(unsigned i = 0; i < 4; ++i)
        if(bits & (1u << i))
        {
            r.pa = r.pa + lambdas[i] * p[i];
            r.pb = r.pb + lambdas[i] * q[i];
        }
    r.dist  = dist;
    r.lower = S(0.0);
    r.iters = num_iterations;
    return r;
}

// the GJK of a variant (GB_GJK_JH | GB_GJK_SV | GB_GJK_NESTEROV), optionally
// with kGjkPaired
template <int VAR, typename S>
GB_D GjkResult<S> gjk(const Body<S>& A, const Body<S>& B, const Tr<S>& b2a)
{
    constexpr bool PAIRED = (VAR & kGjkPaired) != 0;
    constexpr int  KIND   = VAR & ~kGjkPaired;
    if constexpr(KIND == GB_GJK_SV)
        return gjk_sv<S, false, PAIRED>(A, B, b2a);
    else if constexpr(KIND == GB_GJK_NESTEROV)
        return gjk_sv<S, true, PAIRED>(A, B, b2a);
    else
        return gjk_jh<S, PAIRED>(A, B, b2a);
}

} // namespace gb
