// gb_adjoint.cuh -- reverse-mode derivative of one time step (no counterpart
// in the reference).
//
// Scope: spheres, the Hooke law with kr = 0, Rectangle walls, gravity,
// first-order explicit integration, FP64 state.  The step maps
// s = (x, v, omega) to s' = Phi(s, theta), theta = (kn, en, etat, muc) per
// material-pair law, over the contacts found at s.  For spheres the contact
// geometry is closed-form in the centres, so the kernels compute the exact
// vector-Jacobian product of the step wherever the contact set does not
// change.  State adjoints are 9 rows of n doubles: position, velocity,
// angular velocity (x, y, z each).
//
// Deterministic: thread i gathers every contribution to particle i -- from
// its own ordered pairs (i, j) and, recomputed, from the pairs (j, i) that
// act on j -- and the law gradients are reduced in a fixed order.
#pragma once

#include "gb_step.cuh"

namespace gb
{

constexpr int kAdjMaxLaws = 8;

struct AdjLaw
{
    double kn, en, etat, muc;
    double c;     // log(en) / sqrt(pi^2 + log(en)^2), HookeContactForceModel's m_muen
    double dc_en; // dc / den
};

struct AdjLaws
{
    AdjLaw l[kAdjMaxLaws];
    int    n;
};

GB_D int adj_law_index(int ma, int mb)
{
    const int s = ma < mb ? ma : mb, l = ma < mb ? mb : ma;
    return l * (l + 1) / 2 + s;
}

GB_D V3<double> ld3(double* const a[3], uint32_t i)
{
    return mk<double>(a[0][i], a[1][i], a[2][i]);
}

// Reverse of the Hooke law (HookeContactForceModel.cpp:91-186, kr = 0) for a
// contact given by its vector `vec` (overlap times the unit normal), point
// `pt` and torque arm: from the gradients lf of the force and lt of the torque
// arm x f, the gradients of vec, pt, arm, both bodies' velocities, and of the
// law's parameters (added to g_law[4]).
GB_D void hooke_vjp(const AdjLaw& L, double avmass, double omega0, const V3<double>& vec,
                    const V3<double>& pt, const V3<double>& arm, const V3<double>& vA,
                    const V3<double>& wA, const V3<double>& vB, const V3<double>& wB,
                    const V3<double>& lf, const V3<double>& lt, V3<double>& g_vec,
                    V3<double>& g_pt, V3<double>& g_arm, V3<double>& g_vA, V3<double>& g_wA,
                    V3<double>& g_vB, V3<double>& g_wB, double g_law[4])
{
    const double      np  = norm(vec);
    const V3<double>  n   = (1.0 / np) * vec;
    const V3<double>  rel = (vA + cross(wA, pt)) - (vB + cross(wB, pt));
    const double      rn  = dot(rel, n);
    const V3<double>  vn  = rn * n;
    const V3<double>  vt  = rel - vn;
    const double      nvt = norm(vt);
    const V3<double>  th  = nvt > 1e-10 ? (1.0 / nvt) * vt : zero3<double>();
    const V3<double>  FN  = L.kn * vec + (2.0 * omega0 * L.c * avmass) * vn;
    const double      nFN = norm(FN);
    V3<double>        FT  = (-2.0 * L.etat * avmass) * vt;
    const double      fn = L.muc * nFN, ft = norm(FT);
    const bool        capped = fn < ft;
    if(capped)
        FT = (-fn) * th;
    const V3<double> f  = FN + FT;
    const V3<double> gf = lf + cross(lt, arm);
    g_arm               = cross(f, lt);
    V3<double> gFN = gf, gvt = zero3<double>();
    double     g_nFN = 0.0;
    if(capped)
    {
        const double tg = dot(th, gf);
        g_law[3] += -nFN * tg;
        g_nFN = -L.muc * tg;
        if(nvt > 1e-10)
        {
            const V3<double> gth = (-fn) * gf;
            gvt                  = (1.0 / nvt) * (gth - dot(gth, th) * th);
        }
    }
    else
    {
        gvt = (-2.0 * L.etat * avmass) * gf;
        g_law[2] += -2.0 * avmass * dot(vt, gf);
    }
    if(nFN > 0.0)
        gFN = gFN + (g_nFN / nFN) * FN;
    g_law[0] += dot(vec, gFN) + omega0 / (2.0 * L.kn) * 2.0 * L.c * avmass * dot(vn, gFN);
    g_law[1] += 2.0 * omega0 * avmass * dot(vn, gFN) * L.dc_en;
    g_vec                 = L.kn * gFN;
    const V3<double> gvn  = (2.0 * omega0 * L.c * avmass) * gFN - gvt;
    const double     ngvn = dot(n, gvn);
    const V3<double> grel = gvt + ngvn * n;
    const V3<double> gn   = rn * gvn + ngvn * rel;
    g_vec                 = g_vec + (1.0 / np) * (gn - dot(n, gn) * n);
    g_vA                  = grel;
    g_vB                  = -grel;
    g_wA                  = cross(pt, grel);
    g_wB                  = -g_wA;
    g_pt                  = cross(grel, wA - wB);
}

// sphere A against sphere B (closestPointsSpheres, CollisionDetection.cpp:26-48):
// d = xB - xA, u = d/|d|, delta = |d| - rA - rB, vec = delta u,
// pt = xA + (rA + delta/2) u; gradients to xA and xB
GB_D void sphere_pair_vjp(const V3<double>& xa, const V3<double>& xb, double rA, double rB,
                          const AdjLaw& L, double avmass, const V3<double>& vA,
                          const V3<double>& wA, const V3<double>& vB, const V3<double>& wB,
                          const V3<double>& lf, const V3<double>& lt, V3<double>& gxA,
                          V3<double>& gxB, V3<double>& gvA, V3<double>& gwA, V3<double>& gvB,
                          V3<double>& gwB, double g_law[4])
{
    const V3<double> d     = xb - xa;
    const double     dn    = norm(d);
    const V3<double> u     = (1.0 / dn) * d;
    const double     delta = dn - rA - rB;
    const V3<double> vec   = delta * u;
    const V3<double> pt    = xa + (rA + 0.5 * delta) * u;
    const V3<double> arm   = pt - xa;
    V3<double>       gvec, gpt, garm;
    hooke_vjp(L, avmass, sqrt(L.kn / avmass), vec, pt, arm, vA, wA, vB, wB, lf, lt, gvec, gpt,
              garm, gvA, gwA, gvB, gwB, g_law);
    gpt                   = gpt + garm;
    const double     gdel = 0.5 * dot(u, gpt) + dot(u, gvec);
    const V3<double> gu   = (rA + 0.5 * delta) * gpt + delta * gvec;
    const V3<double> gd   = (1.0 / dn) * (gu - dot(u, gu) * u) + gdel * u;
    gxA                   = gpt - garm - gd;
    gxB                   = gd;
}

// integration: x' = x + dt v, v' = v + dt F/m, omega' = omega + dt T/I
__global__ void __launch_bounds__(kBlock)
    k_adj_integrate(int n, double dt, double h, int verlet, State<double> st,
                    const RBInertia<double>* __restrict__ in,
                    const double* __restrict__ adj_next, double* __restrict__ adj_prev,
                    double* __restrict__ lft)
{
    // FirstOrderExplicit: x' = x + dt v, v' = v + dt F/m, w' = w + dt T/I;
    // velocity Verlet (leapfrog): v' = v + h F/m, x' = x + dt v', w' = w + h T/I,
    // with h = dt/2 on a trajectory's first step and dt after it
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const RBInertia<double>* r = in + st.rb_id[i];
    const double             m = r->mass, i1 = r->I1[0];
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        const double lx = adj_next[(size_t)k * n + i], lv = adj_next[(size_t)(3 + k) * n + i];
        const double lw = adj_next[(size_t)(6 + k) * n + i];
        adj_prev[(size_t)k * n + i]       = lx;
        adj_prev[(size_t)(3 + k) * n + i] = lv + dt * lx;
        adj_prev[(size_t)(6 + k) * n + i] = lw;
        lft[(size_t)k * n + i]            = verlet ? h / m * (lv + dt * lx) : dt / m * lv;
        lft[(size_t)(3 + k) * n + i]      = (verlet ? h : dt) * i1 * lw;
    }
}

// contacts: thread i adds to its adjoint the contributions of its own pairs
// (i, j) and walls, and of the pairs (j, i) acting on its partners; block
// partial sums of the law gradients go to partial[block][4 * laws.n]
__global__ void __launch_bounds__(kBlock)
    k_adj_contacts(int n, State<double> st, const RBShape<double>* __restrict__ shape,
                   const RBInertia<double>* __restrict__ in, const uint32_t* __restrict__ off,
                   const uint32_t* __restrict__ pair_b, const uint8_t* __restrict__ contact,
                   const double* __restrict__ lft, const double* __restrict__ obs_tr,
                   const RBShape<double>* __restrict__ obs_shape, AdjLaws laws,
                   double* __restrict__ adj_prev, double* __restrict__ partial)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double    g_law[4 * kAdjMaxLaws];
#pragma unroll
    for(int k = 0; k < 4 * kAdjMaxLaws; ++k)
        g_law[k] = 0.0;
    if(i < n)
    {
        double* const lf_[3] = {const_cast<double*>(lft), const_cast<double*>(lft) + n,
                                const_cast<double*>(lft) + 2 * (size_t)n};
        double* const lt_[3] = {const_cast<double*>(lft) + 3 * (size_t)n,
                                const_cast<double*>(lft) + 4 * (size_t)n,
                                const_cast<double*>(lft) + 5 * (size_t)n};
        const uint32_t   ri = st.rb_id[i];
        const double     r_i = shape[ri].p[0], m_i = in[ri].mass; // the sphere's radius
        const int        mat_i = shape[ri].material;
        const V3<double> xi = ld3(st.pos, i), vi = ld3(st.vel, i), wi = ld3(st.omg, i);
        const V3<double> lfi = ld3(lf_, i), lti = ld3(lt_, i);
        V3<double>       gx = zero3<double>(), gv = zero3<double>(), gw = zero3<double>();
        for(uint32_t p = off[i]; p < off[i + 1]; ++p)
        {
            if(!contact[p])
                continue;
            const uint32_t b = pair_b[p];
            if(b & kObstacleBit)
            {
                // sphere i against a Rectangle wall (closestPointsRectangle,
                // CollisionDetection.cpp:53-90): s = rn . (xi - o) - r,
                // vec = -s rn, pt = xi - r rn - s rn / 2
                const int        o  = (int)(b & ~kObstacleBit);
                const double*    ot = obs_tr + 12 * o;
                V3<double>       rn = mk<double>(ot[2], ot[5], ot[8]);
                const V3<double> e  = xi - mk<double>(ot[9], ot[10], ot[11]);
                rn                  = copysign(1.0, dot(rn, e)) * rn;
                const double     s   = dot(rn, e) - r_i;
                const V3<double> vec = (-s) * rn;
                const V3<double> pt  = xi - r_i * rn - (0.5 * s) * rn;
                const int        l   = adj_law_index(mat_i, obs_shape[o].material);
                const double     avm = 0.5 * m_i; // obstacle mass 0 (HookeContactForceModel's rule)
                V3<double> gvec, gpt, garm, gvA, gwA, gvB, gwB;
                hooke_vjp(laws.l[l], avm, 2.0 * sqrt(laws.l[l].kn / avm), vec, pt, pt - xi, vi, wi,
                          zero3<double>(), zero3<double>(), lfi, lti, gvec, gpt, garm, gvA, gwA, gvB,
                          gwB, g_law + 4 * l);
                gpt             = gpt + garm;
                const double gs = -dot(rn, gvec) - 0.5 * dot(rn, gpt);
                gx              = gx + (gpt - garm) + gs * rn;
                gv              = gv + gvA;
                gw              = gw + gwA;
                continue;
            }
            const uint32_t   rj = st.rb_id[b];
            const double     r_j = shape[rj].p[0], m_j = in[rj].mass;
            const int        l   = adj_law_index(mat_i, shape[rj].material);
            const double     avm = m_i * m_j / (m_i + m_j);
            const V3<double> xj = ld3(st.pos, b), vj = ld3(st.vel, b), wj = ld3(st.omg, b);
            V3<double>       gxA, gxB, gvA, gwA, gvB, gwB;
            // the pair (i, j): force on i
            sphere_pair_vjp(xi, xj, r_i, r_j, laws.l[l], avm, vi, wi, vj, wj, lfi, lti, gxA, gxB,
                            gvA, gwA, gvB, gwB, g_law + 4 * l);
            gx = gx + gxA;
            gv = gv + gvA;
            gw = gw + gwA;
            // the pair (j, i): force on j, its dependence on i (laws counted by j)
            double scratch[4] = {0.0, 0.0, 0.0, 0.0};
            sphere_pair_vjp(xj, xi, r_j, r_i, laws.l[l], avm, vj, wj, vi, wi, ld3(lf_, b),
                            ld3(lt_, b), gxA, gxB, gvA, gwA, gvB, gwB, scratch);
            gx = gx + gxB;
            gv = gv + gvB;
            gw = gw + gwB;
        }
        adj_prev[i]                 += gx.x;
        adj_prev[(size_t)n + i]     += gx.y;
        adj_prev[2 * (size_t)n + i] += gx.z;
        adj_prev[3 * (size_t)n + i] += gv.x;
        adj_prev[4 * (size_t)n + i] += gv.y;
        adj_prev[5 * (size_t)n + i] += gv.z;
        adj_prev[6 * (size_t)n + i] += gw.x;
        adj_prev[7 * (size_t)n + i] += gw.y;
        adj_prev[8 * (size_t)n + i] += gw.z;
    }
    // block sums of the law gradients, in a fixed order: warp shuffles, then warps
    __shared__ double red[kBlock / 32][4 * kAdjMaxLaws];
    const int         nv = 4 * laws.n;
    for(int k = 0; k < nv; ++k)
    {
        double v = g_law[k];
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if((threadIdx.x & 31) == 0)
            red[threadIdx.x >> 5][k] = v;
    }
    __syncthreads();
    if(threadIdx.x < nv)
    {
        double v = 0.0;
        for(int w = 0; w < kBlock / 32; ++w)
            v += red[w][threadIdx.x];
        partial[(size_t)blockIdx.x * nv + threadIdx.x] = v;
    }
}

// grad[k] += sum over blocks of partial[block][k], blocks in order
__global__ void k_adj_reduce(int nblocks, int nv, const double* __restrict__ partial,
                             double* __restrict__ grad)
{
    const int k = threadIdx.x;
    if(k >= nv)
        return;
    double v = 0.0;
    for(int b = 0; b < nblocks; ++b)
        v += partial[(size_t)b * nv + k];
    grad[k] += v;
}

} // namespace gb
