// gb_step.cuh -- candidate pairs, narrow phase + contact law, and the fused
// per-particle reduction / walls / gravity / integration kernel.
#pragma once

#include "gb_broadphase.cuh"
#include "gb_dem.cuh"

namespace gb
{

// Particle state on the device, structure of arrays.  Positions are FP64 in
// every mode.  Orientation: in the FP64 modes the 3x3 basis of Grains'
// Transform3 (9 arrays, row-major), updated exactly as
// Transform3::composeLeftByRotation; in the mixed mode a unit quaternion
// (w, x, y, z) as a compensated FP32 pair: rot[0..3] hold the FP32 value,
// read by the FP32 bounding tests, and rot[4..7] the FP32 remainder, so that
// hi + lo (read by the FP64 contact geometry) keeps the orientation to FP64
// accuracy (an FP32 quaternion alone rounds a pose by ~6e-8 rad, which moves
// GJK's stopping point on resting contacts).
template <typename St>
struct State
{
    double*   pos[3];
    St*       rot[9]; // basis (FP64 modes) or quaternion hi in rot[0..3], lo in rot[4..7] (mixed)
    St*       vel[3];
    St*       omg[3];
    St*       frc[3];
    St*       trq[3];
    uint32_t* rb_id;
};

template <typename S>
struct Tables
{
    const RBShape<store_t<S>>*   shape;
    const RBInertia<store_t<S>>* inertia;
    const Vert<store_t<S>>*      verts;
    const Law<store_t<S>>*       law; // material-pair table
    const RBShape<store_t<S>>*   obs_shape;
    const double*                obs_tr; // 12 per obstacle (basis, origin)
    const double*                obs_mass;
    const double4*               obs_plane; // Rectangle planes: normal, normal . origin
    const double*                obs_vel;   // 6 per obstacle: velocity, angular velocity
    uint32_t                     obs_rect;  // bit o: obstacle o (< 32) is a Rectangle
    int                          n_obs;
    // FP64 copies of the shape tables (read by the mixed mode's FP64 GJK)
    const RBShape<double>* shape64;
    const Vert<double>*    verts64;
    const RBShape<double>* obs_shape64;
};

// ---- mixed precision narrow phase --------------------------------------------
// The bounding-sphere and OBB tests run in FP32 on FP32 poses (their margins
// are absolute: LOWEPS on the OBB axes, the crust-free bounding box), and every
// pair that survives them and that the FP32 stages (GJK's first iteration, the
// FP32 GJK) do not certify as separated is solved by the FP64 GJK of the FP64
// mode, with FP64 shape tables and the compensated quaternion: FP32 support
// points on mm-size grains carry ~1e-10 m of rounding, the order of a resting
// contact's overlap (m g / kn ~ 1e-8 m), so contact points and overlaps come
// from FP64.

GB_D Quat<double> load_quat64(const State<float>& st, uint32_t i)
{
    Quat<double> q;
    q.w = (double)st.rot[0][i] + (double)st.rot[4][i];
    q.v = mk<double>((double)st.rot[1][i] + (double)st.rot[5][i],
                     (double)st.rot[2][i] + (double)st.rot[6][i],
                     (double)st.rot[3][i] + (double)st.rot[7][i]);
    return q;
}

GB_D M3<double> load_rot64(const State<float>& st, uint32_t i)
{
    const Quat<double> q = load_quat64(st, i);
    return quat_to_matrix<double>(q.w, q.v.x, q.v.y, q.v.z);
}

GB_D Contact<float> to_f(const Contact<double>& c)
{
    Contact<float> r;
    r.pt      = cvt3<float>(c.pt);
    r.vec     = cvt3<float>(c.vec);
    r.overlap = (float)c.overlap;
    return r;
}

// closestPointsSpheres (CollisionDetection.cpp:26-48) for the mixed mode:
// the closed form directly in FP64, the point relative to A's centre.
GB_D Contact<float> closest_spheres_mixed(const Tables<float>& tb, uint32_t ra, uint32_t rb,
                                          const double xa[3], const double xb[3])
{
    const V3<double> d64 = mk<double>(xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]);
    const double     rA = tb.shape64[ra].p[0], rB = tb.shape64[rb].p[0]; // the radii
    const double     nd = norm(d64), overlap = nd - rA - rB;
    if(!(overlap < 0.0))
        return no_contact<float>();
    const V3<double> u = d64 / nd;
    Contact<double>  c;
    c.pt      = (rA + 0.5 * overlap) * u;
    c.vec     = overlap * u;
    c.overlap = overlap;
    return to_f(c);
}

// closestPointsRigidBodies for the mixed mode; points relative to A's centre.
// VAR: the GJK variant of the FP64 solve.
template <int VAR>
GB_D Contact<float> closest_mixed(const Tables<float>& tb, const State<float>& st, uint32_t a,
                                  uint32_t b, uint32_t ra, uint32_t rb, const Body<float>& A,
                                  const Body<float>& B, const M3<float>& RA, const M3<float>& RB,
                                  const double xa[3], const double xb[3], int* iters)
{
    const V3<double> d64 = mk<double>(xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]);
    if(A.type == GB_SPHERE && B.type == GB_SPHERE)
        return closest_spheres_mixed(tb, ra, rb, xa, xb);
    const V3<float> d = cvt3<float>(d64);
    if(!(norm(d) - (A.rcirc + B.rcirc) < 0.0f))
        return no_contact<float>();
    if(!obb_overlap(A.bb, B.bb, RA, RB, d))
        return no_contact<float>();
    // every pair that passes the bounding tests is solved on the FP64 path of
    // the FP64 mode
    const Body<double> A64 = load_body<double>(tb.shape64, ra, tb.verts64);
    const Body<double> B64 = load_body<double>(tb.shape64, rb, tb.verts64);
    const M3<double>   RA64 = load_rot64(st, a), RB64 = load_rot64(st, b);
    Tr<double>         b2a64;
    const M3<double>   RAt64 = transpose(RA64);
    b2a64.R                  = mul(RAt64, RB64);
    b2a64.o                  = mul(RAt64, d64);
    const GjkResult<double> g = gjk<VAR>(A64, B64, b2a64);
    *iters += g.iters;
    const double distance = g.dist - (A64.crust + B64.crust);
    if(distance > 0.0)
        return no_contact<float>();
    const V3<double> ptA = mul(RA64, g.pa);
    const V3<double> ptB = mul(RB64, g.pb) + d64;
    Contact<double>  c;
    c.pt      = (ptA + ptB) / 2.0;
    V3<double> vec = ptA - ptB;
    vec            = round3(vec / norm(vec), 1e-10);
    c.vec          = (-distance) * vec;
    c.overlap      = distance;
    return to_f(c);
}

template <typename S>
GB_D constexpr bool is_mixed()
{
    return sizeof(store_t<S>) == 4;
}

template <typename S>
GB_D M3<S> load_rot(const State<store_t<S>>& st, uint32_t i)
{
    if constexpr(is_mixed<S>())
        return quat_to_matrix<S>(S(st.rot[0][i]), S(st.rot[1][i]), S(st.rot[2][i]),
                                 S(st.rot[3][i]));
    else
    {
        M3<S> R;
#pragma unroll
        for(int k = 0; k < 9; ++k)
            R.m[k] = S(st.rot[k][i]);
        return R;
    }
}

template <typename S>
GB_D V3<S> load3(store_t<S>* const a[3], uint32_t i)
{
    return mk<S>(S(a[0][i]), S(a[1][i]), S(a[2][i]));
}

template <typename S>
GB_D Law<S> load_law(const Law<store_t<S>>* t, int ma, int mb)
{
    // ContactForceModelBuilderFactory::computeHash (ContactForceModelBuilderFactory.cpp:77-83)
    const unsigned s = ma < mb ? ma : mb, l = ma < mb ? mb : ma;
    const Law<store_t<S>> L = t[l * (l + 1) / 2 + s];
    Law<S>                r;
    r.kn   = S(L.kn);
    r.muen = S(L.muen);
    r.etat = S(L.etat);
    r.muc  = S(L.muc);
    r.kr   = S(L.kr);
    r.kt   = S(L.kt);
    return r;
}

// ---- candidate pairs ----------------------------------------------------------
// One thread per particle in cell-sorted order.  Enumerates the 27 neighbour
// cells in the reference's order (k = z outer, j = y, i = x inner; the
// neighbour table of LinkedCell.cpp:41-70) and the particles of each cell in
// ascending id, keeping ordered pairs (A, B != A) whose bounding spheres
// overlap: norm(xB - xA) - (rA + rB) < 0 (CollisionDetection.cpp:209-211).
// The three cells x-1, x, x+1 of one (y, z) row have consecutive keys, so
// their particles are one contiguous range of the sorted order: the walk is
// nine ranges, visiting the candidates in the same order as the 27 cells.
// PRE32 (the mixed mode): a conservative FP32 test on spos32 (put_sorted
// inflates its radii by a bound on the FP32 rounding, so an FP32 rejection
// implies an FP64 rejection) skips most non-candidates before the FP64 test:
// the candidate set is the FP64 test's.  The FP64 modes test in FP64 only.
// Candidates kept per particle by the count pass: 32 covers all but ~1e-4 of
// the particles of a dense polydisperse bed (mean ~7, 99.9th percentile ~25);
// the fill pass enumerates the rest again.
constexpr int kPairSlots = 32;

// Particle-obstacle pairs (ComponentManagerCPU.cpp:301-351) share the pair
// list: after the particle pairs of A come A's obstacle candidates in obstacle
// order, as b = kObstacleBit | o, so that the segmented sum adds the obstacle
// forces after the particle forces, in the reference's order.
constexpr uint32_t kObstacleBit     = 0x80000000u;
constexpr uint8_t  kContactParticle = 1; // contact flags of a pair record
constexpr uint8_t  kContactObstacle = 2;
constexpr int      kMaskObstacles   = 32; // obstacles beyond these are always candidates

// Frame of obstacle o for particle A at xa: A's centre oA and the obstacle's
// origin oO (relative to xa in the mixed mode, absolute in the FP64 modes).
template <typename S>
GB_D void obstacle_frame(const Tables<S>& tb, int o, const double xa[3], V3<S>& oA, V3<S>& oO,
                         M3<S>& RO)
{
    const double* ot = tb.obs_tr + 12 * o;
    if constexpr(is_mixed<S>())
    {
        oA = zero3<S>();
        oO = mk<S>(S(ot[9] - xa[0]), S(ot[10] - xa[1]), S(ot[11] - xa[2]));
    }
    else
    {
        oA = mk<S>(S(xa[0]), S(xa[1]), S(xa[2]));
        oO = mk<S>(S(ot[9]), S(ot[10]), S(ot[11]));
    }
#pragma unroll
    for(int k = 0; k < 9; ++k)
        RO.m[k] = S(ot[k]);
}

// Obstacles that particle a may touch, bit o for obstacle o < kMaskObstacles.
// A lies in its bounding box (half extents bb), so its support point towards
// a Rectangle's plane is at most bb . |RA^T n| from its centre: a centre
// farther than that from the plane (plus a bound on the rounding of both
// sides) cannot touch it, and the full test of closest_rectangle would reject
// it too.  Other obstacle types are always candidates.
// The box's extent along any unit normal is at most |bb| (Cauchy-Schwarz), so
// a centre farther than |bb| from every plane is decided without the
// rotation: `rot` (a callable returning RA) runs only for the planes within
// that reach.
template <typename S, typename Rot>
GB_D uint32_t obstacle_mask_at(const Tables<S>& tb, uint32_t r, Rot&& rot, const double xa[3])
{
    const int nm = tb.n_obs < kMaskObstacles ? tb.n_obs : kMaskObstacles;
    if(nm == 0)
        return 0u;
    // in FP64 throughout: the plane distance from the exact centre, the box
    // extent along the normal from this mode's rotation; the slack covers the
    // rounding of both and the 1e-7 difference between the mixed mode's FP32
    // rotation and the FP64 one its contact recomputation uses
    const double bb[3] = {(double)tb.inertia[r].bb[0], (double)tb.inertia[r].bb[1],
                          (double)tb.inertia[r].bb[2]};
    const double ax    = fabs(xa[0]) + fabs(xa[1]) + fabs(xa[2]);
    uint32_t     mask  = ~tb.obs_rect & ((nm == 32) ? ~0u : ((1u << nm) - 1u));
    const double reach = sqrt(bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
    bool         have  = false;
    M3<S>        RA;
    for(int o = 0; o < nm; ++o)
    {
        if(!((tb.obs_rect >> o) & 1u))
            continue;
        const double4 pl = tb.obs_plane[o];
        const double  dc = fabs(pl.x * xa[0] + pl.y * xa[1] + pl.z * xa[2] - pl.w);
        if(dc - reach > 1e-6 * reach + 1e-12 * (1.0 + ax + fabs(pl.w)))
            continue; // beyond the box's reach whatever its orientation
        if(!have)
        {
            RA   = rot();
            have = true;
        }
        double hb, slack;
        if constexpr(is_mixed<S>())
        {
            // the extent from the FP32 rotation in FP32: each |(RA^T n)_k|
            // is off by a few 1e-7 (its rounding, and the FP32 rotation's
            // distance from the FP64 one), so the slack takes 1e-6 of the
            // box's half-extents' sum
            const float n32[3] = {(float)pl.x, (float)pl.y, (float)pl.z};
            float       h32    = 0.0f;
#pragma unroll
            for(int k = 0; k < 3; ++k)
                h32 += (float)bb[k]
                       * fabsf(RA.m[k] * n32[0] + RA.m[3 + k] * n32[1] + RA.m[6 + k] * n32[2]);
            hb    = (double)h32;
            slack = 1e-6 * (bb[0] + bb[1] + bb[2]) + 1e-12 * (1.0 + ax + fabs(pl.w));
        }
        else
        {
            hb = 0.0;
#pragma unroll
            for(int k = 0; k < 3; ++k)
            {
                // (RA^T n)_k = sum_j RA[j][k] n_j
                const double nk = to_d(RA.m[k]) * pl.x + to_d(RA.m[3 + k]) * pl.y
                                  + to_d(RA.m[6 + k]) * pl.z;
                hb += bb[k] * fabs(nk);
            }
            slack = 1e-6 * hb + 1e-12 * (1.0 + ax + fabs(pl.w));
        }
        if(!(dc - hb > slack))
            mask |= 1u << o;
    }
    return mask;
}

// The mask is computed where the pose is at hand: by k_particles right after
// each move, and by k_obstacle_mask after the state was set from the host.
template <typename S>
__global__ void __launch_bounds__(kBlock)
    k_obstacle_mask(int n, State<store_t<S>> st, Tables<S> tb, uint32_t* __restrict__ mask)
{
    grid_dep_sync();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const double xa[3] = {st.pos[0][i], st.pos[1][i], st.pos[2][i]};
    mask[i] = obstacle_mask_at<S>(tb, st.rb_id[i], [&] { return load_rot<S>(st, i); }, xa);
}

// A particle's obstacle candidates, in ascending obstacle order (the order of
// the reference's obstacle loop, ComponentManagerCPU.cpp:301-351).  The
// Rectangles among the first kMaskObstacles are decided by the particle's
// mask (walls within reach after the last move); every other obstacle comes
// from its linked cell's list -- the obstacles whose surface a particle of
// that cell may reach, binned on the host when the obstacles are set.
// Without lists (every obstacle a Rectangle among the first 32, or none) the
// mask decides alone; its bits of the other first-32 obstacles are set.
struct ObsCand
{
    const uint32_t* mask;       // by particle id
    int             n;          // obstacles
    uint32_t        rect;       // bit o: obstacle o (< 32) is a Rectangle
    const uint32_t* cell_start; // C + 1 offsets into cell_ids, by linked cell (or null)
    const uint32_t* cell_ids;   // the listed obstacles, ascending per cell
    const uint32_t* skeys;      // linked-cell key by sorted position
};

GB_D int obstacle_candidates(const ObsCand& oc, uint32_t a, uint32_t s)
{
    if(!oc.n)
        return 0;
    if(oc.cell_start)
    {
        const uint32_t key = oc.skeys[s];
        return __popc(oc.mask[a] & oc.rect) + (int)(oc.cell_start[key + 1] - oc.cell_start[key]);
    }
    return __popc(oc.mask[a]) + (oc.n > kMaskObstacles ? oc.n - kMaskObstacles : 0);
}

template <typename Visit>
GB_D void for_each_obstacle_candidate(const ObsCand& oc, uint32_t a, uint32_t s, Visit&& visit)
{
    if(!oc.n)
        return;
    uint32_t mask = oc.mask[a];
    if(oc.cell_start)
    {
        // the mask's Rectangles merged into the cell's list, both ascending
        mask &= oc.rect;
        const uint32_t key = oc.skeys[s];
        for(uint32_t k = oc.cell_start[key]; k < oc.cell_start[key + 1]; ++k)
        {
            const uint32_t o = oc.cell_ids[k];
            while(mask && (uint32_t)(__ffs(mask) - 1) < o)
            {
                visit((uint32_t)(__ffs(mask) - 1));
                mask &= mask - 1u;
            }
            visit(o);
        }
        for(; mask; mask &= mask - 1u)
            visit((uint32_t)(__ffs(mask) - 1));
        return;
    }
    const int nm = oc.n < kMaskObstacles ? oc.n : kMaskObstacles;
    for(int o = 0; o < nm; ++o)
        if((mask >> o) & 1u)
            visit((uint32_t)o);
    for(int o = kMaskObstacles; o < oc.n; ++o)
        visit((uint32_t)o);
}

template <typename S>
GB_D constexpr bool is_strict()
{
    return std::is_same<S, dstrict>::value;
}

// The candidate test of sorted particles a and b: |d| - (rA + rB) < 0 in
// FP64 (ComponentManagerCPU.cpp:372-380; the strict mode in the reference's
// operation order), behind the FP32 pre-test of the mixed mode, whose
// rejection is certified (put_sorted inflates the FP32 radii).  The
// products and sums are written as explicit round-to-nearest operations, so
// that every kernel that enumerates candidates -- the count pass and the
// re-enumeration of the fill pass -- takes the same decisions.
template <bool PRE32>
GB_D bool pretest_rejects(const float4& a32, const float4& q)
{
    if constexpr(PRE32)
    {
        const float fx = __fsub_rn(q.x, a32.x), fy = __fsub_rn(q.y, a32.y);
        const float fz = __fsub_rn(q.z, a32.z), fr = __fadd_rn(a32.w, q.w);
        return __fmaf_rn(fz, fz, __fmaf_rn(fy, fy, __fmul_rn(fx, fx))) >= __fmul_rn(fr, fr);
    }
    else
        return false;
}

template <bool STRICT>
GB_D bool exact_hit(const double4& pa, const double4& pb)
{
    if constexpr(STRICT)
    {
        const dstrict dx = dstrict(pb.x) - dstrict(pa.x);
        const dstrict dy = dstrict(pb.y) - dstrict(pa.y);
        const dstrict dz = dstrict(pb.z) - dstrict(pa.z);
        return s_sqrt(dx * dx + dy * dy + dz * dz) - (dstrict(pa.w) + dstrict(pb.w))
               < dstrict(0.0);
    }
    else
    {
        const double dx = __dsub_rn(pb.x, pa.x), dy = __dsub_rn(pb.y, pa.y);
        const double dz = __dsub_rn(pb.z, pa.z), r = __dadd_rn(pa.w, pb.w);
        return __fma_rn(dz, dz, __fma_rn(dy, dy, __dmul_rn(dx, dx))) < __dmul_rn(r, r);
    }
}

// The 27 neighbour cells of cell (cx, cy, cz) in the reference's enumeration
// order (LinkedCell.cpp:66-112, k then j then i) are 9 rows of up to 3 cells;
// the cells of a row are consecutive keys, so each row is one contiguous
// range [begin, end) of sorted positions.
GB_D void neighbour_row(const uint32_t* __restrict__ cstart, uint32_t nx, uint32_t ny, uint32_t nz,
                        int cx, int cy, int cz, int r, uint32_t& begin, uint32_t& end)
{
    const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
    begin = end = 0;
    if(z < 0 || z >= (int)nz || y < 0 || y >= (int)ny)
        return;
    const int      x0  = cx > 0 ? cx - 1 : 0, x1 = cx + 1 < (int)nx ? cx + 1 : cx;
    const uint32_t row = ((uint32_t)z * ny + (uint32_t)y) * nx;
    begin              = cstart[row + (uint32_t)x0];
    end                = cstart[row + (uint32_t)x1 + 1];
}

template <bool STRICT, bool PRE32, typename Hit>
GB_D void for_each_candidate(int s, const uint32_t* __restrict__ skeys,
                             const double4* __restrict__ spos,
                             const float4* __restrict__ spos32,
                             const uint32_t* __restrict__ cstart, uint32_t nx, uint32_t ny,
                             uint32_t nz, Hit&& hit)
{
    const uint32_t key = skeys[s];
    const double4  pa  = spos[s];
    float4         pa32;
    if constexpr(PRE32)
        pa32 = spos32[s];
    const int cx = key % nx, cy = (key / nx) % ny, cz = key / (nx * ny);
    for(int r = 0; r < 9; ++r)
    {
        uint32_t t0, t1;
        neighbour_row(cstart, nx, ny, nz, cx, cy, cz, r, t0, t1);
        // the particle itself passes every test below and is dropped
        // only on a hit, which keeps the common path short
#pragma unroll 2
        for(uint32_t t = t0; t < t1; ++t)
        {
            if constexpr(PRE32)
                if(pretest_rejects<PRE32>(pa32, spos32[t]))
                    continue;
            if(exact_hit<STRICT>(pa, spos[t]) && t != (uint32_t)s)
                hit(t);
        }
    }
}

// Count pass over half of the stencil, one thread per sorted particle s.
// The candidate test is symmetric bit for bit (b - a is -(a - b) exactly, and
// the radius sum commutes), so each unordered pair is tested once: by s for
// the partners t after it in the stencil's enumeration order -- the rest of
// its own row (the cells x, x + 1 of row (dz, dy) = (0, 0) from s + 1 on,
// one contiguous range) and the 4 rows (0, +1), (+1, -1), (+1, 0), (+1, +1).
// A hit counts for both particles: count[id] (zeroed; the scan's input) and
// pslot[sorted position] (zeroed; the slot index) by atomics, and the first
// kPairSlots partners of each sorted position go to its slots in arrival
// order.  The enumeration order of a particle's candidates is ascending
// sorted position (rows ascend in (z, y), cells in x, ids within a cell), so
// the fill pass restores it by sorting the slots.  Obstacle candidates are
// added to count[id] by the particle itself.
//
// Reach: a particle b hashed to a neighbour cell lies beyond the cell faces
// that separate that cell from a's (a centre clamped into the grid lies
// further out still), so |a - b| is at least the distance from a to those
// faces, and a candidate needs |a - b| < rA + rB <= rA + rmax.  The rows and
// the end cells of a row that are farther than that, with a margin far above
// the rounding of the hash and of the faces, hold no pair that the exact test
// accepts and are not walked; the pair set is unchanged.  The FP64 modes
// prune so (their exact test on every candidate is the costly part); the
// mixed mode does not, since its FP32 pre-test is cheap and a warp walks the
// longest range among its lanes anyway: pruning measured slower there.
//
// Latency-bound on L1 hits: the mixed instantiation runs at full occupancy
// (32 registers), which measured 5% faster than 40 registers at six blocks
// per SM.
struct CellGeometry
{
    double mn[3]; // grid origin
    double cell;  // cell edge
    double rmax;  // largest bounding radius of any particle
};

template <typename S>
__global__ void __launch_bounds__(kBlock, sizeof(store_t<S>) == 4 ? 8 : 6)
    k_pair_count(int n, const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ sids,
                 const double4* __restrict__ spos, const float4* __restrict__ spos32,
                 const uint32_t* __restrict__ cstart, uint32_t nx, uint32_t ny, uint32_t nz,
                 CellGeometry geo, uint32_t* __restrict__ count, uint32_t* __restrict__ pslot,
                 uint32_t* __restrict__ slot, ObsCand oc, const int* abort_flags)
{
    grid_dep_sync();
    constexpr bool STRICT = is_strict<S>(), PRE32 = is_mixed<S>();
    const int      s      = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= n || step_aborted(abort_flags))
        return;
    if(oc.n)
    {
        const uint32_t a   = sids[s];
        const int      obs = obstacle_candidates(oc, a, (uint32_t)s);
        if(obs)
            atomicAdd(count + a, (uint32_t)obs);
    }
    const uint32_t key = skeys[s];
    const double4  pa  = spos[s];
    float4         pa32;
    if constexpr(PRE32)
        pa32 = spos32[s];
    const int cx = key % nx, cy = (key / nx) % ny, cz = key / (nx * ny);
    auto record = [&](uint32_t u, uint32_t v) {
        const uint32_t k = atomicAdd(pslot + u, 1u);
        if(k < kPairSlots)
            slot[(size_t)u * kPairSlots + k] = v;
        atomicAdd(count + sids[u], 1u);
    };
    // distances from a to the faces of its cell (0 if a lies outside it)
    constexpr bool PRUNE = !PRE32;
    double         r2 = 0.0, gxm = 0.0, gxp = 0.0, gym = 0.0, gyp = 0.0, gzp = 0.0;
    if constexpr(PRUNE)
    {
        const double reach = (pa.w + geo.rmax) * (1.0 + 1e-6) + 1e-6 * geo.cell;
        r2                 = reach * reach;
        gxm = fmax(pa.x - (geo.mn[0] + cx * geo.cell), 0.0);
        gxp = fmax(geo.mn[0] + (cx + 1) * geo.cell - pa.x, 0.0);
        gym = fmax(pa.y - (geo.mn[1] + cy * geo.cell), 0.0);
        gyp = fmax(geo.mn[1] + (cy + 1) * geo.cell - pa.y, 0.0);
        gzp = fmax(geo.mn[2] + (cz + 1) * geo.cell - pa.z, 0.0);
    }
    for(int r = 4; r < 9; ++r)
    {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        const int z = cz + dz, y = cy + dy;
        if(z >= (int)nz || y < 0 || y >= (int)ny)
            continue;
        bool left = cx > 0, right = cx + 1 < (int)nx;
        if constexpr(PRUNE)
        {
            const double gy = dy < 0 ? gym : (dy > 0 ? gyp : 0.0);
            const double gz = dz > 0 ? gzp : 0.0;
            const double d2 = gy * gy + gz * gz;
            if(d2 > r2)
                continue;
            left  = left && !(d2 + gxm * gxm > r2);
            right = right && !(d2 + gxp * gxp > r2);
        }
        const uint32_t row = ((uint32_t)z * ny + (uint32_t)y) * nx;
        const uint32_t t0 = r == 4 ? (uint32_t)s + 1 : cstart[row + (uint32_t)(left ? cx - 1 : cx)];
        const uint32_t t1 = cstart[row + (uint32_t)(right ? cx + 2 : cx + 1)];
#pragma unroll 2
        for(uint32_t t = t0; t < t1; ++t)
        {
            if constexpr(PRE32)
                if(pretest_rejects<PRE32>(pa32, spos32[t]))
                    continue;
            if(exact_hit<STRICT>(pa, spos[t]))
            {
                record((uint32_t)s, t);
                record(t, (uint32_t)s);
            }
        }
    }
}

// A warp walks the concatenation of up to 32 ranges [t0, t1) of sorted
// positions, lane r holding range r (lanes past the last range hold empty
// ones), 32 entries a round in range order: visit(t, valid) runs on every
// lane each round (warp-uniform).  All ranges' bounds are loaded at once, by
// their lanes, and short ranges share rounds, where a range-at-a-time walk
// pays a dependent load pair and a mostly idle round per range.
template <typename Visit>
GB_D void warp_ranges(uint32_t t0, uint32_t t1, Visit&& visit)
{
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t len  = t1 > t0 ? t1 - t0 : 0u;
    uint32_t       inc  = len; // inclusive prefix of the lengths
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if(lane >= (unsigned)o)
            inc += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
    const uint32_t exc   = inc - len;
    for(uint32_t base = 0; base < total; base += 32)
    {
        const uint32_t idx = base + lane;
        // the last range that starts at or before idx (exclusive prefixes
        // do not decrease; an empty range shares its start with the next)
        unsigned r = 0;
#pragma unroll
        for(unsigned step = 16; step >= 1; step >>= 1)
            if(__shfl_sync(0xffffffffu, exc, r + step) <= idx)
                r += step;
        const uint32_t t = __shfl_sync(0xffffffffu, t0, r) + (idx - __shfl_sync(0xffffffffu, exc, r));
        visit(t, idx < total);
    }
}

// ---- candidate search on a finer grid (polydisperse packings) -----------------
// The reference's cell is twice the LARGEST bounding radius, so in a
// polydisperse packing a particle's 27 cells hold hundreds of others (~960 in
// the 2.2 mm bed of 0.5-2 mm grains, 7.2 mm cells).  The same candidate set
// is found with far fewer tests on a second grid of cell h >= 2 r_s, r_s a
// bounding radius that most particles do not exceed ("small"; the others are
// "large"):
//   small-small pairs: |d| < rA + rB <= 2 r_s <= h, adjacent fine cells --
//     the half stencil of k_pair_count on the fine grid (k_pair_count_fine);
//   small-large pairs: the large particle scans the fine cells within its
//     reach rL + r_s (k_pair_count_large, one warp per large particle);
//   large-large pairs: the large particle scans the fine cells within its
//     reach rL + r_max for large partners after it in the fine order.
// Each unordered pair is tested once, with the same symmetric test
// (pretest_rejects + exact_hit), and recorded for both particles into the
// same slots and counts (by reference sorted position and id) as
// k_pair_count: the fill pass's sort restores the reference's order, so
// the pair list is the same, bit for bit.  A large particle's key is its
// fine cell plus nf (the fine cell count): the fine order holds the small
// particles by cell, then the large ones by cell.
struct FineGrid
{
    double   mn[3];
    double   h;    // fine cell edge
    double   rs;   // the small particles' bounding-radius limit
    double   rmax; // the largest bounding radius
    uint32_t nx, ny, nz;
};

GB_D uint32_t fine_axis(double x, double mn, double h, uint32_t n)
{
    const double f = (x - mn) / h; // NaN falls to cell 0
    return f >= 0.0 ? (f < (double)n ? (uint32_t)f : n - 1u) : 0u;
}

__global__ void __launch_bounds__(kBlock)
    k_fine_hash(int n, const double* __restrict__ px, const double* __restrict__ py,
                const double* __restrict__ pz, const uint32_t* __restrict__ rb_id,
                const double* __restrict__ rcirc, FineGrid g, uint32_t* __restrict__ fkey,
                uint32_t* __restrict__ fcount, const int* abort_flags)
{
    grid_dep_sync();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n || step_aborted(abort_flags))
        return;
    uint32_t key = (fine_axis(pz[i], g.mn[2], g.h, g.nz) * g.ny + fine_axis(py[i], g.mn[1], g.h, g.ny))
                       * g.nx
                   + fine_axis(px[i], g.mn[0], g.h, g.nx);
    if(rcirc[rb_id[i]] > g.rs)
        key += g.nx * g.ny * g.nz; // the large particles' cells
    fkey[i] = key;
    atomicAdd(&fcount[key], 1u);
}

// each particle into a free slot of its fine cell (any order within a cell:
// the fill pass sorts), with its key, id, reference sorted position and
// positions (put_sorted); leaves the counts at zero
__global__ void __launch_bounds__(kBlock)
    k_fine_scatter(int n, const uint32_t* __restrict__ fkey, const uint32_t* __restrict__ fstart,
                   uint32_t* __restrict__ fcount, const double* __restrict__ px,
                   const double* __restrict__ py, const double* __restrict__ pz,
                   const uint32_t* __restrict__ rb_id, const double* __restrict__ rcirc,
                   const uint32_t* __restrict__ sorted_of, uint32_t* __restrict__ fskey,
                   uint32_t* __restrict__ fids, uint32_t* __restrict__ fref,
                   double4* __restrict__ fpos, float4* __restrict__ fpos32, const int* abort_flags)
{
    grid_dep_sync();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n || step_aborted(abort_flags))
        return;
    const uint32_t key  = fkey[i];
    const uint32_t slot = fstart[key] + atomicSub(&fcount[key], 1u) - 1u;
    fskey[slot]         = key;
    fids[slot]          = (uint32_t)i;
    fref[slot]          = sorted_of[i];
    put_sorted(slot, (uint32_t)i, px, py, pz, rb_id, rcirc, fpos, fpos32);
}

// a hit between fine entries: both particles' slots and counts, by reference
// sorted position and id, as k_pair_count records them
GB_D void record_pair(uint32_t u, uint32_t id_u, uint32_t v, uint32_t id_v,
                      uint32_t* __restrict__ count, uint32_t* __restrict__ pslot,
                      uint32_t* __restrict__ slot)
{
    uint32_t k = atomicAdd(pslot + u, 1u);
    if(k < kPairSlots)
        slot[(size_t)u * kPairSlots + k] = v;
    atomicAdd(count + id_u, 1u);
    k = atomicAdd(pslot + v, 1u);
    if(k < kPairSlots)
        slot[(size_t)v * kPairSlots + k] = u;
    atomicAdd(count + id_v, 1u);
}

// small particles: k_pair_count's half stencil on the fine grid (whose cells
// hold small particles only); one thread per fine sorted position
template <typename S>
__global__ void __launch_bounds__(kBlock, 6)
    k_pair_count_fine(int n, const uint32_t* __restrict__ fstart, FineGrid g,
                      const uint32_t* __restrict__ fskey, const uint32_t* __restrict__ fids,
                      const uint32_t* __restrict__ fref, const double4* __restrict__ fpos,
                      const float4* __restrict__ fpos32, uint32_t* __restrict__ count,
                      uint32_t* __restrict__ pslot, uint32_t* __restrict__ slot,
                      ObsCand oc, const int* abort_flags)
{
    grid_dep_sync();
    constexpr bool STRICT = is_strict<S>(), PRE32 = is_mixed<S>();
    const int      f      = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nx = g.nx, ny = g.ny, nz = g.nz;
    if(f >= n || step_aborted(abort_flags) || (uint32_t)f >= fstart[nx * ny * nz])
        return;
    const uint32_t a = fids[f], sa = fref[f];
    if(oc.n)
    {
        const int obs = obstacle_candidates(oc, a, sa);
        if(obs)
            atomicAdd(count + a, (uint32_t)obs);
    }
    const uint32_t key = fskey[f];
    const double4  pa  = fpos[f];
    float4         pa32;
    if constexpr(PRE32)
        pa32 = fpos32[f];
    const int cx = key % nx, cy = (key / nx) % ny, cz = key / (nx * ny);
    for(int r = 4; r < 9; ++r)
    {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        const int z = cz + dz, y = cy + dy;
        if(z >= (int)nz || y < 0 || y >= (int)ny)
            continue;
        const bool     left = cx > 0, right = cx + 1 < (int)nx;
        const uint32_t row  = ((uint32_t)z * ny + (uint32_t)y) * nx;
        const uint32_t t0 = r == 4 ? (uint32_t)f + 1 : fstart[row + (uint32_t)(left ? cx - 1 : cx)];
        const uint32_t t1 = fstart[row + (uint32_t)(right ? cx + 2 : cx + 1)];
#pragma unroll 2
        for(uint32_t t = t0; t < t1; ++t)
        {
            if constexpr(PRE32)
                if(pretest_rejects<PRE32>(pa32, fpos32[t]))
                    continue;
            if(exact_hit<STRICT>(pa, fpos[t]))
                record_pair(sa, a, fref[t], fids[t], count, pslot, slot);
        }
    }
}

// large particles (keys past the small ones'), one warp each: small partners
// from the fine cells within reach rL + r_s, then large partners after it in
// the fine order from the large particles' cells within reach rL + r_max
template <typename S>
__global__ void __launch_bounds__(kBlock)
    k_pair_count_large(int n, const uint32_t* __restrict__ fstart, FineGrid g,
                       const uint32_t* __restrict__ fids, const uint32_t* __restrict__ fref,
                       const double4* __restrict__ fpos, const float4* __restrict__ fpos32,
                       uint32_t* __restrict__ count, uint32_t* __restrict__ pslot,
                       uint32_t* __restrict__ slot, ObsCand oc, const int* abort_flags)
{
    grid_dep_sync();
    constexpr bool STRICT = is_strict<S>(), PRE32 = is_mixed<S>();
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t nf   = g.nx * g.ny * g.nz;
    const int64_t  f    = (int64_t)fstart[nf] + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    if(f >= n || step_aborted(abort_flags)) // warp-uniform
        return;
    const uint32_t a = fids[f], sa = fref[f];
    if(oc.n && lane == 0)
    {
        const int obs = obstacle_candidates(oc, a, sa);
        if(obs)
            atomicAdd(count + a, (uint32_t)obs);
    }
    const double4 pa = fpos[f];
    float4        pa32;
    if constexpr(PRE32)
        pa32 = fpos32[f];
    for(int large = 0; large < 2; ++large)
    {
        // the fine cells of the box [x - reach, x + reach]
        const double   reach = (pa.w + (large ? g.rmax : g.rs)) * (1.0 + 1e-6) + 1e-6 * g.h;
        const uint32_t base  = large ? nf : 0u;
        const uint32_t x0    = fine_axis(pa.x - reach, g.mn[0], g.h, g.nx);
        const uint32_t x1    = fine_axis(pa.x + reach, g.mn[0], g.h, g.nx);
        const uint32_t y0    = fine_axis(pa.y - reach, g.mn[1], g.h, g.ny);
        const uint32_t y1    = fine_axis(pa.y + reach, g.mn[1], g.h, g.ny);
        const uint32_t z0    = fine_axis(pa.z - reach, g.mn[2], g.h, g.nz);
        const uint32_t z1    = fine_axis(pa.z + reach, g.mn[2], g.h, g.nz);
        // the rows (z, y) of the box, 32 at a time, lane i holding row i of
        // the chunk, walked as one sequence
        const uint32_t wy = y1 - y0 + 1, rows = (z1 - z0 + 1) * wy;
        for(uint32_t c0 = 0; c0 < rows; c0 += 32)
        {
            uint32_t t0 = 0, t1 = 0;
            if(c0 + lane < rows)
            {
                const uint32_t z   = z0 + (c0 + lane) / wy, y = y0 + (c0 + lane) % wy;
                const uint32_t row = base + (z * g.ny + y) * g.nx;
                t0                 = fstart[row + x0];
                t1                 = fstart[row + x1 + 1];
                if(large && t0 < (uint32_t)f + 1)
                    t0 = (uint32_t)f + 1; // each large pair once
            }
            warp_ranges(t0, t1, [&](uint32_t t, bool valid) {
                if(!valid)
                    return;
                if constexpr(PRE32)
                    if(pretest_rejects<PRE32>(pa32, fpos32[t]))
                        return;
                if(exact_hit<STRICT>(pa, fpos[t]))
                    record_pair(sa, a, fref[t], fids[t], count, pslot, slot);
            });
        }
    }
}

// Ascending sort of t[0, N) in registers by a bitonic network (Batcher, 1968):
// every index is a compile-time constant once unrolled.
template <int N, int M>
GB_D void bitonic_sort(uint32_t (&t)[M])
{
    static_assert(N <= M && (N & (N - 1)) == 0, "a power of two within the array");
#pragma unroll
    for(int k = 2; k <= N; k <<= 1)
#pragma unroll
        for(int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for(int i = 0; i < N; ++i)
            {
                const int l = i ^ j;
                if(l > i)
                {
                    const uint32_t x = t[i], y = t[l];
                    const uint32_t lo = min(x, y), hi = max(x, y);
                    const bool     up = (i & k) == 0;
                    t[i]              = up ? lo : hi;
                    t[l]              = up ? hi : lo;
                }
            }
}

// Fill pass, one thread per particle id a (most have no candidate and read
// only count[a]): the pair records of a at offset[a] -- its particle
// candidates from the slots of its sorted position s = sorted_of[a], sorted
// ascending (the enumeration order), or enumerated again in order when there
// were more than kPairSlots -- then its obstacle candidates.
template <typename S>
__global__ void __launch_bounds__(kBlock)
    k_pair_fill(int n, const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ sids,
                const uint32_t* __restrict__ sorted_of, const double4* __restrict__ spos,
                const float4* __restrict__ spos32, const uint32_t* __restrict__ cstart,
                uint32_t nx, uint32_t ny, uint32_t nz, uint32_t* __restrict__ count,
                const uint32_t* __restrict__ slot, ObsCand oc,
                const uint32_t* __restrict__ offset, uint32_t* __restrict__ pair_a,
                uint32_t* __restrict__ pair_b, int64_t cap, int* __restrict__ flags,
                uint32_t* __restrict__ gjk_count, uint32_t* __restrict__ pslot,
                uint32_t* __restrict__ ovf_list, int ovf_phase, uint32_t* __restrict__ obs_queue)
{
    grid_dep_sync();
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if(a == 0)
    {
        // the narrow phase's GJK queues of this step start empty: [0] the
        // cull pass's, [1] the mixed mode's FP32 stage's; [2 + phase] counts
        // this step's overflowing particles and [4 + phase] its obstacle
        // records, [3 - phase] and [5 - phase] (last step's, read by its
        // overflow and obstacle passes) start the next step at zero
        gjk_count[0]             = 0;
        gjk_count[1]             = 0;
        gjk_count[3 - ovf_phase] = 0;
        gjk_count[5 - ovf_phase] = 0;
    }
    if(a >= n || step_aborted(flags))
        return;
    const uint32_t c = count[a];
    if(c == 0)
        return;
    const int s = (int)sorted_of[a];
    int64_t out = offset[a];
    if(out + c > cap)
    {
        atomicOr(flags, kFlagCapacity);
        return;
    }
    // the count pass's counters start the next step at zero (an aborted step
    // leaves them for the host's memset before its replay)
    count[a] = 0u;
    pslot[s] = 0u;
    const uint32_t cp = c - (uint32_t)obstacle_candidates(oc, a, (uint32_t)s);
    if(cp <= kPairSlots)
    {
        // the slots in registers (unused ones as 0xffffffff, above every
        // sorted position), sorted with static indices only, so nothing goes
        // to local memory
        const uint4* mine = reinterpret_cast<const uint4*>(slot + (size_t)s * kPairSlots);
        uint32_t     t[kPairSlots];
#pragma unroll
        for(int q = 0; q < kPairSlots / 4; ++q)
        {
            uint4 x = make_uint4(~0u, ~0u, ~0u, ~0u);
            if((uint32_t)(4 * q) < cp)
                x = mine[q];
            t[4 * q]     = (uint32_t)(4 * q) < cp ? x.x : ~0u;
            t[4 * q + 1] = (uint32_t)(4 * q + 1) < cp ? x.y : ~0u;
            t[4 * q + 2] = (uint32_t)(4 * q + 2) < cp ? x.z : ~0u;
            t[4 * q + 3] = (uint32_t)(4 * q + 3) < cp ? x.w : ~0u;
        }
        // a bitonic network over the warp's largest count (rounded up to 8,
        // 16 or 32 slots): one code path per warp, ~80 compare-exchanges for
        // the common 16 instead of 32 x 32 rank comparisons
        const uint32_t wmax = __reduce_max_sync(__activemask(), cp);
        if(wmax <= 8)
            bitonic_sort<8>(t);
        else if(wmax <= 16)
            bitonic_sort<16>(t);
        else
            bitonic_sort<kPairSlots>(t);
#pragma unroll
        for(int k = 0; k < kPairSlots; ++k)
            if((uint32_t)k < cp)
            {
                pair_a[out + k] = a;
                pair_b[out + k] = sids[t[k]];
            }
        out += cp;
    }
    else
    {
        // more partners than slots (the largest grains of a polydisperse
        // packing): k_pair_fill_overflow writes them, a warp per particle
        ovf_list[atomicAdd(gjk_count + 2 + ovf_phase, 1u)] = (uint32_t)a;
        out += cp;
    }
    // the particle's obstacle records, contiguous after its particle pairs,
    // into the obstacle pass's queue
    const uint32_t k_obs = c - cp;
    if(k_obs)
    {
        const uint32_t q = atomicAdd(gjk_count + 4 + ovf_phase, k_obs);
        for(uint32_t j = 0; j < k_obs; ++j)
            obs_queue[q + j] = (uint32_t)out + j;
    }
    for_each_obstacle_candidate(oc, a, (uint32_t)s, [&](uint32_t o) {
        pair_a[out] = a;
        pair_b[out] = kObstacleBit | o;
        ++out;
    });
}

// The particle pairs of the particles whose partners overflowed their slots,
// one warp per particle: the 27 cells in the reference's order (as
// for_each_candidate walks them), 32 candidates a round, the hits of a round
// written in lane order (ballot + prefix count), so the list is the one
// for_each_candidate writes.
template <typename S>
__global__ void __launch_bounds__(128)
    k_pair_fill_overflow(const uint32_t* __restrict__ ovf_count,
                         const uint32_t* __restrict__ ovf_list, const uint32_t* __restrict__ skeys,
                         const uint32_t* __restrict__ sids, const uint32_t* __restrict__ sorted_of,
                         const double4* __restrict__ spos, const float4* __restrict__ spos32,
                         const uint32_t* __restrict__ cstart, uint32_t nx, uint32_t ny, uint32_t nz,
                         const uint32_t* __restrict__ offset, uint32_t* __restrict__ pair_a,
                         uint32_t* __restrict__ pair_b, const int* __restrict__ flags)
{
    grid_dep_sync();
    constexpr bool STRICT = is_strict<S>(), PRE32 = is_mixed<S>();
    if(step_aborted(flags))
        return;
    const unsigned lane  = threadIdx.x & 31u;
    const uint32_t total = *ovf_count;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    for(uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) / 32; w < total; w += warps)
    {
        const uint32_t a   = ovf_list[w];
        const uint32_t s   = sorted_of[a];
        uint32_t       out = offset[a];
        const uint32_t key = skeys[s];
        const double4  pa  = spos[s];
        float4         pa32;
        if constexpr(PRE32)
            pa32 = spos32[s];
        const int cx = key % nx, cy = (key / nx) % ny, cz = key / (nx * ny);
        // the 9 rows of 3 cells, lane r holding row r, walked as one sequence
        uint32_t t0 = 0, t1 = 0;
        if(lane < 9)
            neighbour_row(cstart, nx, ny, nz, cx, cy, cz, (int)lane, t0, t1);
        warp_ranges(t0, t1, [&](uint32_t t, bool valid) {
            bool hit = valid && t != s;
            if constexpr(PRE32)
                hit = hit && !pretest_rejects<PRE32>(pa32, spos32[t]);
            hit                 = hit && exact_hit<STRICT>(pa, spos[t]);
            const unsigned bits = __ballot_sync(0xffffffffu, hit);
            if(hit)
            {
                const uint32_t k = out + __popc(bits & ((1u << lane) - 1u));
                pair_a[k]        = a;
                pair_b[k]        = sids[t];
            }
            out += __popc(bits);
        });
    }
}

// ---- narrow phase + contact law, one thread per candidate pair ---------------
template <typename St>
struct PairOut
{
    St*      f[3];
    St*      t[3];
    St*      m[3];     // rolling moment (only when some kr != 0)
    uint8_t* contact;  // kContactParticle / kContactObstacle when overlap < 0, else 0
    uint32_t* pcount;  // contacts per particle id (zero before the narrow phase; the
                       // per-particle kernel reads and clears them)
    double*  info;     // optional: 7 per pair (point, vector, overlap) in world frame
    // tangential history (history law): current step out, previous step in
    St*             xi[3];
    const uint32_t* prev_off;
    const uint32_t* prev_b;
    const St*       prev_xi[3];
};

// the outputs of pair p: force, torque, rolling moment, spring, contact flag,
// and (when recorded) the contact point in world frame, vector and overlap
template <typename S>
GB_D void store_pair(const PairOut<store_t<S>>& po, int64_t p, const Force<S>& F,
                     const V3<S>& xi_new, uint8_t flag, int law_kind, int has_kr,
                     const Contact<S>& ci, const double xa[3])
{
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        const S fk[3] = {F.f.x, F.f.y, F.f.z}, tk[3] = {F.t.x, F.t.y, F.t.z};
        po.f[k][p] = (store_t<S>)to_d(fk[k]);
        po.t[k][p] = (store_t<S>)to_d(tk[k]);
    }
    if(has_kr)
    {
        po.m[0][p] = (store_t<S>)to_d(F.m.x);
        po.m[1][p] = (store_t<S>)to_d(F.m.y);
        po.m[2][p] = (store_t<S>)to_d(F.m.z);
    }
    if(law_kind != GB_LAW_HOOKE)
    {
        po.xi[0][p] = (store_t<S>)to_d(xi_new.x);
        po.xi[1][p] = (store_t<S>)to_d(xi_new.y);
        po.xi[2][p] = (store_t<S>)to_d(xi_new.z);
    }
    po.contact[p] = flag;
    if(po.info)
    {
        double* o = po.info + 7 * p;
        if constexpr(is_mixed<S>())
        {
            o[0] = xa[0] + to_d(ci.pt.x);
            o[1] = xa[1] + to_d(ci.pt.y);
            o[2] = xa[2] + to_d(ci.pt.z);
        }
        else
        {
            o[0] = to_d(ci.pt.x);
            o[1] = to_d(ci.pt.y);
            o[2] = to_d(ci.pt.z);
        }
        o[3] = to_d(ci.vec.x);
        o[4] = to_d(ci.vec.y);
        o[5] = to_d(ci.vec.z);
        o[6] = to_d(ci.overlap);
    }
}

// Pair p of particle a with obstacle o: closestPointsRigidBodies against the
// obstacle and the contact law with the obstacle at rest
// (ComponentManagerCPU.cpp:301-351).  The history law starts a fresh spring
// for obstacle contacts every step.  GEN: some obstacle is not a Rectangle
// and needs the general GJK (of variant VAR).
template <typename S, bool GEN, int VAR>
GB_D void narrow_obstacle(int64_t p, uint32_t a, int o, const State<store_t<S>>& st,
                          const Tables<S>& tb, const PairOut<store_t<S>>& po, int law_kind,
                          int has_kr, S dt, unsigned long long* counters)
{
    const uint32_t ra    = st.rb_id[a];
    const Body<S>  A     = load_body<S>(tb.shape, ra, tb.verts);
    const M3<S>    RA    = load_rot<S>(st, a);
    const double   xa[3] = {st.pos[0][a], st.pos[1][a], st.pos[2][a]};
    const double*  ot    = tb.obs_tr + 12 * o;
    const Body<S>  O     = load_body<S>(tb.obs_shape, o, tb.verts);
    V3<S>          oA, oO;
    M3<S>          RO;
    obstacle_frame(tb, o, xa, oA, oO, RO);
    int        iters = 0;
    Contact<S> ci    = no_contact<S>();
    if constexpr(is_mixed<S>())
    {
        if(O.type == GB_DRUM)
        {
            // the wall point nearest A's centre and its tangent plane, in FP64
            // relative to the centre; the FP32 pre-test, then the FP64 plane
            // contact as for Rectangles
            const V3<double> ax = mk<double>(ot[2], ot[5], ot[8]);
            const V3<double> d  = mk<double>(xa[0] - ot[9], xa[1] - ot[10], xa[2] - ot[11]);
            const V3<double> r  = d - dot(ax, d) * ax;
            const double     nr = norm(r), R = tb.obs_shape64[o].p[0];
            if(nr > 1e-12 * R)
            {
                const V3<double> e  = (1.0 / nr) * r;
                const V3<double> w  = (R - nr) * e; // the wall point, from A's centre
                const V3<S>      e32 = cvt3<S>(e);
                const V3<S>      pA  = mul(RA, support(A, mul_t(RA, e32)));
                if(S(R - nr) - dot(e32, pA) < S(1e-6))
                {
                    const Body<double> A64  = load_body<double>(tb.shape64, ra, tb.verts64);
                    const M3<double>   RA64 = load_rot64(st, a);
                    ci = to_f(closest_rectangle(A64, RA64, zero3<double>(), w, -e));
                }
            }
        }
        else if(O.type == GB_RECTANGLE)
        {
            // FP32 first; a contact (or a near miss within the rounding
            // margin) is recomputed in FP64 relative to the particle centre
            const V3<S> rn  = mk<S>(RO.m[2], RO.m[5], RO.m[8]);
            const V3<S> rnA = s_copysign(S(1.0), dot(rn, oA - oO)) * rn;
            const V3<S> pA  = mul(RA, support(A, mul_t(RA, -rnA)));
            const S     sep = dot(rnA, pA - oO);
            if(sep < S(1e-6))
            {
                const Body<double> A64  = load_body<double>(tb.shape64, ra, tb.verts64);
                const M3<double>   RA64 = load_rot64(st, a);
                const V3<double>   oO64 = mk<double>(ot[9] - xa[0], ot[10] - xa[1], ot[11] - xa[2]);
                ci = to_f(closest_rectangle(A64, RA64, zero3<double>(), oO64,
                                            mk<double>(ot[2], ot[5], ot[8])));
            }
        }
        else if constexpr(GEN)
            ci = closest_points<VAR>(A, O, RA, RO, oA, oO, oO - oA, &iters);
    }
    else if(O.type == GB_RECTANGLE)
        ci = closest_rectangle(A, RA, oA, oO, mk<S>(RO.m[2], RO.m[5], RO.m[8]));
    else if(O.type == GB_DRUM)
        ci = closest_drum(A, RA, oA, oO, mk<S>(RO.m[2], RO.m[5], RO.m[8]), O.p[0]);
    else if constexpr(GEN)
        ci = closest_points<VAR>(A, O, RA, RO, oA, oO, oO - oA, &iters);
    const bool hit = ci.overlap < S(0.0);
    Force<S>   F;
    F.f = F.t = F.m = zero3<S>();
    if(hit)
    {
        const Law<S> L  = load_law<S>(tb.law, tb.shape[ra].material, tb.obs_shape[o].material);
        const S      m1 = S(tb.inertia[ra].mass);
        const S      m2 = S(tb.obs_mass[o]);
        const V3<S>  vA = load3<S>(st.vel, a), wA = load3<S>(st.omg, a);
        V3<S>        arm, ptw, armO;
        if constexpr(is_mixed<S>())
        {
            arm  = ci.pt;
            ptw  = mk<S>(S(xa[0] + to_d(ci.pt.x)), S(xa[1] + to_d(ci.pt.y)), S(xa[2] + to_d(ci.pt.z)));
            armO = mk<S>(S(xa[0] - ot[9]), S(xa[1] - ot[10]), S(xa[2] - ot[11])) + ci.pt;
        }
        else
        {
            arm  = ci.pt - oA;
            ptw  = ci.pt;
            armO = ci.pt - oO;
        }
        // the wall's velocity at the contact point, v + w x (p - origin): zero
        // for the reference's walls at rest (ComponentManagerCPU.cpp:330-340)
        const double* ov  = tb.obs_vel + 6 * o;
        const V3<S>   wO  = mk<S>(S(ov[3]), S(ov[4]), S(ov[5]));
        const V3<S>   vOp = mk<S>(S(ov[0]), S(ov[1]), S(ov[2])) + cross(wO, armO);
        if(law_kind == GB_LAW_HOOKE)
        {
            const V3<S> rel = (vA + cross(wA, ptw)) - vOp;
            F               = hooke(L, ci, rel, wA - wO, m1, m2, arm);
        }
        else
        {
            V3<S> xi;
            F = hooke_history(L, ci, (vA + cross(wA, arm)) - vOp, m1, m2, dt, zero3<S>(), xi,
                              arm);
        }
        atomicAdd(&counters[0], 1ull);
    }
    store_pair<S>(po, p, F, zero3<S>(), hit ? kContactObstacle : uint8_t(0), law_kind, has_kr, ci,
                  xa);
    if(hit)
        atomicAdd(po.pcount + a, 1u);
    if(iters)
        atomicAdd(&counters[1], (unsigned long long)iters);
}

// particle pair record p (obstacle records are k_narrow_obstacles'); VAR: the GJK
// Whether a particle pair reaches GJK: the bounding tests of
// closestPointsRigidBodies (CollisionDetection.cpp:195-228) as closest_mixed
// and closest_points evaluate them -- not two spheres (closed form), bounding
// spheres overlapping, OBBs overlapping -- so that the GJK pass repeats
// exactly these decisions.
template <typename S>
GB_D bool needs_gjk(const Body<S>& A, const Body<S>& B, const M3<S>& RA, const M3<S>& RB,
                    const double xa[3], const double xb[3], const V3<S>& d)
{
    if(A.type == GB_SPHERE && B.type == GB_SPHERE)
        return false;
    if constexpr(is_mixed<S>())
    {
        const V3<double> d64 = mk<double>(xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]);
        const V3<float>  df  = cvt3<float>(d64);
        if(!(norm(df) - (A.rcirc + B.rcirc) < 0.0f))
            return false;
        return obb_overlap(A.bb, B.bb, RA, RB, df);
    }
    else
    {
        if(!(norm(d) - (A.rcirc + B.rcirc) < S(0.0)))
            return false;
        return obb_overlap(A.bb, B.bb, RA, RB, d);
    }
}

// The first iteration of GJK-JH (gjk_jh, GJK_JH.cpp:332-371), where it
// decides the pair on its own.  From v = sA(0) - b2a(sB(0)) and the first
// Minkowski support w = sA(-v) - b2a(sB(R^T v)), g = v.w / |v| is a lower
// bound on the distance of the cores, and GJK returns a distance of at
// least g wherever it stops (|v| of a point of the Minkowski difference).
// So:
//   g > crustA + crustB + margin: GJK's distance exceeds the crusts: no
//     contact;
//   g < -margin: mu stays 0 < the absolute tolerance, GJK stops at this
//     iteration and returns |v|; if that exceeds the crusts: no contact.
// Every other pair (in particular every contact) takes the full GJK.  The
// FP64 modes evaluate exactly GJK's first iteration, with a margin far
// above FP64 rounding; the mixed mode evaluates it in FP32 (supports,
// frames and dot products), with a margin of 1e-4 of the bounding radii,
// some 20 times a bound on the FP32 error of g (support values are
// Lipschitz in the direction with constant |x| <= R_circ, so the FP32
// direction error of ~3e-7 moves them by < 1e-9 m; the FP32 supports and
// frames add a few 1e-9 m): a pair decided here is one that the FP64 GJK
// also finds out of contact, so the mixed mode's contact set and contact
// geometry stay those of its FP64 GJK.
// The first rule holds for every GJK variant (each returns the norm of a
// point of the Minkowski difference, at least the true distance, which g
// bounds from below); the second is GJK-JH's own stopping rule (JH_RULE).
template <typename S, bool JH_RULE = true>
GB_D bool gjk_first_iteration_separates(const Body<S>& A, const Body<S>& B, const M3<S>& RA,
                                        const M3<S>& RB, const V3<S>& d)
{
    Tr<S>       b2a;
    const M3<S> RAt = transpose(RA);
    b2a.R           = mul(RAt, RB);
    b2a.o           = mul(RAt, d);
    const V3<S> s0A = support(A, zero3<S>()), s0B = support(B, zero3<S>());
    const V3<S> v   = s0A - apply(b2a, s0B);
    const S     dist = norm(v);
    const V3<S> pa = support_first(A, -v), qb = support_first(B, mul_t(b2a.R, v));
    const V3<S> w  = pa - apply(b2a, qb);
    const S     g  = dot(v, w) / dist;
    const S     ct = A.crust + B.crust;
    const S     margin = is_mixed<S>() ? S(1e-4) * (A.rcirc + B.rcirc) + S(1e-9)
                                       : S(1e-9) * (A.rcirc + B.rcirc) + S(1e-15);
    if(g > ct + margin)
        return true;
    return JH_RULE && g < -margin && dist - ct > margin;
}

// ---- the mixed mode's FP32 GJK stage ------------------------------------------
// Closest point to the origin of the segment (a, b) or the triangle (a, b, c)
// (Ericson, Real-Time Collision Detection, 5.1.2 and 5.1.5, by Voronoi
// regions), with the vertices of the feature it lies on put in y0..y(n-1).
// The vertices come by value: the callers pass the simplex they overwrite
// (with references, an edge (b, c) result read b after y1 = c had replaced
// it and returned c instead of the edge's closest point).
GB_D V3<float> closest_on_segment(const V3<float> a, const V3<float> b, V3<float>& y0,
                                  V3<float>& y1, int& n)
{
    const V3<float> ab = b - a;
    const float     t  = -dot(a, ab);
    if(t <= 0.0f)
    {
        y0 = a;
        n  = 1;
        return a;
    }
    const float den = dot(ab, ab);
    if(t >= den)
    {
        y0 = b;
        n  = 1;
        return b;
    }
    y0 = a;
    y1 = b;
    n  = 2;
    return a + (t / den) * ab;
}

GB_D V3<float> closest_on_triangle(const V3<float> a, const V3<float> b, const V3<float> c,
                                   V3<float>& y0, V3<float>& y1, V3<float>& y2, int& n)
{
    const V3<float> ab = b - a, ac = c - a;
    const float     d1 = -dot(ab, a), d2 = -dot(ac, a);
    if(d1 <= 0.0f && d2 <= 0.0f)
    {
        y0 = a;
        n  = 1;
        return a;
    }
    const float d3 = -dot(ab, b), d4 = -dot(ac, b);
    if(d3 >= 0.0f && d4 <= d3)
    {
        y0 = b;
        n  = 1;
        return b;
    }
    const float vc = d1 * d4 - d3 * d2;
    if(vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f)
    {
        y0 = a;
        y1 = b;
        n  = 2;
        return a + (d1 / (d1 - d3)) * ab;
    }
    const float d5 = -dot(ab, c), d6 = -dot(ac, c);
    if(d6 >= 0.0f && d5 <= d6)
    {
        y0 = c;
        n  = 1;
        return c;
    }
    const float vb = d5 * d2 - d1 * d6;
    if(vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f)
    {
        y0 = a;
        y1 = c;
        n  = 2;
        return a + (d2 / (d2 - d6)) * ac;
    }
    const float va = d3 * d6 - d5 * d4;
    if(va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f)
    {
        y0 = b;
        y1 = c;
        n  = 2;
        return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
    }
    const float den = 1.0f / (va + vb + vc);
    y0              = a;
    y1              = b;
    y2              = c;
    n               = 3;
    return a + (vb * den) * ab + (vc * den) * ac;
}

constexpr int kGjk32MaxIter = 24;

// For a pair that GJK's first iteration leaves open: GJK iterations in
// FP32 on at most a triangle (a new point added to a triangle keeps the
// nearest of the three faces through it), kept only for their support
// planes.  Any direction v and the Minkowski support w along -v give the
// lower bound v.w/|v| on the distance of the cores, whatever the simplex
// arithmetic did, with the FP32 error bound of gjk_first_iteration_separates.
// True: the largest bound exceeds the crusts by that margin, so the FP64 GJK
// finds no contact either.  False (the FP64 GJK decides): the iterates
// converged below the crusts (a contact or a near miss), reached the
// origin, left the finite range, or ran out of iterations.
GB_D bool gjk_fp32_separates(const Body<float>& A, const Body<float>& B, const M3<float>& RA,
                             const M3<float>& RB, const V3<float>& d)
{
    Tr<float>       b2a;
    const M3<float> RAt = transpose(RA);
    b2a.R               = mul(RAt, RB);
    b2a.o               = mul(RAt, d);
    const float ct      = A.crust + B.crust;
    const float margin  = 1e-4f * (A.rcirc + B.rcirc) + 1e-9f;
    V3<float>   y0 = support(A, zero3<float>()) - apply(b2a, support(B, zero3<float>()));
    V3<float>   y1 = y0, y2 = y0;
    int         n  = 1;
    V3<float>   v  = y0;
    float       mu = -INFINITY;
    for(int k = 0; k < kGjk32MaxIter; ++k)
    {
        const float vv = dot(v, v);
        if(!(vv > 1e-30f))
            return false;
        const V3<float> w = support_first(A, -v)
                            - apply(b2a, support_first(B, mul_t(b2a.R, v)));
        const float vw = dot(v, w);
        const float nv = sqrtf(vv);
        const float g  = vw / nv;
        if(!(g == g))
            return false;
        mu = fmaxf(mu, g);
        if(mu > ct + margin)
            return true;
        if(nv - mu <= margin || vv - vw <= 1e-6f * vv)
            return false;
        if(n == 1)
            v = closest_on_segment(y0, w, y0, y1, n);
        else if(n == 2)
            v = closest_on_triangle(y0, y1, w, y0, y1, y2, n);
        else
        {
            // the faces of the tetrahedron through w: the nearest one
            V3<float>       a0, a1, a2, b0, b1, b2, c0, c1, c2;
            int             na, nb, nc;
            const V3<float> pa = closest_on_triangle(w, y0, y1, a0, a1, a2, na);
            const V3<float> pb = closest_on_triangle(w, y1, y2, b0, b1, b2, nb);
            const V3<float> pc = closest_on_triangle(w, y0, y2, c0, c1, c2, nc);
            const float     da = dot(pa, pa), db = dot(pb, pb), dc = dot(pc, pc);
            if(da <= db && da <= dc)
            {
                v  = pa;
                y0 = a0;
                y1 = a1;
                y2 = a2;
                n  = na;
            }
            else if(db <= dc)
            {
                v  = pb;
                y0 = b0;
                y1 = b1;
                y2 = b2;
                n  = nb;
            }
            else
            {
                v  = pc;
                y0 = c0;
                y1 = c1;
                y2 = c2;
                n  = nc;
            }
        }
    }
    return false;
}

// Pair record p: contact detection, contact law, outputs.  QUEUE (the cull
// pass, k_narrow): the pair is finished here when it is two spheres (closed
// form) or out of contact by the bounding tests or GJK-JH's first iteration,
// and queued for the GJK pass otherwise -- no GJK is compiled into this
// pass, which keeps its registers low.  Without QUEUE (k_narrow_gjk): the
// full closestPointsRigidBodies.
template <typename S, int VAR, bool QUEUE = false>
GB_D void narrow_pair(int64_t p, const uint32_t* __restrict__ pair_a,
                      const uint32_t* __restrict__ pair_b, const State<store_t<S>>& st,
                      const Tables<S>& tb, const PairOut<store_t<S>>& po, int law_kind, int has_kr,
                      S dt, unsigned long long* __restrict__ counters,
                      uint32_t* __restrict__ gjk_queue = nullptr,
                      uint32_t* __restrict__ gjk_count = nullptr)
{
    const uint32_t a = pair_a[p], b = pair_b[p];
    if(b & kObstacleBit) // k_narrow_obstacles
        return;
    const uint32_t ra = st.rb_id[a], rb = st.rb_id[b];
    const Body<S>  A = load_body<S>(tb.shape, ra, tb.verts);
    const Body<S>  B = load_body<S>(tb.shape, rb, tb.verts);
    const M3<S>    RA = load_rot<S>(st, a), RB = load_rot<S>(st, b);
    const double   xa[3] = {st.pos[0][a], st.pos[1][a], st.pos[2][a]};
    const double   xb[3] = {st.pos[0][b], st.pos[1][b], st.pos[2][b]};
    V3<S>          oA, oB, d;
    if constexpr(is_mixed<S>())
    {
        d  = mk<S>(S(xb[0] - xa[0]), S(xb[1] - xa[1]), S(xb[2] - xa[2]));
        oA = zero3<S>();
        oB = d;
    }
    else
    {
        oA = mk<S>(S(xa[0]), S(xa[1]), S(xa[2]));
        oB = mk<S>(S(xb[0]), S(xb[1]), S(xb[2]));
        d  = oB - oA;
    }
    int        iters = 0;
    Contact<S> ci;
    if constexpr(QUEUE)
    {
        constexpr bool JH = (VAR & ~kGjkPaired) == GB_GJK_JH;
        if(A.type == GB_SPHERE && B.type == GB_SPHERE)
        {
            if constexpr(is_mixed<S>())
                ci = closest_spheres_mixed(tb, ra, rb, xa, xb);
            else
                ci = closest_spheres(A, B, oA, oB);
        }
        else if(!needs_gjk<S>(A, B, RA, RB, xa, xb, d)
                || (JH && gjk_first_iteration_separates<S, true>(A, B, RA, RB, d))
                || (!JH && is_mixed<S>()
                    && gjk_first_iteration_separates<S, false>(A, B, RA, RB, d)))
            ci = no_contact<S>();
        else
        {
            // the GJK pass (k_narrow_gjk) takes this pair and stores its outputs
            gjk_queue[atomicAdd(gjk_count, 1u)] = (uint32_t)p;
            return;
        }
    }
    else if constexpr(is_mixed<S>())
        ci = closest_mixed<VAR>(tb, st, a, b, ra, rb, A, B, RA, RB, xa, xb, &iters);
    else
        ci = closest_points<VAR>(A, B, RA, RB, oA, oB, d, &iters);
    const bool hit = ci.overlap < S(0.0);
    Force<S>         F;
    F.f = F.t = F.m = zero3<S>();
    V3<S> xi_new    = zero3<S>();
    if(hit)
    {
        const Law<S> L  = load_law<S>(tb.law, tb.shape[ra].material, tb.shape[rb].material);
        const S      m1 = S(tb.inertia[ra].mass), m2 = S(tb.inertia[rb].mass);
        const V3<S>  vA = load3<S>(st.vel, a), vB = load3<S>(st.vel, b);
        const V3<S>  wA = load3<S>(st.omg, a), wB = load3<S>(st.omg, b);
        // arm = contact point - A's centre
        V3<S> arm, ptw;
        if constexpr(is_mixed<S>())
        {
            arm = ci.pt;
            ptw = mk<S>(S(xa[0] + to_d(ci.pt.x)), S(xa[1] + to_d(ci.pt.y)),
                        S(xa[2] + to_d(ci.pt.z)));
        }
        else
        {
            arm = ci.pt - oA;
            ptw = ci.pt;
        }
        if(law_kind == GB_LAW_HOOKE)
        {
            // Kinematics::kinematicsAtPoint with the absolute contact point
            const V3<S> rel = (vA + cross(wA, ptw)) - (vB + cross(wB, ptw));
            F               = hooke(L, ci, rel, wA - wB, m1, m2, arm);
        }
        else
        {
            const V3<S> armB = is_mixed<S>() ? ci.pt - d : ci.pt - oB;
            const V3<S> rel  = (vA + cross(wA, arm)) - (vB + cross(wB, armB));
            V3<S>       xi_prev = zero3<S>();
            for(uint32_t k = po.prev_off[a]; k < po.prev_off[a + 1]; ++k)
                if(po.prev_b[k] == b)
                {
                    xi_prev = mk<S>(S(po.prev_xi[0][k]), S(po.prev_xi[1][k]), S(po.prev_xi[2][k]));
                    break;
                }
            F = hooke_history(L, ci, rel, m1, m2, dt, xi_prev, xi_new, arm);
        }
    }
    // a lane pair (kGjkPaired) holds the same results: its even lane stores them
    if((VAR & kGjkPaired) && (threadIdx.x & 1u))
        return;
    store_pair<S>(po, p, F, xi_new, hit ? kContactParticle : uint8_t(0), law_kind, has_kr, ci, xa);
    if(hit)
        atomicAdd(po.pcount + a, 1u);
    if(iters)
        atomicAdd(&counters[1], (unsigned long long)iters);
}

// The pair records of a narrow-phase launch, p in [0, npairs).  A list longer
// than the grid is walked with a grid stride (consecutive records in
// consecutive lanes).  A shorter one -- the common case of a loose packing,
// a few thousand candidates -- is spread over all warps, ceil(npairs / warps)
// consecutive records per warp: one thread's GJK is a long dependent chain,
// and the divergent chains of a warp run one after the other, so the step
// waits for the warp with the most records, not for the longest chain alone.
template <typename F>
GB_D void for_each_pair(int64_t npairs, F&& f)
{
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid      = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(npairs < nthreads)
    {
        const int64_t nwarps = nthreads >> 5;
        const int64_t k      = (npairs + nwarps - 1) / nwarps; // <= 32
        const int64_t lane   = threadIdx.x & 31;
        const int64_t p      = (tid >> 5) * k + lane;
        if(lane < k && p < npairs)
            f(p);
    }
    else
        for(int64_t p = tid; p < npairs; p += nthreads)
            f(p);
}

// The particle-particle narrow phase in two passes.  k_narrow walks the pair
// list (its length is read on the device, *total, the scan's grand total, so
// the host launches a resident-sized grid without waiting for it): every
// pair that its bounding tests cull, and every sphere pair, is finished
// there; a pair that needs GJK goes to a queue instead.  k_narrow_gjk then
// spreads the queue -- a few hundred to a few thousand pairs -- over all
// resident warps, so that a warp holds one or two GJK chains rather than
// every GJK pair among 32 consecutive records of the list.
template <typename S, int VAR>
__global__ void __launch_bounds__(128, sizeof(store_t<S>) == 4 ? 5 : 1)
    k_narrow(const uint32_t* __restrict__ total, const int* __restrict__ flags,
             const uint32_t* __restrict__ pair_a, const uint32_t* __restrict__ pair_b,
             State<store_t<S>> st, Tables<S> tb, PairOut<store_t<S>> po, int law_kind, int has_kr,
             S dt, unsigned long long* __restrict__ counters, uint32_t* __restrict__ gjk_queue,
             uint32_t* __restrict__ gjk_count)
{
    grid_dep_sync();
    if(step_aborted(flags))
        return;
    for_each_pair(*total, [&](int64_t p) {
        narrow_pair<S, VAR, true>(p, pair_a, pair_b, st, tb, po, law_kind, has_kr, dt, counters,
                            gjk_queue, gjk_count);
    });
}

// The mixed mode's FP32 stage over the cull pass's queue: a pair that
// gjk_fp32_separates decides is finished here (no contact, the outputs the
// FP64 GJK would store), the others go to the FP64 GJK's queue.
__global__ void __launch_bounds__(128)
    k_narrow_gjk32(const uint32_t* __restrict__ gjk_count, const int* __restrict__ flags,
                   const uint32_t* __restrict__ gjk_queue, const uint32_t* __restrict__ pair_a,
                   const uint32_t* __restrict__ pair_b, State<float> st, Tables<float> tb,
                   PairOut<float> po, int law_kind, int has_kr, uint32_t* __restrict__ queue64,
                   uint32_t* __restrict__ count64)
{
    grid_dep_sync();
    if(step_aborted(flags))
        return;
    for_each_pair(*gjk_count, [&](int64_t q) {
        const uint32_t    p = gjk_queue[q];
        const uint32_t    a = pair_a[p], b = pair_b[p];
        const uint32_t    ra = st.rb_id[a], rb = st.rb_id[b];
        const Body<float> A  = load_body<float>(tb.shape, ra, tb.verts);
        const Body<float> B  = load_body<float>(tb.shape, rb, tb.verts);
        const M3<float>   RA = load_rot<float>(st, a), RB = load_rot<float>(st, b);
        const V3<float>   d  = mk<float>(float(st.pos[0][b] - st.pos[0][a]),
                                         float(st.pos[1][b] - st.pos[1][a]),
                                         float(st.pos[2][b] - st.pos[2][a]));
        if(gjk_fp32_separates(A, B, RA, RB, d))
        {
            const double xa[3] = {st.pos[0][a], st.pos[1][a], st.pos[2][a]};
            Force<float> F;
            F.f = F.t = F.m = zero3<float>();
            store_pair<float>(po, p, F, zero3<float>(), uint8_t(0), law_kind, has_kr,
                              no_contact<float>(), xa);
        }
        else
            queue64[atomicAdd(count64, 1u)] = p;
    });
}

// One queued pair per lane pair (kGjkPaired: the two supports of a GJK
// iteration in parallel); a short queue is spread over all warps as in
// for_each_pair, a long one walked with a stride.  Both lanes of a pair take
// the same path throughout, so their shuffles always meet.  MIN_BLOCKS > 1
// caps its registers for more resident warps (Johnson's tables and some
// values spill to local memory): faster where the supports are closed forms
// (superquadrics) and the queue outnumbers the default's lane pairs, slower
// where they loop over polyhedron vertices or one round takes the queue.
// The launch does its work only for a queue length in [min_queue,
// max_queue), read on the device, so that the host can launch both forms
// and let the queue pick one.
template <typename S, int VAR, int MIN_BLOCKS = 1>
__global__ void __launch_bounds__(128, MIN_BLOCKS)
    k_narrow_gjk(const uint32_t* __restrict__ gjk_count, const int* __restrict__ flags,
                 const uint32_t* __restrict__ gjk_queue, const uint32_t* __restrict__ pair_a,
                 const uint32_t* __restrict__ pair_b, State<store_t<S>> st, Tables<S> tb,
                 PairOut<store_t<S>> po, int law_kind, int has_kr, S dt,
                 unsigned long long* __restrict__ counters, uint32_t min_queue,
                 uint32_t max_queue)
{
    grid_dep_sync();
    if(step_aborted(flags))
        return;
    const int64_t nq     = *gjk_count;
    if(nq < (int64_t)min_queue || nq >= (int64_t)max_queue)
        return;
    const int64_t nslots = ((int64_t)gridDim.x * blockDim.x) >> 1;
    const int64_t slot   = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 1;
    auto          one    = [&](int64_t q) {
        narrow_pair<S, VAR | kGjkPaired>(gjk_queue[q], pair_a, pair_b, st, tb, po, law_kind,
                                         has_kr, dt, counters);
    };
    if(nq < nslots)
    {
        const int64_t nwarps = nslots >> 4;                 // 16 lane pairs per warp
        const int64_t k      = (nq + nwarps - 1) / nwarps;  // <= 16
        const int64_t pl     = (threadIdx.x & 31) >> 1;     // the lane pair within the warp
        const int64_t q      = (slot >> 4) * k + pl;
        if(pl < k && q < nq)
            one(q);
    }
    else
        for(int64_t q = slot; q < nq; q += nslots)
            one(q);
}

// ---- per-particle kernel -------------------------------------------------------
// PHASE_DETECT:  torce = sum of the particle's pair forces in enumeration
//                order, then obstacle contacts in obstacle order
//                (ComponentManagerCPU.cpp:356-423 then :301-351).
// PHASE_GRAVITY: torce.force += m g (ComponentManagerCPU.cpp:448-460).
// PHASE_MOVE:    integrate from the stored torce, then reset it
//                (ComponentManagerCPU.cpp:465-500).
// PHASE_STEP:    all three fused, no torce round trip.
enum Phase
{
    PHASE_DETECT  = 1,
    PHASE_GRAVITY = 2,
    PHASE_MOVE    = 4,
    PHASE_STEP    = 7
};

template <typename S>
struct StepParams
{
    S        dt;      // time step
    S        h;       // velocity kick of this move (dt; dt/2 on the first Verlet move)
    V3<S>    g;       // gravity
    int      integrator;
    int      law_kind;
    int      has_kr;
    int      phases;
    int      accumulate; // PHASE_DETECT adds to the stored torce instead of to zero
    int      rb_identity; // particle i's rigid body is body i
};

// The particle-obstacle records of the pair list, one thread per record, in a
// kernel of their own: the two kinds interleave in the list, and one kernel
// for both would run both code paths in every warp.
template <typename S, bool GEN, int VAR>
__global__ void __launch_bounds__(128)
    k_narrow_obstacles(const uint32_t* __restrict__ n_obs_records,
                       const uint32_t* __restrict__ obs_queue, const int* __restrict__ flags,
                       const uint32_t* __restrict__ pair_a, const uint32_t* __restrict__ pair_b,
                       State<store_t<S>> st, Tables<S> tb, PairOut<store_t<S>> po, int law_kind,
                       int has_kr, S dt, unsigned long long* __restrict__ counters)
{
    if(step_aborted(flags))
        return;
    // the step's obstacle records, queued by the fill pass
    for_each_pair(*n_obs_records, [&](int64_t q) {
        const uint32_t p = obs_queue[q];
        narrow_obstacle<S, GEN, VAR>(p, pair_a[p], (int)(pair_b[p] & ~kObstacleBit), st, tb, po,
                                     law_kind, has_kr, dt, counters);
    });
}

// ---- per-particle kernel: segmented sum, gravity, integration -----------------
// A latency-bound streaming kernel.  Its loads are all issued before the pair
// loop; the mixed instantiation runs four 256-thread blocks per SM at 64
// registers with a few spilled (measured 3% faster than three blocks at 79
// registers without, and than five at 48); the FP64 ones need about 125
// registers and get two blocks.
template <typename S>
__global__ void __launch_bounds__(kBlock, sizeof(store_t<S>) == 4 ? 4 : 2)
    k_particles(int n, State<store_t<S>> st, Tables<S> tb, const uint32_t* __restrict__ off,
                PairOut<store_t<S>> po, StepParams<S> sp, int* __restrict__ contacts_out,
                uint32_t* __restrict__ mask_out, int* __restrict__ flags,
                unsigned int* __restrict__ done)
{
    grid_dep_sync();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n || step_aborted(flags))
        return;
    const uint32_t            r   = sp.rb_identity ? (uint32_t)i : st.rb_id[i];
    const RBInertia<store_t<S>>* in = tb.inertia + r;
    // the body record (mass, inertia, inverse inertia, box) in 16-byte loads
    store_t<S> rec[16];
    {
        constexpr int per = 16 / sizeof(store_t<S>);
        using Vec         = typename std::conditional<per == 4, float4, double2>::type;
        const Vec* v4     = reinterpret_cast<const Vec*>(in);
#pragma unroll
        for(int k = 0; k < 16 / per; ++k)
        {
            const Vec x = __ldg(v4 + k);
            if constexpr(per == 4)
            {
                rec[4 * k]     = x.x;
                rec[4 * k + 1] = x.y;
                rec[4 * k + 2] = x.z;
                rec[4 * k + 3] = x.w;
            }
            else
            {
                rec[2 * k]     = x.x;
                rec[2 * k + 1] = x.y;
            }
        }
    }
    const S                   m   = S(rec[0]);
    V3<S>                     F, T;
    V3<S>                     v = load3<S>(st.vel, i), w = load3<S>(st.omg, i);
    int                       nc = 0;
    // The pose and the body record do not depend on the pair loop: they are
    // loaded before it, and every store comes after all loads, so that these
    // loads and the loop's gathers are in flight together.
    const bool move = (sp.phases & PHASE_MOVE) != 0;
    S            I[6], I1[6];
    Quat<S>      q;
    float        qlo[4]; // mixed: the orientation's FP32 remainder (q + qlo is the orientation)
    M3<S>        R;
    double       x0[3];
    if(move)
    {
#pragma unroll
        for(int k = 0; k < 6; ++k)
        {
            I[k]  = S(rec[1 + k]);
            I1[k] = S(rec[7 + k]);
        }
        if constexpr(is_mixed<S>())
        {
            q.w = S(st.rot[0][i]);
            q.v = mk<S>(S(st.rot[1][i]), S(st.rot[2][i]), S(st.rot[3][i]));
#pragma unroll
            for(int k = 0; k < 4; ++k)
                qlo[k] = st.rot[4 + k][i];
        }
        else
            R = load_rot<S>(st, i);
#pragma unroll
        for(int k = 0; k < 3; ++k)
            x0[k] = st.pos[k][i];
    }
    if(sp.phases & PHASE_DETECT)
    {
        // Torce::addForce onto the torce accumulated since the last move
        // (zero unless set_torces, add_external_forces or a detect came first)
        if(sp.accumulate)
        {
            F = load3<S>(st.frc, i);
            T = load3<S>(st.trq, i);
        }
        else
        {
            F = zero3<S>();
            T = zero3<S>();
        }
        // the particle's pairs, then its obstacle pairs, in list order; most
        // particles have no contact (the narrow phase counts them) and skip
        // their list
        const uint32_t ncon = po.pcount[i];
        if(ncon)
            po.pcount[i] = 0u;
        for(uint32_t p = ncon ? off[i] : 0u, pe = ncon ? off[i + 1] : 0u; p < pe; ++p)
        {
            const uint8_t hit = po.contact[p];
            if(!hit)
                continue;
            nc += hit == kContactParticle;
            F = F + mk<S>(S(po.f[0][p]), S(po.f[1][p]), S(po.f[2][p]));
            T = T + mk<S>(S(po.t[0][p]), S(po.t[1][p]), S(po.t[2][p]));
            if(sp.has_kr)
                T = T + mk<S>(S(po.m[0][p]), S(po.m[1][p]), S(po.m[2][p]));
        }
    }
    else
    {
        F = load3<S>(st.frc, i);
        T = load3<S>(st.trq, i);
    }
    if(sp.phases & PHASE_GRAVITY)
        F = F + m * sp.g; // Torce::addForce(mass * g)
    if(move)
    {
        // RigidBody::computeMomentum + FirstOrderExplicit::Move
        // (RigidBody.cpp:267-307, FirstOrderExplicit.cpp:46-60) or the Verlet kick-drift
        if constexpr(!is_mixed<S>())
            q = quat_from_basis(R);
        const V3<S> acc   = mk<S>(F.x / m, F.y / m, F.z / m);
        const V3<S> alpha = angular_acceleration(I, I1, w, T, q);
        V3<S>       trans;
        Quat<S>     dq;
        if(sp.integrator == GB_FIRST_ORDER_EXPLICIT)
        {
            trans = sp.dt * v;
            v     = v + sp.dt * acc;
            dq    = quaternion_change(w, sp.dt);
            w     = w + sp.dt * alpha;
        }
        else
        {
            v     = v + sp.h * acc;
            w     = w + sp.h * alpha;
            trans = sp.dt * v;
            dq    = quaternion_change(w, sp.dt);
        }
        // Transform3::updateTransform (Transform3.cpp:324-329)
        double xn[3];
#pragma unroll
        for(int k = 0; k < 3; ++k)
        {
            const S tk[3] = {trans.x, trans.y, trans.z};
            if constexpr(is_mixed<S>())
                xn[k] = x0[k] + (double)tk[k];
            else
                xn[k] = to_d(S(x0[k]) + tk[k]);
            st.pos[k][i] = xn[k];
        }
        float hi[4]; // mixed: the new orientation's FP32 part
        if constexpr(is_mixed<S>())
        {
            // the increment from the FP32 angular velocity, composed with the
            // compensated orientation and renormalised in FP64
            Quat<double> dq64, q64;
            dq64.w          = (double)dq.w;
            dq64.v          = cvt3<double>(dq.v);
            q64.w           = (double)q.w + (double)qlo[0];
            q64.v           = mk<double>((double)q.v.x + (double)qlo[1], (double)q.v.y + (double)qlo[2],
                                         (double)q.v.z + (double)qlo[3]);
            Quat<double> qn = qmul(dq64, q64);
            const double rn = 1.0 / sqrt(qn.w * qn.w + norm2(qn.v));
            const double c[4] = {qn.w * rn, qn.v.x * rn, qn.v.y * rn, qn.v.z * rn};
#pragma unroll
            for(int k = 0; k < 4; ++k)
            {
                hi[k]            = (float)c[k];
                st.rot[k][i]     = hi[k];
                st.rot[4 + k][i] = (float)(c[k] - (double)hi[k]);
            }
        }
        else
        {
            compose_left_by_rotation(R, dq);
#pragma unroll
            for(int k = 0; k < 9; ++k)
                st.rot[k][i] = to_d(R.m[k]);
        }
        // the obstacle candidates of the next detect, from the new pose
        if(mask_out)
            mask_out[i] = obstacle_mask_at<S>(
                tb, r,
                [&] {
                    if constexpr(is_mixed<S>())
                        return quat_to_matrix<S>(hi[0], hi[1], hi[2], hi[3]);
                    else
                        return R;
                },
                xn);
        st.vel[0][i] = (store_t<S>)to_d(v.x);
        st.vel[1][i] = (store_t<S>)to_d(v.y);
        st.vel[2][i] = (store_t<S>)to_d(v.z);
        st.omg[0][i] = (store_t<S>)to_d(w.x);
        st.omg[1][i] = (store_t<S>)to_d(w.y);
        st.omg[2][i] = (store_t<S>)to_d(w.z);
        // a move that leaves a non-finite state is reported by its own step
        // (the next step's hash would report it one step late)
        if(!(isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]) && isfinite(to_d(v.x))
             && isfinite(to_d(v.y)) && isfinite(to_d(v.z)) && isfinite(to_d(w.x))
             && isfinite(to_d(w.y)) && isfinite(to_d(w.z))))
            atomicOr(flags, kFlagNonFinite);
        if(sp.phases != PHASE_STEP || sp.accumulate)
        {
            // Torce::reset
#pragma unroll
            for(int k = 0; k < 3; ++k)
            {
                st.frc[k][i] = store_t<S>(0);
                st.trq[k][i] = store_t<S>(0);
            }
        }
    }
    else
    {
        st.frc[0][i] = (store_t<S>)to_d(F.x);
        st.frc[1][i] = (store_t<S>)to_d(F.y);
        st.frc[2][i] = (store_t<S>)to_d(F.z);
        st.trq[0][i] = (store_t<S>)to_d(T.x);
        st.trq[1][i] = (store_t<S>)to_d(T.y);
        st.trq[2][i] = (store_t<S>)to_d(T.z);
    }
    if(contacts_out && (sp.phases & PHASE_DETECT))
        contacts_out[i] = nc;
    if(i == 0)
        atomicAdd(done, 1u); // the host counts the launches that completed
}

} // namespace gb
