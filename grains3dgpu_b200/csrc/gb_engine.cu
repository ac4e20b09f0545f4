// gb_engine.cu -- the C ABI of include/grains_b200.h: context, device memory,
// host<->device conversion of the Grains state layout, and the launch
// sequence of one time step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "gb_io.cuh"
#include "gb_adjoint.cuh"
#include "gb_step.cuh"
#include "gb_rawdata.cuh"

using namespace gb;

namespace
{

thread_local cudaError_t g_last_cuda = cudaSuccess;

#define GB_CK(x)                               \
    do                                         \
    {                                          \
        cudaError_t e_ = (x);                  \
        if(e_ != cudaSuccess)                  \
        {                                      \
            g_last_cuda = e_;                  \
            return e_ == cudaErrorMemoryAllocation ? GB_E_OUT_OF_MEMORY : GB_E_CUDA; \
        }                                      \
    } while(0)

#define GB_TRY(x)            \
    do                       \
    {                        \
        int st_ = (x);       \
        if(st_ != GB_OK)     \
            return st_;      \
    } while(0)

inline int blocks(int64_t n, int b)
{
    return (int)((n + b - 1) / b);
}

// Launches kernel k.  With pdl set, the launch is a programmatic dependent
// one: the GPU may schedule it while the stream's previous kernel drains, and
// the kernel's grid_dep_sync() holds it until that kernel has completed.
// Only kernels that call grid_dep_sync() first are launched this way, and only
// where their other dependencies are stream order (no cross-stream wait).
template <typename... P, typename... A>
cudaError_t launch(bool pdl, void (*k)(P...), int grid, int block, cudaStream_t s, A&&... args)
{
    cudaLaunchAttribute attr[1];
    attr[0].id                                         = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg                             = {};
    cfg.gridDim                                        = dim3((unsigned)grid);
    cfg.blockDim                                       = dim3((unsigned)block);
    cfg.dynamicSmemBytes                               = 0;
    cfg.stream                                         = s;
    cfg.attrs                                          = attr;
    cfg.numAttrs                                       = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

template <typename T>
int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if(count == 0)
        count = 1;
    GB_CK(cudaMalloc((void**)p, count * sizeof(T)));
    return GB_OK;
}

template <typename T>
void dfree(T*& p)
{
    if(p)
        cudaFree((void*)p);
    p = nullptr;
}

} // namespace

struct gb_ctx
{
    gb_config    cfg;
    int          prec = GB_FP64;
    cudaStream_t stream = nullptr;
    int          n = 0, nrb = 0, nob = 0, nmat = 0;
    bool         rb_set = false, law_set = false, ids_set = false, tr_set = false,
         vel_set = false, obs_set = false;
    // every particle has its own rigid body, id i for particle i: the
    // per-particle kernel reads body i without the dependent id load (off once
    // the ids' device array is handed out for writing)
    bool rb_identity = false;

    // host copies of the set-up
    std::vector<gb_rigid_body_desc>  rbs;
    std::vector<gb_rigid_body_props> props;
    std::vector<double>              verts;
    std::vector<gb_rigid_body_desc>  obs;
    std::vector<gb_rigid_body_props> obs_props;
    std::vector<double>              obs_tr;
    std::vector<gb_contact_model>    laws;
    bool                             has_kr = false;

    // linked cell
    double   cell = 0, lc_max[3] = {0, 0, 0};
    uint32_t dims[3] = {0, 0, 0};
    uint32_t ncells = 0;
    int      key_bits = 0;

    // device tables (storage type of the run mode)
    void*    d_shape = nullptr;
    void*    d_inertia = nullptr;
    void*    d_verts = nullptr;
    void*    d_law = nullptr;
    void*    d_obs_shape = nullptr;
    double*  d_obs_tr = nullptr;
    double*  d_obs_mass = nullptr;
    double4* d_obs_plane = nullptr; // Rectangle planes: normal, normal . origin
    uint32_t obs_rect    = 0u;      // bit o: obstacle o (< 32) is a Rectangle
    bool     obs_gjk     = false;   // some obstacle is neither a Rectangle nor a drum
    bool     poly_bodies = false;   // some rigid body is a polyhedron
    std::vector<double> obs_vel;    // 6 per obstacle: velocity, angular velocity
    double*  d_obs_vel   = nullptr;
    double*  d_rcirc64 = nullptr;
    double   rmax      = 0.0;     // the largest circumscribed radius (the candidate test's radius)
    // FP64 shape tables: aliases of the above in the FP64 modes, separate
    // copies in the mixed mode (read by its FP64 GJK)
    void* d_shape64 = nullptr;
    void* d_verts64 = nullptr;
    void* d_obs_shape64 = nullptr;

    // state
    double*   d_pos = nullptr; // 3n
    void*     d_rot = nullptr; // 9n (FP64) or 8n (mixed: quaternion hi, lo)
    void*     d_vel = nullptr; // 3n
    void*     d_omg = nullptr;
    void*     d_frc = nullptr;
    void*     d_trq = nullptr;
    uint32_t* d_rb_id = nullptr;
    bool      torce_dirty = false;

    // broad phase
    uint32_t *d_hash = nullptr, *d_iota = nullptr, *d_k[2] = {nullptr, nullptr},
             *d_i[2] = {nullptr, nullptr};
    uint32_t *d_skeys = nullptr, *d_sids = nullptr; // results (alias into d_k/d_i)
    uint32_t *d_hist = nullptr, *d_part = nullptr, *d_cstart = nullptr;
    uint32_t* d_ccount   = nullptr; // per-cell counts of the counting sort (C + 1)
    bool      count_zero = false;   // the fill pass leaves the candidate counts at zero
    bool      ccount_zero = false;   // the scatter pass leaves every count at zero
    bool      radix_sort = false;   // a crowded cell was seen: sort with the radix kernels
    bool      pdl        = true;    // programmatic dependent launches within a step
    double4*  d_spos = nullptr;
    float4*   d_spos32 = nullptr; // FP32 copy for the candidate pre-test
    uint32_t* d_slot   = nullptr; // kPairSlots candidates per particle (count pass)
    uint32_t* d_gjkq   = nullptr; // the step's pairs that need GJK (pair capacity; the
                                  // mixed mode: a second queue for its FP64 GJK after it)
    uint32_t* d_obsq   = nullptr; // the step's obstacle records (pair capacity)
    uint32_t* d_gjkn   = nullptr; // their numbers (reset by the fill pass)
    uint32_t* d_ovf    = nullptr; // particles with more partners than pair slots
    uint32_t* d_pcount = nullptr; // contacts per particle of the step (cleared as read)
    // obstacles past the mask's 32, binned by linked cell (obstacle_cells)
    uint32_t* d_cobs_start = nullptr;
    uint32_t* d_cobs_ids   = nullptr;
    bool      cobs_valid   = false;
    bool      cobs_used    = false; // lists built (some obstacle is not a masked wall)
    std::vector<uint32_t> h_cobs_ids;
    int64_t   cobs_entries = 0;
    int       ovf_phase = 0;      // which of d_gjkn[2], [3] counts them this step
    uint32_t* d_sorted_of = nullptr; // sorted position of each particle id
    // the finer candidate grid of polydisperse packings (k_pair_count_fine)
    bool      fine_planned = false, fine = false, fcount_zero = false;
    FineGrid  fine_g{};
    uint32_t  fine_nf = 0, fine_nlarge = 0;
    std::vector<uint32_t> h_rb_id; // the rigid-body ids as last set from the host
    uint32_t *d_fkey = nullptr, *d_fcount = nullptr, *d_fstart = nullptr, *d_fskey = nullptr,
             *d_fids = nullptr, *d_fref = nullptr;
    double4*  d_fpos   = nullptr;
    float4*   d_fpos32 = nullptr;
    uint32_t* d_obsmask_id = nullptr; // the same per particle id, from the last move
    bool      mask_valid   = false;   // d_obsmask_id matches the current poses
    size_t    part_cap = 0, hist_cap = 0;
    // one-pass scans: per-tile state words, the tile ticket counter, the
    // tickets taken so far and the epoch of the next scan
    unsigned long long* d_tile_state = nullptr;
    unsigned long long* d_ticket     = nullptr;
    size_t              tile_cap     = 0;
    unsigned long long  tickets      = 0;
    uint32_t            scan_epoch   = 0;
    uint32_t            scan_spin_limit = kScanSpinLimit; // GB_DEBUG_SCAN_SPIN_LIMIT
    int                 fine_mode       = -1; // GB_DEBUG_FINE_GRID: 0 off, 1 on, -1 by crowding

    // pairs (double-buffered for the tangential history)
    uint32_t* d_count = nullptr;
    uint32_t* d_off[2] = {nullptr, nullptr};
    uint32_t* d_pb[2] = {nullptr, nullptr};
    uint32_t* d_pa = nullptr;
    void*     d_pf = nullptr; // 9 * cap storage values: f, t, m
    uint8_t*  d_pc = nullptr;
    double*   d_info = nullptr;
    void*     d_xi[2] = {nullptr, nullptr}; // 3 * cap each
    int64_t   cap = 0;
    int64_t   cap_hint = 0; // capacity the next step allocates up front (grows after an overflow)
    int       cur = 0;
    int64_t   npairs = 0; // of the last detect (read back after it)
    int       sms    = 148; // multiprocessors of the context's device
    bool      have_prev = false;

    // counters and flags
    int*                d_flags = nullptr;
    unsigned long long* d_counters = nullptr; // [0] wall contacts [1] gjk iterations [2] contacts
    int*                d_contacts = nullptr;  // per-particle contact count of the last detect
    uint32_t*           h_pinned = nullptr;    // [0] pair total [1] flags [2] flags to restore
    int64_t             steps_done = 0;
    bool                verlet_started = false;
    bool                links_valid = false, detect_valid = false;
    bool                contacts_loaded = false; // gb_load_contacts: the next adjoint step's
    gb_stats            last{};

    cudaStream_t own_stream = nullptr; // the context's stream (gb_set_stream may replace it)
    // the particle-obstacle narrow phase runs beside the particle-particle
    // one: forked from the context's stream and joined back by these events
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t  ev_fork = nullptr, ev_join = nullptr;
    // phase timing: two alternating event sets; a set is read once the next
    // step's host synchronisation has passed it
    bool                 timing = false, in_step = false;
    static constexpr int kEvRing = 16; // steps whose phase events are kept until a sync
    cudaEvent_t          ev[kEvRing][GB_N_PHASES + 1];
    int                  ev_next = 0, ev_npending = 0;
    unsigned int*        d_done  = nullptr; // k_particles launches that completed (not aborted)
    double      phase_ms[GB_N_PHASES] = {0};
    int64_t     phase_steps = 0;
    int64_t     launches = 0;
    // staging buffer for the host layouts (12 doubles per particle)
    double* d_stage = nullptr;
    // adjoint scratch: force/torque adjoints (6n) and block partial sums
    double* d_adj   = nullptr;
    size_t  adj_cap = 0;
};

namespace
{

// event `idx` of the current step's set (0 = step start, k+1 = end of phase k)
void mark(gb_ctx* c, int idx)
{
    if(c->timing && c->in_step)
        cudaEventRecord(c->ev[c->ev_next][idx], c->stream);
}

// the current step's event set is complete: move to the next one
void close_event_set(gb_ctx* c)
{
    if(!c->timing)
        return;
    c->ev_next = (c->ev_next + 1) % gb_ctx::kEvRing;
    c->ev_npending++;
}

// adds the phase times of the steps recorded since the last call (at most
// the last kEvRing of them; call only after a host sync that follows them)
void accumulate_pending(gb_ctx* c)
{
    if(!c->timing || c->ev_npending == 0)
        return;
    const int m = std::min(c->ev_npending, gb_ctx::kEvRing);
    for(int j = 0; j < m; ++j)
    {
        const int set = (c->ev_next - m + j + gb_ctx::kEvRing) % gb_ctx::kEvRing;
        for(int k = 0; k < GB_N_PHASES; ++k)
        {
            float ms = 0.f;
            if(cudaEventElapsedTime(&ms, c->ev[set][k], c->ev[set][k + 1]) == cudaSuccess)
                c->phase_ms[k] += ms;
        }
        c->phase_steps++;
    }
    c->ev_npending = 0;
}

size_t store_size(int prec)
{
    return prec == GB_MIXED ? sizeof(float) : sizeof(double);
}

int rot_count(int prec)
{
    return prec == GB_MIXED ? 8 : 9; // mixed: quaternion hi (4) and lo (4)
}

template <typename St>
State<St> state_of(gb_ctx* c)
{
    State<St> s;
    const int n = c->n;
    for(int k = 0; k < 3; ++k)
    {
        s.pos[k] = c->d_pos + (size_t)k * n;
        s.vel[k] = (St*)c->d_vel + (size_t)k * n;
        s.omg[k] = (St*)c->d_omg + (size_t)k * n;
        s.frc[k] = (St*)c->d_frc + (size_t)k * n;
        s.trq[k] = (St*)c->d_trq + (size_t)k * n;
    }
    for(int k = 0; k < 9; ++k)
        s.rot[k] = k < rot_count(c->prec) ? (St*)c->d_rot + (size_t)k * n : nullptr;
    s.rb_id = c->d_rb_id;
    return s;
}

template <typename S>
Tables<S> tables_of(gb_ctx* c)
{
    using St = store_t<S>;
    Tables<S> t;
    t.shape     = (const RBShape<St>*)c->d_shape;
    t.inertia   = (const RBInertia<St>*)c->d_inertia;
    t.verts     = (const Vert<St>*)c->d_verts;
    t.law       = (const Law<St>*)c->d_law;
    t.obs_shape = (const RBShape<St>*)c->d_obs_shape;
    t.obs_tr      = c->d_obs_tr;
    t.obs_mass    = c->d_obs_mass;
    t.obs_plane   = c->d_obs_plane;
    t.obs_vel     = c->d_obs_vel;
    t.obs_rect    = c->obs_rect;
    t.n_obs       = c->nob;
    t.shape64     = (const RBShape<double>*)c->d_shape64;
    t.verts64     = (const Vert<double>*)c->d_verts64;
    t.obs_shape64 = (const RBShape<double>*)c->d_obs_shape64;
    return t;
}

bool crust_bounds(const gb_ctx* c) { return (c->cfg.flags & GB_FLAG_CRUST_BOUNDS) != 0; }

// the bounding radius of rigid body i in the candidate test and the cell size
double bound_radius(const gb_ctx* c, int i)
{
    return c->props[i].circumscribed_radius + (crust_bounds(c) ? c->rbs[i].crust_thickness : 0.0);
}

template <typename St>
RBShape<St> shape_record(const gb_rigid_body_desc& d, const gb_rigid_body_props& p,
                         bool crust_bounds)
{
    // the bounding tests' radius and half-extents (GB_FLAG_CRUST_BOUNDS)
    const double grow = crust_bounds ? d.crust_thickness : 0.0;
    RBShape<St> r;
    std::memset(&r, 0, sizeof(r));
    r.type       = d.convex.type;
    r.nverts     = d.convex.n_vertices;
    r.first_vert = d.convex.type == GB_POLYHEDRON ? d.convex.first_vertex : 0;
    for(int i = 0; i < 5; ++i)
        r.p[i] = (St)d.convex.p[i];
    if(d.convex.type == GB_SUPERQUADRIC)
    {
        const double a = d.convex.p[0], b = d.convex.p[1], c = d.convex.p[2],
                     n1 = d.convex.p[3], n2 = d.convex.p[4];
        r.k[0] = (St)(b / a);
        r.k[1] = (St)(c / a);
        r.k[2] = (St)(c / b);
        r.k[3] = (St)(1.0 / (n1 - 1.0));
        r.k[4] = (St)(1.0 / (n2 - 1.0));
        r.k[5] = (St)((n1 - n2) / (n2 * (n1 - 1.0)));
        r.k[6] = (St)(n1 / n2);
        r.k[7] = (St)(1.0 / n1);
    }
    r.crust    = (St)d.crust_thickness;
    r.rcirc    = (St)(p.circumscribed_radius + grow);
    for(int k = 0; k < 3; ++k)
        r.bb[k] = (St)(p.bounding_box[k] + grow);
    r.material = d.material;
    return r;
}

template <typename St>
int upload_tables(gb_ctx* c)
{
    std::vector<RBShape<St>>   sh(c->nrb);
    std::vector<RBInertia<St>> in(c->nrb);
    std::vector<double>        rc(c->nrb);
    for(int i = 0; i < c->nrb; ++i)
    {
        sh[i] = shape_record<St>(c->rbs[i], c->props[i], crust_bounds(c));
        std::memset(&in[i], 0, sizeof(in[i]));
        in[i].mass = (St)c->props[i].mass;
        for(int k = 0; k < 6; ++k)
        {
            in[i].I[k]  = (St)c->props[i].inertia[k];
            in[i].I1[k] = (St)c->props[i].inertia_inv[k];
        }
        for(int k = 0; k < 3; ++k)
            in[i].bb[k] = sh[i].bb[k];
        rc[i] = bound_radius(c, i);
    }
    const size_t nv = c->verts.size() / 3;
    std::vector<Vert<St>> vv(std::max<size_t>(nv, 1));
    for(size_t i = 0; i < nv; ++i)
        vv[i] = {(St)c->verts[3 * i], (St)c->verts[3 * i + 1], (St)c->verts[3 * i + 2], (St)0};
    dfree(c->d_shape);
    dfree(c->d_inertia);
    dfree(c->d_verts);
    dfree(c->d_rcirc64);
    GB_TRY(dalloc((RBShape<St>**)&c->d_shape, sh.size()));
    GB_TRY(dalloc((RBInertia<St>**)&c->d_inertia, in.size()));
    GB_TRY(dalloc((Vert<St>**)&c->d_verts, vv.size()));
    GB_TRY(dalloc(&c->d_rcirc64, rc.size()));
    GB_CK(cudaMemcpy(c->d_shape, sh.data(), sh.size() * sizeof(sh[0]), cudaMemcpyHostToDevice));
    GB_CK(cudaMemcpy(c->d_inertia, in.data(), in.size() * sizeof(in[0]), cudaMemcpyHostToDevice));
    GB_CK(cudaMemcpy(c->d_verts, vv.data(), vv.size() * sizeof(vv[0]), cudaMemcpyHostToDevice));
    GB_CK(cudaMemcpy(c->d_rcirc64, rc.data(), rc.size() * sizeof(double), cudaMemcpyHostToDevice));
    return GB_OK;
}

template <typename St>
int upload_laws(gb_ctx* c)
{
    const int         nl = c->nmat * (c->nmat + 1) / 2;
    std::vector<Law<St>> L(nl);
    c->has_kr = false;
    for(int i = 0; i < nl; ++i)
    {
        const gb_contact_model& m = c->laws[i];
        L[i].kn   = (St)m.kn;
        // m_muen = log(en)/sqrt(PI^2 + log(en)^2) (HookeContactForceModel.cpp:56)
        L[i].muen = (St)(std::log(m.en)
                         / std::sqrt(3.1415926535897932385 * 3.1415926535897932385
                                     + std::log(m.en) * std::log(m.en)));
        L[i].etat = (St)m.etat;
        L[i].muc  = (St)m.muc;
        L[i].kr   = (St)m.kr;
        L[i].kt   = (St)m.kt;
        c->has_kr = c->has_kr || m.kr != 0.0;
    }
    dfree(c->d_law);
    GB_TRY(dalloc((Law<St>**)&c->d_law, L.size()));
    GB_CK(cudaMemcpy(c->d_law, L.data(), L.size() * sizeof(L[0]), cudaMemcpyHostToDevice));
    return GB_OK;
}

template <typename St>
int upload_obstacles(gb_ctx* c)
{
    std::vector<RBShape<St>> sh(std::max(c->nob, 1));
    std::vector<double>      mass(std::max(c->nob, 1), 0.0);
    for(int i = 0; i < c->nob; ++i)
    {
        sh[i]   = shape_record<St>(c->obs[i], c->obs_props[i], crust_bounds(c));
        mass[i] = c->obs_props[i].mass;
    }
    dfree(c->d_obs_shape);
    dfree(c->d_obs_tr);
    dfree(c->d_obs_mass);
    GB_TRY(dalloc((RBShape<St>**)&c->d_obs_shape, sh.size()));
    GB_TRY(dalloc(&c->d_obs_tr, std::max<size_t>(c->obs_tr.size(), 12)));
    GB_TRY(dalloc(&c->d_obs_mass, mass.size()));
    GB_CK(cudaMemcpy(c->d_obs_shape, sh.data(), sh.size() * sizeof(sh[0]), cudaMemcpyHostToDevice));
    if(!c->obs_tr.empty())
        GB_CK(cudaMemcpy(c->d_obs_tr, c->obs_tr.data(), c->obs_tr.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
    GB_CK(cudaMemcpy(c->d_obs_mass, mass.data(), mass.size() * sizeof(double), cudaMemcpyHostToDevice));
    // planes of the Rectangle obstacles (normal = the frame's z axis, n . origin)
    std::vector<double4> plane(std::max(c->nob, 1), make_double4(0, 0, 0, 0));
    c->obs_rect = 0u;
    c->obs_gjk  = false;
    for(int i = 0; i < c->nob; ++i)
    {
        const double* t = c->obs_tr.data() + 12 * i;
        plane[i]        = make_double4(t[2], t[5], t[8], t[2] * t[9] + t[5] * t[10] + t[8] * t[11]);
        if(i < kMaskObstacles && c->obs[i].convex.type == GB_RECTANGLE)
            c->obs_rect |= 1u << i;
        c->obs_gjk = c->obs_gjk || (c->obs[i].convex.type != GB_RECTANGLE
                                    && c->obs[i].convex.type != GB_DRUM);
    }
    // wall velocities (zero until gb_set_obstacle_velocities)
    c->obs_vel.resize(6 * (size_t)c->nob, 0.0);
    dfree(c->d_obs_vel);
    GB_TRY(dalloc(&c->d_obs_vel, std::max<size_t>(c->obs_vel.size(), 6)));
    GB_CK(cudaMemset(c->d_obs_vel, 0, std::max<size_t>(c->obs_vel.size(), 6) * sizeof(double)));
    if(!c->obs_vel.empty())
        GB_CK(cudaMemcpy(c->d_obs_vel, c->obs_vel.data(), c->obs_vel.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
    dfree(c->d_obs_plane);
    GB_TRY(dalloc(&c->d_obs_plane, plane.size()));
    GB_CK(cudaMemcpy(c->d_obs_plane, plane.data(), plane.size() * sizeof(double4),
                     cudaMemcpyHostToDevice));
    return GB_OK;
}

int ensure_stage(gb_ctx* c)
{
    if(!c->d_stage)
        GB_TRY(dalloc(&c->d_stage, 12 * (size_t)std::max(c->n, 1)));
    return GB_OK;
}

int alloc_state(gb_ctx* c)
{
    const size_t n = c->n, ss = store_size(c->prec);
    GB_TRY(dalloc(&c->d_pos, 3 * n));
    GB_CK(cudaMalloc(&c->d_rot, std::max<size_t>(1, rot_count(c->prec) * n) * ss));
    GB_CK(cudaMalloc(&c->d_vel, std::max<size_t>(1, 3 * n) * ss));
    GB_CK(cudaMalloc(&c->d_omg, std::max<size_t>(1, 3 * n) * ss));
    GB_CK(cudaMalloc(&c->d_frc, std::max<size_t>(1, 3 * n) * ss));
    GB_CK(cudaMalloc(&c->d_trq, std::max<size_t>(1, 3 * n) * ss));
    GB_CK(cudaMemset(c->d_frc, 0, std::max<size_t>(1, 3 * n) * ss));
    GB_CK(cudaMemset(c->d_trq, 0, std::max<size_t>(1, 3 * n) * ss));
    GB_TRY(dalloc(&c->d_rb_id, n));
    GB_CK(cudaMemset(c->d_rb_id, 0, std::max<size_t>(1, n) * sizeof(uint32_t)));
    GB_TRY(dalloc(&c->d_hash, n));
    GB_TRY(dalloc(&c->d_iota, n));
    for(int b = 0; b < 2; ++b)
    {
        GB_TRY(dalloc(&c->d_k[b], n));
        GB_TRY(dalloc(&c->d_i[b], n));
        GB_TRY(dalloc(&c->d_off[b], n + 1));
    }
    GB_TRY(dalloc(&c->d_spos, n));
    GB_TRY(dalloc(&c->d_spos32, n));
    GB_TRY(dalloc(&c->d_slot, (size_t)n * kPairSlots));
    GB_TRY(dalloc(&c->d_sorted_of, n));
    GB_TRY(dalloc(&c->d_obsmask_id, n));
    GB_TRY(dalloc(&c->d_count, 2 * ((size_t)n + 1))); // count by id, then slot index by sorted position
    GB_TRY(dalloc(&c->d_contacts, n));
    GB_TRY(dalloc(&c->d_flags, 1));
    GB_TRY(dalloc(&c->d_counters, 4));
    // [0], [1]: the GJK queues' lengths; [2], [3]: the fill pass's overflow
    // counts and [4], [5] its obstacle-record counts, alternating by step
    GB_TRY(dalloc(&c->d_gjkn, 6));
    GB_CK(cudaMemset(c->d_gjkn, 0, 6 * sizeof(uint32_t)));
    GB_TRY(dalloc(&c->d_ovf, n));
    GB_TRY(dalloc(&c->d_pcount, n));
    GB_CK(cudaMemset(c->d_pcount, 0, (size_t)n * sizeof(uint32_t)));
    if(!c->d_ticket)
    {
        GB_TRY(dalloc(&c->d_ticket, 1));
        GB_CK(cudaMemset(c->d_ticket, 0, sizeof(unsigned long long)));
        c->tickets = 0;
    }
    GB_CK(cudaMemset(c->d_flags, 0, sizeof(int)));
    GB_CK(cudaMemset(c->d_counters, 0, 4 * sizeof(unsigned long long)));
    GB_CK(cudaMemset(c->d_contacts, 0, std::max<size_t>(1, n) * sizeof(int)));
    GB_CK(cudaMallocHost((void**)&c->h_pinned, 4 * sizeof(uint32_t)));
    GB_TRY(dalloc(&c->d_done, 1));
    GB_CK(cudaMemset(c->d_done, 0, sizeof(unsigned int)));
    return GB_OK;
}

int ensure_pairs(gb_ctx* c, int64_t need)
{
    if(need <= c->cap)
        return GB_OK;
    int64_t ncap = c->cap == 0 ? std::max<int64_t>(need, 1024)
                               : std::max<int64_t>(need + need / 2, 1024);
    const size_t ss = store_size(c->prec);
    const bool   hist = c->cfg.contact_law == GB_LAW_HOOKE_HISTORY;
    // the previous step's history buffers must survive the growth
    uint32_t* npb[2] = {nullptr, nullptr};
    void*     nxi[2] = {nullptr, nullptr};
    for(int b = 0; b < 2; ++b)
    {
        GB_TRY(dalloc(&npb[b], ncap));
        if(hist)
            GB_CK(cudaMalloc(&nxi[b], 3 * ncap * ss));
    }
    // (the previous step's pair count is on the device: copy the whole old
    // capacity)
    const int prev = 1 - c->cur;
    if(c->have_prev && c->cap > 0)
    {
        GB_CK(cudaMemcpy(npb[prev], c->d_pb[prev], c->cap * sizeof(uint32_t),
                         cudaMemcpyDeviceToDevice));
        if(hist)
            for(int k = 0; k < 3; ++k)
                GB_CK(cudaMemcpy((char*)nxi[prev] + k * ncap * ss,
                                 (char*)c->d_xi[prev] + k * c->cap * ss, c->cap * ss,
                                 cudaMemcpyDeviceToDevice));
    }
    for(int b = 0; b < 2; ++b)
    {
        dfree(c->d_pb[b]);
        c->d_pb[b] = npb[b];
        dfree(c->d_xi[b]);
        c->d_xi[b] = nxi[b];
    }
    dfree(c->d_pa);
    dfree(c->d_pf);
    dfree(c->d_pc);
    dfree(c->d_info);
    dfree(c->d_gjkq);
    GB_TRY(dalloc(&c->d_gjkq, (c->prec == GB_MIXED ? 2 : 1) * ncap));
    dfree(c->d_obsq);
    GB_TRY(dalloc(&c->d_obsq, ncap));
    GB_TRY(dalloc(&c->d_pa, ncap));
    GB_CK(cudaMalloc(&c->d_pf, 9 * ncap * ss));
    GB_TRY(dalloc(&c->d_pc, ncap));
    if(c->cfg.flags & GB_FLAG_RECORD_CONTACT_INFO)
        GB_TRY(dalloc(&c->d_info, 7 * ncap));
    c->cap = ncap;
    return GB_OK;
}

// exclusive scan of n uint32 (in place allowed); *d_total (device) gets the sum
// exclusive scan of n values; with abort_flags, an aborted step's scan writes
// nothing
// exclusive scan of n counts in one launch (k_scan_onepass); every block
// takes a ticket, so the host knows the counter's value before each launch
int scan_u32(gb_ctx* c, const uint32_t* in, uint32_t* out, int64_t n, uint32_t* d_total,
             const int* abort_flags = nullptr)
{
    const int nb = std::max(1, blocks(n, kTile));
    if((size_t)nb > c->tile_cap)
    {
        // growing the state mid-step: wait for the scans that may still read it
        GB_CK(cudaStreamSynchronize(c->stream));
        dfree(c->d_tile_state);
        GB_TRY(dalloc(&c->d_tile_state, nb));
        GB_CK(cudaMemset(c->d_tile_state, 0, nb * sizeof(unsigned long long)));
        c->tile_cap = nb;
    }
    c->scan_epoch = (c->scan_epoch + 1) & kScanEpochMask;
    if(c->scan_epoch == 0)
    {
        // the epoch wrapped: clear the words so that no old one can match
        GB_CK(cudaMemsetAsync(c->d_tile_state, 0, c->tile_cap * sizeof(unsigned long long),
                              c->stream));
        c->scan_epoch = 1;
    }
    GB_CK(launch(c->pdl, k_scan_onepass, nb, kBlock, c->stream, in, out, n, c->d_tile_state,
                 c->d_ticket, c->tickets, c->scan_epoch, d_total, abort_flags, c->d_flags,
                 c->scan_spin_limit));
    c->tickets += (unsigned long long)nb;
    c->launches += 1;
    GB_CK(cudaGetLastError());
    return GB_OK;
}

// hash -> stable radix sort of (cell, id) -> cell-start table -> sorted
// positions (ComponentManager::updateLinks)
// Stable LSD radix sort of (cell key, id), then the cell-start search and the
// gather of sorted positions: the fallback for cells too full for the
// counting sort's rank pass.
int broad_phase_radix(gb_ctx* c)
{
    const int n = c->n;
    const int nb = std::max(1, blocks(n, kBlock));
    cudaStream_t s = c->stream;
    mark(c, 0);
    k_hash<<<nb, kBlock, 0, s>>>(n, c->d_pos, c->d_pos + n, c->d_pos + 2 * (size_t)n,
                                 c->cfg.origin[0], c->cfg.origin[1], c->cfg.origin[2], c->cell,
                                 c->dims[0], c->dims[1], c->dims[2], c->d_hash, c->d_iota,
                                 c->d_flags);
    c->launches += 1;
    GB_CK(cudaGetLastError());
    mark(c, 1);
    const uint32_t* src_k = c->d_hash;
    const uint32_t* src_i = c->d_iota;
    const int       passes = c->key_bits == 0 ? 0 : (c->key_bits + 7) / 8;
    const int       bits_per = passes ? (c->key_bits + passes - 1) / passes : 0;
    const int       ntile = std::max(1, blocks(n, kTile));
    int             dst = 0;
    for(int p = 0; p < passes; ++p)
    {
        const int      shift = p * bits_per;
        const int      b     = std::min(bits_per, c->key_bits - shift);
        const uint32_t mask  = (1u << b) - 1u;
        const size_t   hn    = (size_t)(mask + 1) * ntile;
        if(hn > c->hist_cap)
        {
            dfree(c->d_hist);
            GB_TRY(dalloc(&c->d_hist, hn));
            c->hist_cap = hn;
        }
        k_radix_hist<<<ntile, kBlock, 0, s>>>(src_k, n, shift, mask, c->d_hist);
        GB_TRY(scan_u32(c, c->d_hist, c->d_hist, (int64_t)hn, nullptr));
        k_radix_scatter<<<ntile, kBlock, 0, s>>>(src_k, src_i, c->d_k[dst], c->d_i[dst], n, shift,
                                                 mask, c->d_hist);
        c->launches += 2;
        GB_CK(cudaGetLastError());
        src_k = c->d_k[dst];
        src_i = c->d_i[dst];
        dst ^= 1;
    }
    if(passes == 0)
    {
        GB_CK(cudaMemcpyAsync(c->d_k[0], c->d_hash, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        GB_CK(cudaMemcpyAsync(c->d_i[0], c->d_iota, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        src_k = c->d_k[0];
        src_i = c->d_i[0];
    }
    c->d_skeys = const_cast<uint32_t*>(src_k);
    c->d_sids  = const_cast<uint32_t*>(src_i);
    mark(c, 2);
    k_cell_start<<<blocks((int64_t)c->ncells + 1, kCellsPerBlock), kBlock, 0, s>>>(
        c->d_skeys, (uint32_t)n, c->ncells, c->d_cstart);
    k_gather_sorted<<<nb, kBlock, 0, s>>>(n, c->d_sids, c->d_pos, c->d_pos + n,
                                          c->d_pos + 2 * (size_t)n, c->d_rb_id, c->d_rcirc64,
                                          c->d_spos,
                                          c->prec == GB_MIXED ? c->d_spos32 : nullptr,
                                          c->d_sorted_of);
    c->launches += 2;
    GB_CK(cudaGetLastError());
    mark(c, 3);
    c->links_valid = true;
    return GB_OK;
}

// Counting sort by cell (gb_broadphase.cuh): the cell counts' scan is the
// cell-start table and the rank pass writes the sorted positions.
int broad_phase_counting(gb_ctx* c)
{
    const int    n  = c->n;
    const int    nb = std::max(1, blocks(n, kBlock));
    cudaStream_t s  = c->stream;
    mark(c, 0);
    if(!c->ccount_zero)
        GB_CK(cudaMemsetAsync(c->d_ccount, 0, ((size_t)c->ncells + 1) * sizeof(uint32_t), s));
    GB_CK(launch(c->pdl, k_hash_count, nb, kBlock, s, n, c->d_pos, c->d_pos + n,
                 c->d_pos + 2 * (size_t)n, c->cfg.origin[0], c->cfg.origin[1], c->cfg.origin[2],
                 c->cell, c->dims[0], c->dims[1], c->dims[2], c->d_hash, c->d_ccount,
                 c->d_flags));
    c->launches += 1;
    GB_CK(cudaGetLastError());
    mark(c, 1);
    GB_TRY(scan_u32(c, c->d_ccount, c->d_cstart, (int64_t)c->ncells + 1, nullptr));
    GB_CK(launch(c->pdl, k_cell_scatter, nb, kBlock, s, n, c->d_hash, c->d_cstart, c->d_ccount,
                 c->d_i[0], (const int*)c->d_flags));
    c->ccount_zero = true; // each particle took back the count it added
    c->launches += 1;
    GB_CK(cudaGetLastError());
    mark(c, 2);
    c->d_skeys = c->d_k[1];
    c->d_sids  = c->d_i[1];
    GB_CK(launch(c->pdl, k_cell_rank, nb, kBlock, s, n, c->d_i[0], c->d_hash, c->d_cstart,
                 c->d_skeys, c->d_sids, c->d_pos, c->d_pos + n, c->d_pos + 2 * (size_t)n,
                 c->d_rb_id, c->d_rcirc64, c->d_spos, c->prec == GB_MIXED ? c->d_spos32 : nullptr,
                 c->d_sorted_of, c->d_flags));
    c->launches += 1;
    GB_CK(cudaGetLastError());
    mark(c, 3);
    c->links_valid = true;
    return GB_OK;
}

int broad_phase(gb_ctx* c)
{
    return c->radix_sort ? broad_phase_radix(c) : broad_phase_counting(c);
}

// after a kFlagCellCrowded report: clear that flag and redo the broad phase
// with the radix sort (kept for the rest of the context's life)
int redo_with_radix(gb_ctx* c)
{
    const int keep = (int)c->h_pinned[1] & ~kFlagCellCrowded;
    std::memcpy(c->h_pinned + 2, &keep, sizeof(int));
    GB_CK(cudaMemcpyAsync(c->d_flags, c->h_pinned + 2, sizeof(int), cudaMemcpyHostToDevice,
                          c->stream));
    c->radix_sort = true;
    return broad_phase(c);
}

// The finer candidate grid (k_pair_count_fine): r_s is the bounding radius
// that 95% of the particles do not exceed; the grid is used where that is
// below 0.7 of the largest radius (a polydisperse packing), the rigid-body
// ids are known on the host, and its cell count stays moderate.  The split
// only decides which kernel tests a pair, never whether it is tested, so a
// stale plan costs time, not results.
// the mean reference-cell occupancy seen by a particle above which the finer
// grid pays for its extra passes (~27 x 8 = 216 candidates per particle)
constexpr double kFineCrowding = 8.0;

int fine_plan(gb_ctx* c)
{
    c->fine_planned = true;
    c->fine         = false;
    const int n     = c->n;
    if(c->fine_mode == 0 || n < 1024 || (int)c->h_rb_id.size() != n || c->props.empty())
        return GB_OK;
    std::vector<double> r(n);
    for(int i = 0; i < n; ++i)
        r[i] = bound_radius(c, c->h_rb_id[i]);
    std::vector<double> q(r);
    const size_t k = (size_t)(0.95 * (n - 1));
    std::nth_element(q.begin(), q.begin() + k, q.end());
    const double rs = q[k];
    if(!(rs > 0.0) || !(rs < 0.7 * c->rmax))
        return GB_OK;
    FineGrid g{};
    g.rs   = rs;
    g.rmax = c->rmax;
    g.h    = 2.0 * rs * (1.0 + 1e-9);
    uint64_t nf = 1;
    uint32_t dim[3];
    for(int a = 0; a < 3; ++a)
    {
        g.mn[a]      = c->cfg.origin[a];
        const double e = std::ceil((c->lc_max[a] - c->cfg.origin[a]) / g.h);
        if(!(e >= 1.0) || e > 4.0e9)
            return GB_OK;
        dim[a] = (uint32_t)e;
        nf *= dim[a];
    }
    if(2 * nf + 1 > kMaxCells || nf > 16ull * (uint64_t)n + 4096)
        return GB_OK;
    g.nx = dim[0], g.ny = dim[1], g.nz = dim[2];
    if(c->fine_mode < 0)
    {
        // worth it where the reference cells are crowded: a particle shares
        // its cell with sum(n_c^2) / n others on average (the cell starts of
        // this step's sort, read once per plan)
        std::vector<uint32_t> cs((size_t)c->ncells + 1);
        GB_CK(cudaMemcpyAsync(cs.data(), c->d_cstart, cs.size() * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, c->stream));
        GB_CK(cudaStreamSynchronize(c->stream));
        double sq = 0.0;
        for(uint32_t k = 0; k < c->ncells; ++k)
        {
            const double m = cs[k + 1] >= cs[k] ? double(cs[k + 1] - cs[k]) : 0.0;
            sq += m * m;
        }
        if(sq < kFineCrowding * (double)n)
            return GB_OK;
    }
    uint32_t nlarge = 0;
    for(int i = 0; i < n; ++i)
        nlarge += r[i] > rs;
    // keys: the small particles' fine cells, then the large particles' (+ nf)
    if(nf > c->fine_nf || !c->d_fcount)
    {
        dfree(c->d_fcount);
        dfree(c->d_fstart);
        GB_TRY(dalloc(&c->d_fcount, 2 * (size_t)nf + 1));
        GB_TRY(dalloc(&c->d_fstart, 2 * (size_t)nf + 1));
    }
    if(!c->d_fkey)
    {
        GB_TRY(dalloc(&c->d_fkey, n));
        GB_TRY(dalloc(&c->d_fskey, n));
        GB_TRY(dalloc(&c->d_fids, n));
        GB_TRY(dalloc(&c->d_fref, n));
        GB_TRY(dalloc(&c->d_fpos, n));
        GB_TRY(dalloc(&c->d_fpos32, n));
    }
    GB_CK(cudaMemsetAsync(c->d_fcount, 0, (2 * (size_t)nf + 1) * sizeof(uint32_t), c->stream));
    c->fcount_zero = true;
    c->fine_g      = g;
    c->fine_nf     = (uint32_t)nf;
    c->fine_nlarge = nlarge;
    c->fine        = true;
    return GB_OK;
}

// The obstacles that the wall mask does not decide (all but the Rectangles
// among the first kMaskObstacles), binned by linked cell: an obstacle is
// listed for every cell from which a particle's surface can reach it, so a
// particle's candidates are its cell's list (the reference tests
// every particle against every obstacle, ComponentManagerCPU.cpp:301-351;
// the contact test is unchanged).  Reach = the largest particle bounding
// radius plus crust, plus the obstacle's crust; a cell is a box (a boundary
// cell reaches past the grid, where out-of-domain centres are clamped in).
// Rectangles are met as their planes (closestPointsRectangle) and drums as
// their cylinders, both from either side: a cell is listed when its box may
// come within reach of the plane (separating-axis bound along the normal) or
// of the cylinder (the radial distance is 1-Lipschitz: its centre's, within
// the box's half-diagonal); other obstacles by their circumscribed spheres.
int obstacle_cells(gb_ctx* c)
{
    c->cobs_valid = true;
    c->cobs_used  = false;
    if(c->props.empty())
        return GB_OK;
    auto listed = [&](int o) {
        return !(o < kMaskObstacles && c->obs[o].convex.type == GB_RECTANGLE);
    };
    bool any = false;
    for(int o = 0; o < c->nob; ++o)
        any = any || listed(o);
    if(!any)
        return GB_OK;
    const uint32_t nx = c->dims[0], ny = c->dims[1], nz = c->dims[2];
    const uint32_t dn[3] = {nx, ny, nz};
    const uint64_t nc = (uint64_t)nx * ny * nz;
    if(nc > (1ull << 28))
        return GB_OK; // a grid too large to bin on the host: those obstacles stay
                      // candidates of every particle
    double         rp = 0.0, cp = 0.0;
    for(int i = 0; i < c->nrb; ++i)
    {
        rp = std::max(rp, bound_radius(c, i));
        cp = std::max(cp, c->rbs[i].crust_thickness);
    }
    const double hd = 0.5 * c->cell * std::sqrt(3.0);
    // is cell (x, y, z) within reach of obstacle o?
    auto near = [&](int o, uint32_t x, uint32_t y, uint32_t z) {
        const double* t      = c->obs_tr.data() + 12 * o;
        const double  reach  = (rp + cp + c->obs[o].crust_thickness) * (1.0 + 1e-6) + 1e-9;
        const int     type   = c->obs[o].convex.type;
        const double  n[3]   = {t[2], t[5], t[8]}; // the frame's z axis
        const double  org[3] = {t[9], t[10], t[11]};
        const uint32_t ix[3] = {x, y, z};
        double         ctr[3], hx[3];
        bool           unbounded = false;
        for(int k = 0; k < 3; ++k)
        {
            double lo = c->cfg.origin[k] + c->cell * ix[k], hi = lo + c->cell;
            if(ix[k] == 0)
                lo = -1e30;
            if(ix[k] + 1 == dn[k])
                hi = 1e30;
            unbounded = unbounded || ix[k] == 0 || ix[k] + 1 == dn[k];
            ctr[k]    = 0.5 * (lo + hi);
            hx[k]     = 0.5 * (hi - lo);
        }
        if(type == GB_RECTANGLE)
        {
            double dc = 0.0, ext = 0.0;
            for(int k = 0; k < 3; ++k)
            {
                dc += n[k] * (ctr[k] - org[k]);
                ext += std::fabs(n[k]) * hx[k];
            }
            return ext > 1e29 || std::fabs(dc) - ext <= reach;
        }
        if(unbounded)
            return true;
        double d[3], a = 0.0, r2 = 0.0;
        for(int k = 0; k < 3; ++k)
        {
            d[k] = ctr[k] - org[k];
            a += n[k] * d[k];
        }
        if(type == GB_DRUM)
        {
            for(int k = 0; k < 3; ++k)
                r2 += (d[k] - a * n[k]) * (d[k] - a * n[k]);
            return std::fabs(std::sqrt(r2) - c->obs[o].convex.p[0]) <= reach + hd;
        }
        return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
               <= c->obs_props[o].circumscribed_radius + reach + hd;
    };
    // the cells worth testing: all for planes and drums, the box of the
    // circumscribed sphere plus reach for the others
    auto range = [&](int o, uint32_t lo[3], uint32_t hi[3]) {
        const int type = c->obs[o].convex.type;
        for(int k = 0; k < 3; ++k)
        {
            lo[k] = 0;
            hi[k] = dn[k] - 1;
        }
        if(type == GB_RECTANGLE || type == GB_DRUM)
            return;
        const double* t = c->obs_tr.data() + 12 * o;
        const double  r = c->obs_props[o].circumscribed_radius
                         + (rp + cp + c->obs[o].crust_thickness) * 1.01 + c->cell;
        for(int k = 0; k < 3; ++k)
        {
            const double a = std::floor((t[9 + k] - r - c->cfg.origin[k]) / c->cell);
            const double b = std::floor((t[9 + k] + r - c->cfg.origin[k]) / c->cell);
            lo[k] = a <= 0.0 ? 0u : (a >= dn[k] - 1.0 ? dn[k] - 1 : (uint32_t)a);
            hi[k] = b <= 0.0 ? 0u : (b >= dn[k] - 1.0 ? dn[k] - 1 : (uint32_t)b);
        }
    };
    // two passes over the listed obstacles in ascending order: counts per
    // cell, then the lists at their offsets
    std::vector<uint32_t> start(nc + 1, 0u);
    for(int pass = 0; pass < 2; ++pass)
    {
        std::vector<uint32_t> fill;
        if(pass == 1)
        {
            uint64_t run = 0;
            for(uint64_t k = 0; k < nc; ++k)
            {
                const uint64_t m = start[k];
                start[k]         = (uint32_t)run;
                run += m;
            }
            if(run > 0xFFFFFFFFull)
                return GB_OK; // too many entries for 32-bit offsets: every such obstacle
                              // stays a candidate of every particle
            start[nc] = (uint32_t)run;
            fill.assign(start.begin(), start.end() - 1);
        }
        std::vector<uint32_t>& ids = c->h_cobs_ids;
        if(pass == 1)
            ids.assign(start[nc], 0u);
        for(int o = 0; o < c->nob; ++o)
        {
            if(!listed(o))
                continue;
            uint32_t lo[3], hi[3];
            range(o, lo, hi);
            for(uint32_t z = lo[2]; z <= hi[2]; ++z)
                for(uint32_t y = lo[1]; y <= hi[1]; ++y)
                    for(uint32_t x = lo[0]; x <= hi[0]; ++x)
                        if(near(o, x, y, z))
                        {
                            const uint64_t k = ((uint64_t)z * ny + y) * nx + x;
                            if(pass == 0)
                                ++start[k];
                            else
                                ids[fill[k]++] = (uint32_t)o;
                        }
        }
    }
    const std::vector<uint32_t>& ids = c->h_cobs_ids;
    dfree(c->d_cobs_start);
    dfree(c->d_cobs_ids);
    GB_TRY(dalloc(&c->d_cobs_start, start.size()));
    GB_TRY(dalloc(&c->d_cobs_ids, std::max<size_t>(ids.size(), 1)));
    GB_CK(cudaMemcpy(c->d_cobs_start, start.data(), start.size() * sizeof(uint32_t),
                     cudaMemcpyHostToDevice));
    if(!ids.empty())
        GB_CK(cudaMemcpy(c->d_cobs_ids, ids.data(), ids.size() * sizeof(uint32_t),
                         cudaMemcpyHostToDevice));
    c->cobs_entries = (int64_t)ids.size();
    c->cobs_used    = true;
    return GB_OK;
}

// candidate pairs (particles, then obstacles): count -> scan -> fill, with no
// host round trip: the total stays on the device (off[n]); a total beyond the
// capacity aborts the step (kFlagCapacity) and the host replays it larger
template <typename S>
int build_pairs(gb_ctx* c)
{
    using St = store_t<S>;
    const int    n = c->n;
    const int    nb = std::max(1, blocks(n, kBlock));
    cudaStream_t s = c->stream;
    if(c->cfg.contact_law == GB_LAW_HOOKE_HISTORY)
        c->cur ^= 1; // last step's pair list becomes the history
    GB_TRY(ensure_pairs(c, c->cap_hint));
    uint32_t*       off    = c->d_off[c->cur];
    const float4*   spos32 = c->prec == GB_MIXED ? c->d_spos32 : nullptr;
    if(c->nob && !c->mask_valid)
    {
        GB_CK(launch(c->pdl, k_obstacle_mask<S>, nb, kBlock, s, n, state_of<St>(c),
                     tables_of<S>(c), c->d_obsmask_id));
        c->launches += 1;
        GB_CK(cudaGetLastError());
        c->mask_valid = true;
    }
    if(!c->count_zero)
        GB_CK(cudaMemsetAsync(c->d_count, 0, 2 * ((size_t)n + 1) * sizeof(uint32_t), s));
    CellGeometry geo;
    for(int k = 0; k < 3; ++k)
        geo.mn[k] = c->cfg.origin[k];
    geo.cell = c->cell;
    geo.rmax = c->rmax;
    if(!c->fine_planned)
        GB_TRY(fine_plan(c));
    if(!c->cobs_valid)
        GB_TRY(obstacle_cells(c));
    ObsCand oc;
    oc.mask       = c->d_obsmask_id;
    oc.n          = c->nob;
    oc.rect       = c->obs_rect;
    oc.cell_start = c->cobs_used ? c->d_cobs_start : nullptr;
    oc.cell_ids   = c->d_cobs_ids;
    oc.skeys      = c->d_skeys;
    if(c->fine)
    {
        // the finer grid of the small particles, then the count passes
        const FineGrid& g   = c->fine_g;
        float4*         f32 = c->prec == GB_MIXED ? c->d_fpos32 : nullptr;
        if(!c->fcount_zero)
            GB_CK(cudaMemsetAsync(c->d_fcount, 0, (2 * (size_t)c->fine_nf + 1) * sizeof(uint32_t),
                                  s));
        GB_CK(launch(c->pdl, k_fine_hash, nb, kBlock, s, n, (const double*)c->d_pos,
                     (const double*)c->d_pos + n, (const double*)c->d_pos + 2 * (size_t)n,
                     (const uint32_t*)c->d_rb_id, (const double*)c->d_rcirc64, g, c->d_fkey,
                     c->d_fcount, (const int*)c->d_flags));
        GB_TRY(scan_u32(c, c->d_fcount, c->d_fstart, 2 * (int64_t)c->fine_nf + 1, nullptr,
                        c->d_flags));
        GB_CK(launch(c->pdl, k_fine_scatter, nb, kBlock, s, n, (const uint32_t*)c->d_fkey,
                     (const uint32_t*)c->d_fstart, c->d_fcount, (const double*)c->d_pos,
                     (const double*)c->d_pos + n, (const double*)c->d_pos + 2 * (size_t)n,
                     (const uint32_t*)c->d_rb_id, (const double*)c->d_rcirc64,
                     (const uint32_t*)c->d_sorted_of, c->d_fskey, c->d_fids, c->d_fref, c->d_fpos,
                     f32, (const int*)c->d_flags));
        c->fcount_zero = true; // each particle took back the count it added
        GB_CK(launch(c->pdl, k_pair_count_fine<S>, nb, kBlock, s, n,
                     (const uint32_t*)c->d_fstart, g, (const uint32_t*)c->d_fskey,
                     (const uint32_t*)c->d_fids, (const uint32_t*)c->d_fref,
                     (const double4*)c->d_fpos, (const float4*)f32, c->d_count,
                     c->d_count + n + 1, c->d_slot, oc, (const int*)c->d_flags));
        const int nbl = std::max(1, blocks((int64_t)c->fine_nlarge * 32, kBlock));
        GB_CK(launch(c->pdl, k_pair_count_large<S>, nbl, kBlock, s, n,
                     (const uint32_t*)c->d_fstart, g, (const uint32_t*)c->d_fids,
                     (const uint32_t*)c->d_fref, (const double4*)c->d_fpos, (const float4*)f32,
                     c->d_count, c->d_count + n + 1, c->d_slot, oc, (const int*)c->d_flags));
        c->launches += 4;
    }
    else
    {
        GB_CK(launch(c->pdl, k_pair_count<S>, nb, kBlock, s, n, c->d_skeys, c->d_sids,
                     c->d_spos, spos32, c->d_cstart, c->dims[0], c->dims[1], c->dims[2], geo,
                     c->d_count, c->d_count + n + 1, c->d_slot, oc, (const int*)c->d_flags));
        c->launches += 1;
    }
    GB_CK(cudaGetLastError());
    GB_TRY(scan_u32(c, c->d_count, off, n, off + n, c->d_flags));
    mark(c, 4);
    c->ovf_phase ^= 1;
    GB_CK(launch(c->pdl, k_pair_fill<S>, nb, kBlock, s, n, c->d_skeys, c->d_sids, c->d_sorted_of,
                 c->d_spos, spos32, c->d_cstart, c->dims[0], c->dims[1], c->dims[2], c->d_count,
                 c->d_slot, oc, off, c->d_pa, c->d_pb[c->cur], c->cap,
                 c->d_flags, c->d_gjkn, c->d_count + n + 1, c->d_ovf, c->ovf_phase, c->d_obsq));
    c->count_zero = true; // the fill pass zeroes each count it reads
    GB_CK(launch(c->pdl, k_pair_fill_overflow<S>, 4 * c->sms, 128, s,
                 (const uint32_t*)c->d_gjkn + 2 + c->ovf_phase, (const uint32_t*)c->d_ovf,
                 (const uint32_t*)c->d_skeys, (const uint32_t*)c->d_sids,
                 (const uint32_t*)c->d_sorted_of, (const double4*)c->d_spos, spos32,
                 (const uint32_t*)c->d_cstart, c->dims[0], c->dims[1], c->dims[2],
                 (const uint32_t*)off, c->d_pa, c->d_pb[c->cur], (const int*)c->d_flags));
    c->launches += 2;
    GB_CK(cudaGetLastError());
    mark(c, 5);
    return GB_OK;
}

template <typename S>
PairOut<store_t<S>> pair_out(gb_ctx* c)
{
    using St = store_t<S>;
    PairOut<St> po;
    const int64_t cap = c->cap;
    for(int k = 0; k < 3; ++k)
    {
        po.f[k] = (St*)c->d_pf + k * cap;
        po.t[k] = (St*)c->d_pf + (3 + k) * cap;
        po.m[k] = (St*)c->d_pf + (6 + k) * cap;
        po.xi[k] = c->d_xi[c->cur] ? (St*)c->d_xi[c->cur] + k * cap : nullptr;
    }
    po.contact  = c->d_pc;
    po.pcount   = c->d_pcount;
    po.info     = c->d_info;
    const int prev = 1 - c->cur;
    po.prev_off = c->d_off[prev];
    po.prev_b   = c->d_pb[prev];
    for(int k = 0; k < 3; ++k)
        po.prev_xi[k] = c->d_xi[prev] ? (const St*)c->d_xi[prev] + k * cap : nullptr;
    return po;
}

template <typename S>
int launch_particles(gb_ctx* c, const State<store_t<S>>& st, const Tables<S>& tb,
                      const PairOut<store_t<S>>& po, const StepParams<S>& sp, int* contacts_out)
{
    const int  nb   = std::max(1, blocks(c->n, kBlock));
    const bool move = (sp.phases & PHASE_MOVE) != 0;
    // after a detect with obstacles the stream waits on the auxiliary one:
    // a plain launch there
    const bool pdl = c->pdl && !(c->nob && (sp.phases & PHASE_DETECT));
    GB_CK(launch(pdl, k_particles<S>, nb, kBlock, c->stream, c->n, st, tb, c->d_off[c->cur], po,
                 sp, contacts_out, move && c->nob ? c->d_obsmask_id : nullptr, c->d_flags,
                 c->d_done));
    c->launches += 1;
    if(move)
        c->mask_valid = c->nob > 0;
    return GB_OK;
}

template <typename S>
int run_detect(gb_ctx* c, int phases)
{
    using St = store_t<S>;
    cudaStream_t s = c->stream;
    c->in_step     = true;
    GB_TRY(broad_phase(c));
    GB_TRY(build_pairs<S>(c));
    PairOut<St> po = pair_out<S>(c);
    const bool hist = c->cfg.contact_law == GB_LAW_HOOKE_HISTORY;
    if(hist && !c->have_prev)
    {
        // no history yet: an empty previous list for every particle
        GB_CK(cudaMemsetAsync(c->d_off[1 - c->cur], 0, (c->n + 1) * sizeof(uint32_t), s));
    }
    const State<St> st = state_of<St>(c);
    const Tables<S> tb = tables_of<S>(c);
    {
        // one wave of resident blocks walks the device-side total (off[n]):
        // a short list is spread over all of its warps (for_each_pair)
        const uint32_t* total = c->d_off[c->cur] + c->n;
        auto one_wave = [&](const void* kernel) {
            int per_sm = 0;
            if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0)
                   != cudaSuccess
               || per_sm < 1)
                per_sm = 1;
            return (int)std::max<int64_t>(
                1, std::min<int64_t>(blocks(c->cap, 128), (int64_t)per_sm * c->sms));
        };
        const int kr  = c->has_kr ? 1 : 0;
        const int law = c->cfg.contact_law;
        // the GJK variant is a template parameter: each run compiles in one.
        // The two kernels write disjoint records (particle pairs, obstacle
        // pairs); both are latency-bound on few warps, so they run side by
        // side, the obstacle one on the auxiliary stream.
        // the fill pass's count of this step's obstacle records
        const uint32_t* nobs_rec = c->d_gjkn + 4 + c->ovf_phase;
        auto with_variant = [&](auto var) -> int {
            constexpr int VAR = decltype(var)::value;
            cudaStream_t  so  = s;
            if(c->nob)
            {
                GB_CK(cudaEventRecord(c->ev_fork, s));
                GB_CK(cudaStreamWaitEvent(c->aux_stream, c->ev_fork, 0));
                so = c->aux_stream;
            }
            GB_CK(launch(c->pdl, k_narrow<S, VAR>, one_wave((const void*)k_narrow<S, VAR>), 128, s,
                         total, c->d_flags, c->d_pa, c->d_pb[c->cur], st, tb, po, law, kr,
                         S(c->cfg.dt), c->d_counters, c->d_gjkq, c->d_gjkn));
            // the FP64 GJK's queue: the cull pass's, or in the mixed mode
            // what the FP32 stage leaves of it (its certificate, a lower
            // bound on the distance, holds for every GJK variant)
            const uint32_t* q64 = c->d_gjkq;
            const uint32_t* n64 = c->d_gjkn;
            if constexpr(is_mixed<S>())
            {
                GB_CK(launch(c->pdl, k_narrow_gjk32, one_wave((const void*)k_narrow_gjk32), 128, s,
                             (const uint32_t*)c->d_gjkn, (const int*)c->d_flags,
                             (const uint32_t*)c->d_gjkq, (const uint32_t*)c->d_pa,
                             (const uint32_t*)c->d_pb[c->cur], st, tb, po, law, kr,
                             c->d_gjkq + c->cap, c->d_gjkn + 1));
                c->launches += 1;
                q64 = c->d_gjkq + c->cap;
                n64 = c->d_gjkn + 1;
            }
            auto launch_gjk = [&](auto kernel, uint32_t lo, uint32_t hi) -> int {
                GB_CK(launch(c->pdl, kernel, one_wave((const void*)kernel), 128, s, n64,
                             c->d_flags, q64, c->d_pa, c->d_pb[c->cur], st, tb, po, law, kr,
                             S(c->cfg.dt), c->d_counters, lo, hi));
                return GB_OK;
            };
            // The mixed mode's FP64 GJK at three blocks per SM where no body
            // is a polyhedron and the queue outnumbers the lane pairs of the
            // default form's wave (1M bed, ~75k pairs: 1.584 -> 1.550 ms per
            // step; 200k bed, ~15k pairs, one round either way: 0.424 ->
            // 0.441 ms; 200k polyhedra: 0.199 -> 0.206 ms).  Both forms are
            // launched; the queue length, on the device, picks the one that
            // works.
            uint32_t split = UINT32_MAX;
            if constexpr(is_mixed<S>())
                if(!c->poly_bodies)
                {
                    split = (uint32_t)(one_wave((const void*)k_narrow_gjk<S, VAR>) * 128 / 2);
                    GB_TRY(launch_gjk(k_narrow_gjk<S, VAR, 3>, split, UINT32_MAX));
                    c->launches += 1;
                }
            GB_TRY(launch_gjk(k_narrow_gjk<S, VAR>, 0u, split));
            c->launches += 2;
            if(!c->nob)
                return GB_OK;
            // Rectangles and drums are met by their own closed forms; any
            // other obstacle needs the general GJK compiled in
            if(!c->obs_gjk)
                k_narrow_obstacles<S, false, GB_GJK_JH>
                    <<<one_wave((const void*)k_narrow_obstacles<S, false, GB_GJK_JH>), 128, 0, so>>>(
                    nobs_rec, c->d_obsq, c->d_flags, c->d_pa, c->d_pb[c->cur], st, tb, po, law,
                    kr, S(c->cfg.dt), c->d_counters);
            else
                k_narrow_obstacles<S, true, VAR>
                    <<<one_wave((const void*)k_narrow_obstacles<S, true, VAR>), 128, 0, so>>>(
                    nobs_rec, c->d_obsq, c->d_flags, c->d_pa, c->d_pb[c->cur], st, tb, po, law,
                    kr, S(c->cfg.dt), c->d_counters);
            c->launches += 1;
            GB_CK(cudaEventRecord(c->ev_join, so));
            GB_CK(cudaStreamWaitEvent(s, c->ev_join, 0));
            return GB_OK;
        };
        if(c->cfg.gjk_variant == GB_GJK_SV)
            GB_TRY(with_variant(std::integral_constant<int, GB_GJK_SV>{}));
        else if(c->cfg.gjk_variant == GB_GJK_NESTEROV)
            GB_TRY(with_variant(std::integral_constant<int, GB_GJK_NESTEROV>{}));
        else
            GB_TRY(with_variant(std::integral_constant<int, GB_GJK_JH>{}));
        GB_CK(cudaGetLastError());
    }
    mark(c, 6);
    StepParams<S> sp;
    sp.dt         = S(c->cfg.dt);
    sp.h          = S(c->cfg.integrator == GB_VELOCITY_VERLET && !c->verlet_started
                          ? 0.5 * c->cfg.dt
                          : c->cfg.dt);
    sp.g          = mk<S>(S(c->cfg.gravity[0]), S(c->cfg.gravity[1]), S(c->cfg.gravity[2]));
    sp.integrator = c->cfg.integrator;
    sp.law_kind   = c->cfg.contact_law;
    sp.has_kr     = c->has_kr ? 1 : 0;
    sp.phases     = phases;
    sp.accumulate = (phases & PHASE_DETECT) && c->torce_dirty ? 1 : 0;
    sp.rb_identity = c->rb_identity ? 1 : 0;
    // the per-particle contact counts are read only by the detect call
    GB_TRY(launch_particles<S>(c, st, tb, po, sp, phases == PHASE_STEP ? nullptr : c->d_contacts));
    GB_CK(cudaGetLastError());
    mark(c, 7);
    close_event_set(c);
    c->in_step = false;
    if(phases & PHASE_MOVE)
    {
        c->verlet_started = true;
        c->steps_done++;
    }
    c->detect_valid = true;
    c->have_prev    = hist;
    return GB_OK;
}

template <typename S>
int run_particles(gb_ctx* c, int phases)
{
    using St = store_t<S>;
    StepParams<S> sp;
    sp.dt         = S(c->cfg.dt);
    sp.h          = S(c->cfg.integrator == GB_VELOCITY_VERLET && !c->verlet_started
                          ? 0.5 * c->cfg.dt
                          : c->cfg.dt);
    sp.g          = mk<S>(S(c->cfg.gravity[0]), S(c->cfg.gravity[1]), S(c->cfg.gravity[2]));
    sp.integrator = c->cfg.integrator;
    sp.law_kind   = c->cfg.contact_law;
    sp.has_kr     = c->has_kr ? 1 : 0;
    sp.phases     = phases;
    sp.accumulate = (phases & PHASE_DETECT) && c->torce_dirty ? 1 : 0;
    sp.rb_identity = c->rb_identity ? 1 : 0;
    PairOut<St> po = pair_out<S>(c);
    GB_TRY(launch_particles<S>(c, state_of<St>(c), tables_of<S>(c), po, sp, nullptr));
    GB_CK(cudaGetLastError());
    if(phases & PHASE_MOVE)
    {
        c->verlet_started = true;
        c->steps_done++;
    }
    return GB_OK;
}

template <typename F>
int dispatch(gb_ctx* c, F&& f)
{
    switch(c->prec)
    {
        case GB_FP64:
            return f((double)0);
        case GB_MIXED:
            return f((float)0);
        case GB_FP64_STRICT:
            return f(dstrict(0.0));
        default:
            return GB_E_INVALID_ARG;
    }
}

int ready(gb_ctx* c)
{
    if(!c)
        return GB_E_INVALID_ARG;
    if(!(c->rb_set && c->law_set && c->tr_set && (c->nob == 0 || c->obs_set)))
        return GB_E_NOT_READY;
    return GB_OK;
}

int finish(gb_ctx* c)
{
    // read and clear the device status flags; out-of-domain and non-finite
    // states are reported, capacity overflow is an error
    int flags = 0;
    GB_CK(cudaMemcpyAsync(&flags, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    GB_CK(cudaMemsetAsync(c->d_flags, 0, sizeof(int), c->stream));
    GB_CK(cudaStreamSynchronize(c->stream));
    accumulate_pending(c);
    c->last.status_flags |= flags;
    if(flags & kFlagCapacity)
        return GB_E_CAPACITY;
    if(flags & kFlagScanStall)
        return GB_E_CUDA;
    if(flags & kFlagNonFinite)
        return GB_E_NONFINITE;
    if(flags & kFlagOutOfDomain)
        return GB_E_OUT_OF_DOMAIN;
    return GB_OK;
}

// the host-side bookkeeping of one step, kept to replay aborted steps
struct StepSnap
{
    int     cur;
    bool    have_prev, verlet_started, torce_dirty, mask_valid, detect_valid, links_valid;
    int64_t steps_done;
};

StepSnap snap(const gb_ctx* c)
{
    return {c->cur,         c->have_prev,    c->verlet_started, c->torce_dirty,
            c->mask_valid,  c->detect_valid, c->links_valid,    c->steps_done};
}

void restore(gb_ctx* c, const StepSnap& s)
{
    c->cur            = s.cur;
    c->have_prev      = s.have_prev;
    c->verlet_started = s.verlet_started;
    c->torce_dirty    = s.torce_dirty;
    c->mask_valid     = s.mask_valid;
    c->detect_valid   = s.detect_valid;
    c->links_valid    = s.links_valid;
    c->steps_done     = s.steps_done;
    c->count_zero     = false; // an aborted fill pass may have left counts behind
    c->ccount_zero    = false; // ... and an aborted scatter pass cell counts
    c->fcount_zero    = false; // ... or fine-cell counts
    // ... and an aborted step its contact counts per particle
    if(c->d_pcount)
        cudaMemsetAsync(c->d_pcount, 0, (size_t)c->n * sizeof(uint32_t), c->stream);
}

// Launches n_steps detects (PHASE_DETECT) or fused steps (PHASE_STEP) with no
// host synchronisation between them, then reads the device status once.  A
// step that aborted -- more candidate pairs than the capacity, or a cell too
// full for the counting sort -- left the state untouched, and so did every
// step launched after it (they return at entry): the host grows the capacity
// or switches to the radix sort, restores its bookkeeping to the aborted step
// and launches the remaining steps again.
int run_steps(gb_ctx* c, int32_t n_steps, int phases, int32_t* result)
{
    c->contacts_loaded = false; // a detect replaces a loaded contact set
    cudaStream_t s    = c->stream;
    const bool   hist = c->cfg.contact_law == GB_LAW_HOOKE_HISTORY;
    int32_t      done = 0;
    for(int attempt = 0; done < n_steps; ++attempt)
    {
        if(attempt > 16)
            return GB_E_CAPACITY;
        std::vector<StepSnap> snaps;
        GB_CK(cudaMemsetAsync(c->d_done, 0, sizeof(unsigned int), s));
        for(int32_t k = done; k < n_steps; ++k)
        {
            snaps.push_back(snap(c));
            GB_TRY(dispatch(c, [&](auto z) { return run_detect<decltype(z)>(c, phases); }));
            if(phases & PHASE_MOVE)
            {
                // the first step adds to a torce left by separate calls, then resets it
                c->links_valid = false;
                c->torce_dirty = false;
            }
            else
                c->torce_dirty = true;
        }
        // one synchronisation: status flags, completed launches and the last
        // step's pair count together
        GB_CK(cudaMemcpyAsync(c->h_pinned + 1, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost, s));
        GB_CK(cudaMemcpyAsync(c->h_pinned + 2, c->d_done, sizeof(unsigned int),
                              cudaMemcpyDeviceToHost, s));
        GB_CK(cudaMemcpyAsync(c->h_pinned + 3, c->d_off[c->cur] + c->n, sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
        GB_CK(cudaStreamSynchronize(s));
        const int      flags = (int)c->h_pinned[1];
        const uint32_t ok    = c->h_pinned[2];
        if(!(flags & kFlagAbort))
        {
            accumulate_pending(c);
            c->npairs = c->h_pinned[3];
            done      = n_steps;
            break;
        }
        if(ok >= snaps.size())
            return GB_E_CUDA; // an abort flag with every launch completed: inconsistent
        c->ev_npending = 0;   // the aborted launches' phase times mean nothing
        restore(c, snaps[ok]);
        if(flags & kFlagScanStall)
        {
            // a scan gave up waiting: the step is not replayed; the state is
            // that before the aborted step, the flags are cleared
            c->last.status_flags |= flags;
            GB_CK(cudaMemset(c->d_flags, 0, sizeof(int)));
            return GB_E_CUDA;
        }
        if(flags & kFlagCellCrowded)
            c->radix_sort = true;
        if(flags & kFlagCapacity)
        {
            // the aborted step's own pair total is in its offsets buffer (the
            // steps after it skipped their scans)
            const int cur_k = hist ? (c->cur ^ 1) : c->cur;
            GB_CK(cudaMemcpy(c->h_pinned + 3, c->d_off[cur_k] + c->n, sizeof(uint32_t),
                             cudaMemcpyDeviceToHost));
            const int64_t need = c->h_pinned[3];
            c->cap_hint        = std::max<int64_t>(2 * c->cap, need + need / 4);
        }
        const int keep = flags & ~kFlagAbort;
        std::memcpy(c->h_pinned + 1, &keep, sizeof(int));
        GB_CK(cudaMemcpy(c->d_flags, c->h_pinned + 1, sizeof(int), cudaMemcpyHostToDevice));
        done += (int32_t)ok;
    }
    if(result)
    {
        std::vector<int> cnt(c->n);
        GB_CK(cudaMemcpy(cnt.data(), c->d_contacts, c->n * sizeof(int), cudaMemcpyDeviceToHost));
        for(int i = 0; i < c->n; ++i)
            result[i] += cnt[i];
    }
    // the status (finish() without another synchronisation)
    const int flags = n_steps > 0 ? (int)c->h_pinned[1] : 0;
    GB_CK(cudaMemsetAsync(c->d_flags, 0, sizeof(int), s));
    c->last.status_flags |= flags;
    if(flags & kFlagScanStall)
        return GB_E_CUDA;
    if(flags & kFlagNonFinite)
        return GB_E_NONFINITE;
    if(flags & kFlagOutOfDomain)
        return GB_E_OUT_OF_DOMAIN;
    return GB_OK;
}

} // namespace

// ============================================================================
extern "C" {

int gb_abi_version(void)
{
    return GB_ABI_VERSION;
}

const char* gb_status_string(int status)
{
    switch(status)
    {
        case GB_OK:
            return "ok";
        case GB_E_INVALID_ARG:
            return "invalid argument";
        case GB_E_CUDA:
            return g_last_cuda != cudaSuccess ? cudaGetErrorString(g_last_cuda) : "CUDA error";
        case GB_E_OUT_OF_MEMORY:
            return "device out of memory";
        case GB_E_NOT_READY:
            return "context not fully set up";
        case GB_E_OUT_OF_DOMAIN:
            return "a particle centre left the linked-cell grid";
        case GB_E_NONFINITE:
            return "non-finite particle state";
        case GB_E_NO_DEVICE:
            return "no usable CUDA device";
        case GB_E_CAPACITY:
            return "buffer capacity exceeded";
        case GB_E_UNSUPPORTED:
            return "unsupported feature";
        default:
            return "unknown status";
    }
}

gb_ctx* gb_create(const gb_config* cfg, int* status)
{
    auto fail = [&](int st) -> gb_ctx* {
        if(status)
            *status = st;
        return nullptr;
    };
    if(!cfg || cfg->n_particles < 0 || cfg->n_rigid_bodies < 1 || cfg->n_obstacles < 0
       || cfg->n_materials < 1 || !(cfg->dt > 0.0)
       || (cfg->precision != GB_FP64 && cfg->precision != GB_MIXED
           && cfg->precision != GB_FP64_STRICT)
       || (cfg->contact_law != GB_LAW_HOOKE && cfg->contact_law != GB_LAW_HOOKE_HISTORY)
       || (cfg->integrator != GB_FIRST_ORDER_EXPLICIT && cfg->integrator != GB_VELOCITY_VERLET))
        return fail(GB_E_INVALID_ARG);
    if(cfg->gjk_variant != GB_GJK_JH && cfg->gjk_variant != GB_GJK_SV
       && cfg->gjk_variant != GB_GJK_NESTEROV)
        return fail(GB_E_INVALID_ARG);
    int ndev = 0;
    if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0)
        return fail(GB_E_NO_DEVICE);
    if(cudaSetDevice(cfg->device) != cudaSuccess)
        return fail(GB_E_NO_DEVICE);
    gb_ctx* c = new gb_ctx;
    c->cfg    = *cfg;
    // test knob: a lower bound on the one-pass scans' look-back wait makes it
    // run out, which a step reports as GB_E_CUDA with the state untouched
    if(const char* lim = std::getenv("GB_DEBUG_SCAN_SPIN_LIMIT"))
        c->scan_spin_limit = (uint32_t)std::strtoul(lim, nullptr, 10);
    // test knob: the finer candidate grid off (0) or on wherever it applies
    // (1) instead of where the reference cells are crowded
    if(const char* fg = std::getenv("GB_DEBUG_FINE_GRID"))
        c->fine_mode = std::atoi(fg) ? 1 : 0;
    c->prec   = cfg->precision;
    c->n      = cfg->n_particles;
    c->nrb    = cfg->n_rigid_bodies;
    c->nob    = cfg->n_obstacles;
    c->nmat   = cfg->n_materials;
    int st    = GB_OK;
    int sms   = 0;
    if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device) == cudaSuccess
       && sms > 0)
        c->sms = sms;
    if(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess
       || cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking) != cudaSuccess
       || cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess
       || cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)
        st = GB_E_CUDA;
    c->stream = c->own_stream;
    c->timing = (cfg->flags & GB_FLAG_PHASE_TIMING) != 0;
    if(st == GB_OK && c->timing)
        for(int b = 0; b < gb_ctx::kEvRing && st == GB_OK; ++b)
            for(int k = 0; k <= GB_N_PHASES; ++k)
                if(cudaEventCreate(&c->ev[b][k]) != cudaSuccess)
                {
                    st        = GB_E_CUDA;
                    c->timing = false;
                    break;
                }
    if(st == GB_OK)
        st = alloc_state(c);
    if(st == GB_OK)
        st = ensure_pairs(c, cfg->pair_capacity > 0 ? cfg->pair_capacity
                                                    : std::max<int64_t>(1 << 16, 8 * (int64_t)c->n));
    c->cap_hint = c->cap;
    if(st != GB_OK)
    {
        gb_destroy(c);
        return fail(st);
    }
    if(status)
        *status = GB_OK;
    return c;
}

int gb_destroy(gb_ctx* c)
{
    if(!c)
        return GB_E_INVALID_ARG;
    if(c->stream)
        cudaStreamSynchronize(c->stream);
    void* ptrs[] = {c->d_shape, c->d_inertia, c->d_verts, c->d_law, c->d_obs_shape, c->d_obs_tr,
                    c->d_obs_mass, c->d_obs_plane, c->d_obs_vel, c->d_rcirc64, c->d_pos, c->d_rot, c->d_vel, c->d_omg, c->d_frc,
                    c->d_trq, c->d_rb_id, c->d_hash, c->d_iota, c->d_k[0], c->d_k[1], c->d_i[0],
                    c->d_i[1], c->d_hist, c->d_part, c->d_cstart, c->d_ccount, c->d_spos, c->d_spos32, c->d_slot, c->d_sorted_of, c->d_obsmask_id, c->d_count,
                    c->d_off[0], c->d_off[1], c->d_pb[0], c->d_pb[1], c->d_pa, c->d_pf, c->d_pc,
                    c->d_info, c->d_xi[0], c->d_xi[1], c->d_flags, c->d_counters, c->d_done,
                    c->d_contacts,
                    c->d_stage,     c->d_adj, c->d_tile_state, c->d_ticket, c->d_gjkq, c->d_gjkn,
                    c->d_fkey, c->d_fcount, c->d_fstart, c->d_fskey, c->d_fids, c->d_fref,
                    c->d_fpos, c->d_fpos32, c->d_ovf, c->d_pcount, c->d_cobs_start,
                    c->d_cobs_ids, c->d_obsq};
    for(void* p : ptrs)
        if(p)
            cudaFree(p);
    if(c->d_shape64 && c->d_shape64 != c->d_shape)
        cudaFree(c->d_shape64);
    if(c->d_verts64 && c->d_verts64 != c->d_verts)
        cudaFree(c->d_verts64);
    if(c->d_obs_shape64 && c->d_obs_shape64 != c->d_obs_shape)
        cudaFree(c->d_obs_shape64);
    if(c->h_pinned)
        cudaFreeHost(c->h_pinned);
    if(c->timing)
        for(int b = 0; b < gb_ctx::kEvRing; ++b)
            for(int k = 0; k <= GB_N_PHASES; ++k)
                cudaEventDestroy(c->ev[b][k]);
    if(c->ev_fork)
        cudaEventDestroy(c->ev_fork);
    if(c->ev_join)
        cudaEventDestroy(c->ev_join);
    if(c->aux_stream)
        cudaStreamDestroy(c->aux_stream);
    if(c->own_stream)
        cudaStreamDestroy(c->own_stream);
    delete c;
    return GB_OK;
}

int gb_set_stream(gb_ctx* c, void* cuda_stream)
{
    if(!c)
        return GB_E_INVALID_ARG;
    GB_CK(cudaStreamSynchronize(c->stream));
    c->stream = cuda_stream ? (cudaStream_t)cuda_stream : c->own_stream;
    return GB_OK;
}

int gb_get_phase_times(gb_ctx* c, double* ms, int64_t* steps, int32_t reset)
{
    if(!c || !ms)
        return GB_E_INVALID_ARG;
    if(!c->timing)
        return GB_E_NOT_READY;
    GB_CK(cudaStreamSynchronize(c->stream));
    accumulate_pending(c);
    for(int k = 0; k < GB_N_PHASES; ++k)
        ms[k] = c->phase_ms[k];
    if(steps)
        *steps = c->phase_steps;
    if(reset)
    {
        for(int k = 0; k < GB_N_PHASES; ++k)
            c->phase_ms[k] = 0;
        c->phase_steps = 0;
    }
    return GB_OK;
}

int gb_set_rigid_bodies(gb_ctx* c, const gb_rigid_body_desc* rbs, const double* vertices,
                        int64_t n_vertices)
{
    if(!c || !rbs || n_vertices < 0 || (n_vertices && !vertices))
        return GB_E_INVALID_ARG;
    c->rbs.assign(rbs, rbs + c->nrb);
    c->fine_planned = false;
    c->cobs_valid   = false; // the cell size may change
    c->verts.assign(vertices, vertices + 3 * n_vertices);
    c->props.resize(c->nrb);
    double rmax = 0.0;
    c->poly_bodies = false;
    for(int i = 0; i < c->nrb; ++i)
    {
        const gb_convex& cv = rbs[i].convex;
        c->poly_bodies = c->poly_bodies || cv.type == GB_POLYHEDRON;
        if(cv.type == GB_POLYHEDRON
           && (cv.first_vertex < 0 || cv.first_vertex + cv.n_vertices > n_vertices))
            return GB_E_INVALID_ARG;
        if(cv.type == GB_CYLINDER || cv.type == GB_CONE)
            return GB_E_UNSUPPORTED;
        if(rbs[i].material < 0 || rbs[i].material >= c->nmat)
            return GB_E_INVALID_ARG;
        GB_TRY(gb_rigid_body_properties(&rbs[i], vertices, &c->props[i]));
        rmax = std::max(rmax, bound_radius(c, i)); // Grains.cpp:226-231
    }
    // linked cell: cell = factor * 2 * max circumscribed radius (Grains.cpp:233-246)
    double coeff = c->cfg.cell_size_factor;
    if(coeff < 1.0)
        coeff = 1.0;
    c->cell = coeff * 2.0 * rmax;
    c->rmax = rmax;
    for(int k = 0; k < 3; ++k)
    {
        c->lc_max[k] = c->cfg.max_coordinate[k] + (c->cfg.pad_grid ? c->cell : 0.0);
        double t     = 1.e-10; // LinkedCell.cpp:23-28
        t += c->lc_max[k] - c->cfg.origin[k];
        t /= c->cell;
        if(!(t >= 1.0) || t > 4.0e9)
            return GB_E_INVALID_ARG;
        c->dims[k] = (uint32_t)t;
    }
    const uint64_t nc = (uint64_t)c->dims[0] * c->dims[1] * c->dims[2];
    if(nc == 0 || nc > kMaxCells)
        return GB_E_INVALID_ARG;
    c->ncells   = (uint32_t)nc;
    c->key_bits = 0;
    while(c->key_bits < 32 && (1ull << c->key_bits) < nc)
        ++c->key_bits;
    dfree(c->d_cstart);
    GB_TRY(dalloc(&c->d_cstart, (size_t)nc + 1));
    dfree(c->d_ccount);
    c->ccount_zero = false;
    GB_TRY(dalloc(&c->d_ccount, (size_t)nc + 1));
    if(c->d_shape64 && c->d_shape64 != c->d_shape)
    {
        cudaFree(c->d_shape64);
        cudaFree(c->d_verts64);
    }
    c->d_shape64 = c->d_verts64 = nullptr;
    int st       = upload_tables<double>(c);
    c->d_shape64 = c->d_shape;
    c->d_verts64 = c->d_verts;
    if(st == GB_OK && c->prec == GB_MIXED)
    {
        c->d_shape = c->d_verts = nullptr; // keep the FP64 copies, add FP32 ones
        st                      = upload_tables<float>(c);
    }
    if(st)
        return st;
    c->rb_set     = true;
    c->mask_valid = false;
    return GB_OK;
}

int gb_get_rigid_body_props(gb_ctx* c, int32_t rb, gb_rigid_body_props* out)
{
    if(!c || !out || rb < 0 || rb >= c->nrb || !c->rb_set)
        return GB_E_INVALID_ARG;
    *out = c->props[rb];
    return GB_OK;
}

int gb_set_contact_models(gb_ctx* c, const gb_contact_model* table)
{
    if(!c || !table)
        return GB_E_INVALID_ARG;
    c->laws.assign(table, table + c->nmat * (c->nmat + 1) / 2);
    for(auto& m : c->laws)
        if(!(m.kn >= 0.0) || !(m.en > 0.0 && m.en <= 1.0))
            return GB_E_INVALID_ARG;
    int st = c->prec == GB_MIXED ? upload_laws<float>(c) : upload_laws<double>(c);
    if(st)
        return st;
    c->law_set = true;
    return GB_OK;
}

int gb_set_obstacles(gb_ctx* c, const gb_rigid_body_desc* obst, const double* transforms)
{
    if(!c || (c->nob && (!obst || !transforms)))
        return GB_E_INVALID_ARG;
    c->obs.assign(obst, obst + c->nob);
    c->obs_tr.assign(transforms, transforms + 12 * (size_t)c->nob);
    c->obs_props.resize(c->nob);
    for(int i = 0; i < c->nob; ++i)
    {
        if(obst[i].convex.type == GB_POLYHEDRON || obst[i].convex.type == GB_CYLINDER
           || obst[i].convex.type == GB_CONE)
            return GB_E_UNSUPPORTED;
        if(obst[i].convex.type == GB_DRUM && !(obst[i].convex.p[0] > 0.0))
            return GB_E_INVALID_ARG;
        if(obst[i].material < 0 || obst[i].material >= c->nmat)
            return GB_E_INVALID_ARG;
        GB_TRY(gb_rigid_body_properties(&obst[i], nullptr, &c->obs_props[i]));
    }
    if(c->d_obs_shape64 && c->d_obs_shape64 != c->d_obs_shape)
        cudaFree(c->d_obs_shape64);
    c->d_obs_shape64 = nullptr;
    int st           = upload_obstacles<double>(c);
    c->d_obs_shape64 = c->d_obs_shape;
    if(st == GB_OK && c->prec == GB_MIXED)
    {
        c->d_obs_shape = nullptr;
        st             = upload_obstacles<float>(c);
    }
    if(st)
        return st;
    c->obs_set    = true;
    c->mask_valid = false;
    c->cobs_valid = false;
    return GB_OK;
}

int gb_set_obstacle_velocities(gb_ctx* c, const double* kin)
{
    if(!c || (c->nob && !kin))
        return GB_E_INVALID_ARG;
    if(!c->obs_set)
        return GB_E_NOT_READY;
    for(size_t k = 0; k < 6 * (size_t)c->nob; ++k)
        if(!std::isfinite(kin[k]))
            return GB_E_INVALID_ARG;
    c->obs_vel.assign(kin, kin + 6 * (size_t)c->nob);
    if(c->nob)
    {
        // ordered after the steps already launched, as every state update
        GB_CK(cudaStreamSynchronize(c->stream));
        GB_CK(cudaMemcpy(c->d_obs_vel, c->obs_vel.data(), c->obs_vel.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
    }
    return GB_OK;
}

int gb_set_rigid_body_ids(gb_ctx* c, const uint32_t* ids)
{
    if(!c || !ids)
        return GB_E_INVALID_ARG;
    for(int i = 0; i < c->n; ++i)
        if(ids[i] >= (uint32_t)c->nrb)
            return GB_E_INVALID_ARG;
    GB_CK(cudaMemcpy(c->d_rb_id, ids, c->n * sizeof(uint32_t), cudaMemcpyHostToDevice));
    c->h_rb_id.assign(ids, ids + c->n);
    c->fine_planned = false;
    c->ids_set     = true;
    c->mask_valid  = false;
    c->rb_identity = c->nrb == c->n;
    for(int i = 0; i < c->n && c->rb_identity; ++i)
        c->rb_identity = ids[i] == (uint32_t)i;
    return GB_OK;
}

int gb_set_transforms(gb_ctx* c, const double* t)
{
    if(!c || !t)
        return GB_E_INVALID_ARG;
    const int n = c->n;
    if(n == 0)
        return c->tr_set = true, GB_OK;
    GB_TRY(ensure_stage(c));
    GB_CK(cudaMemcpyAsync(c->d_stage, t, 12 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice,
                          c->stream));
    if(c->prec == GB_MIXED)
        k_set_transforms<float><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
            n, c->d_stage, c->d_pos, (float*)c->d_rot, 1);
    else
        k_set_transforms<double><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
            n, c->d_stage, c->d_pos, (double*)c->d_rot, 0);
    c->launches += 1;
    GB_CK(cudaGetLastError());
    GB_CK(cudaStreamSynchronize(c->stream));
    c->tr_set      = true;
    c->links_valid = c->detect_valid = c->mask_valid = false;
    return GB_OK;
}

static int set_soa6(gb_ctx* c, const double* kin, void* a, void* b)
{
    const int n = c->n;
    if(n == 0)
        return GB_OK;
    GB_TRY(ensure_stage(c));
    GB_CK(cudaMemcpyAsync(c->d_stage, kin, 6 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice,
                          c->stream));
    if(c->prec == GB_MIXED)
        k_set_pairs3<float><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(n, c->d_stage, (float*)a,
                                                                         (float*)b);
    else
        k_set_pairs3<double><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(n, c->d_stage,
                                                                          (double*)a, (double*)b);
    c->launches += 1;
    GB_CK(cudaGetLastError());
    GB_CK(cudaStreamSynchronize(c->stream));
    return GB_OK;
}

static int get_soa6(gb_ctx* c, double* kin, const void* a, const void* b)
{
    const int n = c->n;
    if(n == 0)
        return GB_OK;
    GB_TRY(ensure_stage(c));
    if(c->prec == GB_MIXED)
        k_get_pairs3<float><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
            n, c->d_stage, (const float*)a, (const float*)b);
    else
        k_get_pairs3<double><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
            n, c->d_stage, (const double*)a, (const double*)b);
    c->launches += 1;
    GB_CK(cudaGetLastError());
    GB_CK(cudaMemcpyAsync(kin, c->d_stage, 6 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
    GB_CK(cudaStreamSynchronize(c->stream));
    return GB_OK;
}

int gb_set_velocities(gb_ctx* c, const double* kin)
{
    if(!c || !kin)
        return GB_E_INVALID_ARG;
    GB_TRY(set_soa6(c, kin, c->d_vel, c->d_omg));
    c->vel_set = true;
    return GB_OK;
}

int gb_get_velocities(gb_ctx* c, double* kin)
{
    if(!c || !kin)
        return GB_E_INVALID_ARG;
    return get_soa6(c, kin, c->d_vel, c->d_omg);
}

int gb_get_torces(gb_ctx* c, double* torce)
{
    if(!c || !torce)
        return GB_E_INVALID_ARG;
    return get_soa6(c, torce, c->d_frc, c->d_trq);
}

int gb_set_torces(gb_ctx* c, const double* torce)
{
    if(!c || !torce)
        return GB_E_INVALID_ARG;
    GB_TRY(set_soa6(c, torce, c->d_frc, c->d_trq));
    c->torce_dirty = true;
    return GB_OK;
}

int gb_get_transforms(gb_ctx* c, double* t)
{
    if(!c || !t)
        return GB_E_INVALID_ARG;
    const int n = c->n;
    if(n == 0)
        return GB_OK;
    GB_TRY(ensure_stage(c));
    if(c->prec == GB_MIXED)
        k_get_transforms<float><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
            n, c->d_stage, c->d_pos, (const float*)c->d_rot, 1);
    else
        k_get_transforms<double><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
            n, c->d_stage, c->d_pos, (const double*)c->d_rot, 0);
    c->launches += 1;
    GB_CK(cudaGetLastError());
    GB_CK(cudaMemcpyAsync(t, c->d_stage, 12 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                          c->stream));
    GB_CK(cudaStreamSynchronize(c->stream));
    return GB_OK;
}

int gb_update_links(gb_ctx* c)
{
    GB_TRY(ready(c));
    GB_TRY(broad_phase(c));
    if(!c->radix_sort)
    {
        GB_CK(cudaMemcpyAsync(c->h_pinned + 1, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost,
                              c->stream));
        GB_CK(cudaStreamSynchronize(c->stream));
        if(c->h_pinned[1] & kFlagCellCrowded)
            GB_TRY(redo_with_radix(c));
    }
    return finish(c);
}

int gb_detect_collision_and_compute_contact_forces(gb_ctx* c, int32_t* result)
{
    GB_TRY(ready(c));
    GB_CK(cudaMemsetAsync(c->d_counters, 0, 4 * sizeof(unsigned long long), c->stream));
    return run_steps(c, 1, PHASE_DETECT, result);
}

int gb_add_external_forces(gb_ctx* c)
{
    GB_TRY(ready(c));
    GB_TRY(dispatch(c, [&](auto z) { return run_particles<decltype(z)>(c, PHASE_GRAVITY); }));
    c->torce_dirty = true;
    return finish(c);
}

int gb_move_particles(gb_ctx* c)
{
    GB_TRY(ready(c));
    GB_TRY(dispatch(c, [&](auto z) { return run_particles<decltype(z)>(c, PHASE_MOVE); }));
    c->torce_dirty      = false;
    c->links_valid      = false;
    return finish(c);
}

int gb_step(gb_ctx* c, int32_t n_steps)
{
    GB_TRY(ready(c));
    if(n_steps < 0)
        return GB_E_INVALID_ARG;
    GB_CK(cudaMemsetAsync(c->d_counters, 0, 4 * sizeof(unsigned long long), c->stream));
    return run_steps(c, n_steps, PHASE_STEP, nullptr);
}

// ---- differentiable stepping (no counterpart in the reference) ----------------
int gb_save_state(gb_ctx* c, double* dst)
{
    if(!c || !dst)
        return GB_E_INVALID_ARG;
    if(c->prec == GB_MIXED)
        return GB_E_UNSUPPORTED;
    const size_t n = c->n;
    cudaStream_t s = c->stream;
    GB_CK(cudaMemcpyAsync(dst, c->d_pos, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(dst + 3 * n, c->d_rot, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(dst + 12 * n, c->d_vel, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(dst + 15 * n, c->d_omg, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaStreamSynchronize(s));
    return GB_OK;
}

int gb_load_state(gb_ctx* c, const double* src)
{
    if(!c || !src)
        return GB_E_INVALID_ARG;
    if(c->prec == GB_MIXED)
        return GB_E_UNSUPPORTED;
    const size_t n = c->n;
    cudaStream_t s = c->stream;
    GB_CK(cudaMemcpyAsync(c->d_pos, src, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_rot, src + 3 * n, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_vel, src + 12 * n, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_omg, src + 15 * n, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaStreamSynchronize(s));
    c->tr_set = c->vel_set = true;
    c->links_valid = c->detect_valid = c->mask_valid = false;
    c->contacts_loaded = false;
    return GB_OK;
}

int gb_set_integrator_phase(gb_ctx* c, int32_t started)
{
    if(!c || (started != 0 && started != 1))
        return GB_E_INVALID_ARG;
    c->verlet_started = started != 0;
    return GB_OK;
}

// A saved contact set: a 16-byte header (n, pair count as int64), the pair
// offsets (n + 1 uint32), the partners (uint32 per pair), the contact flags
// (one byte per pair).
int gb_save_contacts(gb_ctx* c, void* buf, int64_t capacity, int64_t* size)
{
    if(!c || !size || capacity < 0)
        return GB_E_INVALID_ARG;
    if(!c->detect_valid)
        return GB_E_NOT_READY;
    const int64_t n = c->n, np = c->npairs;
    const int64_t need = 16 + 4 * (n + 1) + 5 * np;
    *size = need;
    if(!buf)
        return GB_OK;
    if(capacity < need)
        return GB_E_CAPACITY;
    char*         b      = static_cast<char*>(buf);
    const int64_t hdr[2] = {n, np};
    cudaStream_t  s      = c->stream;
    GB_CK(cudaMemcpyAsync(b, hdr, sizeof(hdr), cudaMemcpyHostToDevice, s));
    GB_CK(cudaMemcpyAsync(b + 16, c->d_off[c->cur], 4 * (size_t)(n + 1),
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(b + 16 + 4 * (n + 1), c->d_pb[c->cur], 4 * (size_t)np,
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(b + 16 + 4 * (n + 1) + 4 * np, c->d_pc, (size_t)np,
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaStreamSynchronize(s));
    return GB_OK;
}

int gb_load_contacts(gb_ctx* c, const void* buf)
{
    if(!c || !buf)
        return GB_E_INVALID_ARG;
    int64_t hdr[2];
    GB_CK(cudaMemcpy(hdr, buf, sizeof(hdr), cudaMemcpyDeviceToHost));
    if(hdr[0] != c->n || hdr[1] < 0 || hdr[1] > UINT32_MAX)
        return GB_E_INVALID_ARG;
    const int64_t n = c->n, np = hdr[1];
    GB_TRY(ensure_pairs(c, np));
    const char*  b = static_cast<const char*>(buf);
    cudaStream_t s = c->stream;
    GB_CK(cudaMemcpyAsync(c->d_off[c->cur], b + 16, 4 * (size_t)(n + 1),
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_pb[c->cur], b + 16 + 4 * (n + 1), 4 * (size_t)np,
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_pc, b + 16 + 4 * (n + 1) + 4 * np, (size_t)np,
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaStreamSynchronize(s));
    c->npairs          = np;
    c->contacts_loaded = true;
    return GB_OK;
}

int gb_adjoint_step(gb_ctx* c, const double* adj_next, double* adj_prev, double* grad_laws)
{
    GB_TRY(ready(c));
    if(!adj_next || !adj_prev || !grad_laws)
        return GB_E_INVALID_ARG;
    const int nl = c->nmat * (c->nmat + 1) / 2;
    if(c->prec == GB_MIXED || c->cfg.contact_law != GB_LAW_HOOKE || nl > kAdjMaxLaws)
        return GB_E_UNSUPPORTED;
    for(const auto& rb : c->rbs)
        if(rb.convex.type != GB_SPHERE)
            return GB_E_UNSUPPORTED;
    for(const auto& ob : c->obs)
        if(ob.convex.type != GB_RECTANGLE)
            return GB_E_UNSUPPORTED;
    for(double v : c->obs_vel) // walls at rest only
        if(v != 0.0)
            return GB_E_UNSUPPORTED;
    AdjLaws laws{};
    laws.n = nl;
    for(int l = 0; l < nl; ++l)
    {
        const gb_contact_model& m = c->laws[l];
        if(m.kr != 0.0)
            return GB_E_UNSUPPORTED;
        const double pi = 3.14159265358979323846, L = std::log(m.en), q = pi * pi + L * L;
        laws.l[l] = {m.kn, m.en, m.etat, m.muc, L / std::sqrt(q), pi * pi / (q * std::sqrt(q)) / m.en};
    }
    const int    n  = c->n;
    const int    nb = std::max(1, blocks(n, kBlock));
    cudaStream_t s  = c->stream;
    if(!c->d_adj || c->adj_cap < (size_t)(6 * n + nb * 4 * kAdjMaxLaws))
    {
        dfree(c->d_adj);
        c->adj_cap = (size_t)6 * n + (size_t)nb * 4 * kAdjMaxLaws;
        GB_TRY(dalloc(&c->d_adj, c->adj_cap));
    }
    // the contacts of the current state; the accumulated torces are kept aside
    GB_TRY(ensure_stage(c));
    GB_CK(cudaMemcpyAsync(c->d_stage, c->d_frc, 3 * (size_t)n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_stage + 3 * (size_t)n, c->d_trq, 3 * (size_t)n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
    const bool dirty = c->torce_dirty;
    c->torce_dirty   = false;
    int        st    = GB_OK;
    if(c->contacts_loaded)
        c->contacts_loaded = false; // the contacts of this state, saved when it was stepped
    else
    {
        GB_CK(cudaMemsetAsync(c->d_counters, 0, 4 * sizeof(unsigned long long), s));
        st = run_steps(c, 1, PHASE_DETECT, nullptr);
        if(st != GB_OK && st != GB_E_OUT_OF_DOMAIN)
            return st;
    }
    const State<double> state = state_of<double>(c);
    const auto*         in    = (const RBInertia<double>*)c->d_inertia;
    double*             lft   = c->d_adj;
    double*             part  = c->d_adj + 6 * (size_t)n;
    const bool   verlet = c->cfg.integrator == GB_VELOCITY_VERLET;
    const double h      = verlet && !c->verlet_started ? 0.5 * c->cfg.dt : c->cfg.dt;
    k_adj_integrate<<<nb, kBlock, 0, s>>>(n, c->cfg.dt, h, verlet ? 1 : 0, state, in, adj_next,
                                          adj_prev, lft);
    k_adj_contacts<<<nb, kBlock, 0, s>>>(n, state, (const RBShape<double>*)c->d_shape, in,
                                         c->d_off[c->cur], c->d_pb[c->cur], c->d_pc, lft,
                                         c->d_obs_tr, (const RBShape<double>*)c->d_obs_shape,
                                         laws, adj_prev, part);
    k_adj_reduce<<<1, 4 * kAdjMaxLaws, 0, s>>>(nb, 4 * nl, part, grad_laws);
    c->launches += 3;
    GB_CK(cudaGetLastError());
    GB_CK(cudaMemcpyAsync(c->d_frc, c->d_stage, 3 * (size_t)n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
    GB_CK(cudaMemcpyAsync(c->d_trq, c->d_stage + 3 * (size_t)n, 3 * (size_t)n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
    c->torce_dirty = dirty;
    GB_CK(cudaStreamSynchronize(s));
    return st;
}

int gb_synchronize(gb_ctx* c)
{
    if(!c)
        return GB_E_INVALID_ARG;
    return finish(c);
}

int gb_get_stats(gb_ctx* c, gb_stats* o)
{
    if(!c || !o)
        return GB_E_INVALID_ARG;
    GB_CK(cudaStreamSynchronize(c->stream));
    unsigned long long cnt[4];
    GB_CK(cudaMemcpy(cnt, c->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost));
    std::memset(o, 0, sizeof(*o));
    o->steps_done        = c->steps_done;
    o->candidate_pairs   = c->npairs;
    o->obstacle_contacts = (int64_t)cnt[0];
    o->gjk_iterations    = (int64_t)cnt[1];
    if(c->d_gjkn)
    {
        // particle pairs queued for GJK by the last detect (past the bounding
        // tests and GJK's first iteration), and those solved by the FP64 GJK
        uint32_t q[2] = {0, 0};
        GB_CK(cudaMemcpy(q, c->d_gjkn, sizeof(q), cudaMemcpyDeviceToHost));
        const bool stage32 = c->prec == GB_MIXED;
        o->gjk_calls       = c->detect_valid ? (int64_t)q[0] : 0;
        o->gjk_fp64_calls  = c->detect_valid ? (int64_t)q[stage32 ? 1 : 0] : 0;
        o->fine_grid_cells = c->fine ? (int64_t)c->fine_nf : 0;
    }
    if(c->detect_valid && c->npairs > 0)
    {
        // particle pairs only: obstacle candidates share the list
        std::vector<uint8_t>  pc(c->npairs);
        std::vector<uint32_t> pb(c->npairs);
        GB_CK(cudaMemcpy(pc.data(), c->d_pc, c->npairs, cudaMemcpyDeviceToHost));
        GB_CK(cudaMemcpy(pb.data(), c->d_pb[c->cur], c->npairs * sizeof(uint32_t),
                         cudaMemcpyDeviceToHost));
        int64_t k = 0, obs = 0, ko = 0;
        for(int64_t p = 0; p < c->npairs; ++p)
        {
            k += pc[p] == kContactParticle;
            ko += pc[p] == kContactObstacle;
            obs += (pb[p] & kObstacleBit) != 0;
        }
        o->contacts            = k;
        o->obstacle_contacts   = ko; // of the last step, as the particle contacts
        o->candidate_pairs     = c->npairs - obs;
        o->obstacle_candidates = obs;
    }
    o->status_flags = c->last.status_flags;
    o->n_cells      = (int32_t)c->ncells;
    for(int k = 0; k < 3; ++k)
    {
        o->cells_per_dir[k] = (int32_t)c->dims[k];
        o->grid_max[k]      = c->lc_max[k];
    }
    o->key_bits        = c->key_bits;
    o->cell_size       = c->cell;
    o->kernel_launches = c->launches;
    return GB_OK;
}

int gb_debug_dump(gb_ctx* c, int32_t kind, void* out, int64_t capacity, int64_t* count)
{
    if(!c || !count)
        return GB_E_INVALID_ARG;
    GB_CK(cudaStreamSynchronize(c->stream));
    const int64_t n = c->n;
    auto copy_u32 = [&](const uint32_t* d, int64_t m) -> int {
        *count = m;
        if(out && capacity > 0)
            GB_CK(cudaMemcpy(out, d, std::min(m, capacity) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        return GB_OK;
    };
    switch(kind)
    {
        case GB_DUMP_NEIGHBORS:
        {
            // the reference's 27-entry neighbour table (LinkedCell.cpp:35-72)
            if(!c->rb_set)
                return GB_E_NOT_READY;
            const int64_t m = (int64_t)c->ncells * 27;
            *count          = m;
            if(!out)
                return GB_OK;
            uint32_t*      o  = (uint32_t*)out;
            const uint32_t nx = c->dims[0], ny = c->dims[1], nz = c->dims[2];
            int64_t        w  = 0;
            for(uint32_t h = 0; h < c->ncells && w < capacity; ++h)
            {
                const int cx = h % nx, cy = (h / nx) % ny, cz = h / (nx * ny);
                for(int k = -1; k < 2; ++k)
                    for(int j = -1; j < 2; ++j)
                        for(int i = -1; i < 2; ++i)
                        {
                            const int x = cx + i, y = cy + j, z = cz + k;
                            const bool in = x >= 0 && x < (int)nx && y >= 0 && y < (int)ny && z >= 0
                                            && z < (int)nz;
                            if(w < capacity)
                                o[w] = in ? (uint32_t)x + (uint32_t)y * nx + (uint32_t)z * nx * ny
                                          : UINT32_MAX;
                            ++w;
                        }
            }
            return GB_OK;
        }
        case GB_DUMP_CELL_HASH:
            if(!c->links_valid && !c->detect_valid)
                return GB_E_NOT_READY;
            return copy_u32(c->d_hash, n);
        case GB_DUMP_SORTED_IDS:
            if(!c->links_valid && !c->detect_valid)
                return GB_E_NOT_READY;
            return copy_u32(c->d_sids, n);
        case GB_DUMP_CELL_START:
            if(!c->links_valid && !c->detect_valid)
                return GB_E_NOT_READY;
            return copy_u32(c->d_cstart, (int64_t)c->ncells + 1);
        case GB_DUMP_CANDIDATE_PAIRS:
        case GB_DUMP_CONTACT_PAIRS:
        case GB_DUMP_CONTACT_INFO:
        case GB_DUMP_CONTACT_FORCES:
        {
            if(!c->detect_valid)
                return GB_E_NOT_READY;
            if(kind == GB_DUMP_CONTACT_INFO && !c->d_info)
                return GB_E_UNSUPPORTED;
            const int64_t         P = c->npairs;
            std::vector<uint32_t> a(P), b(P);
            std::vector<uint8_t>  pc(P);
            if(P)
            {
                GB_CK(cudaMemcpy(a.data(), c->d_pa, P * 4, cudaMemcpyDeviceToHost));
                GB_CK(cudaMemcpy(b.data(), c->d_pb[c->cur], P * 4, cudaMemcpyDeviceToHost));
                GB_CK(cudaMemcpy(pc.data(), c->d_pc, P, cudaMemcpyDeviceToHost));
            }
            std::vector<double> info;
            if(kind == GB_DUMP_CONTACT_INFO && P)
            {
                info.resize(7 * P);
                GB_CK(cudaMemcpy(info.data(), c->d_info, 7 * P * sizeof(double), cudaMemcpyDeviceToHost));
            }
            // force and torque of each pair (the storage type of the mode)
            std::vector<double> ft;
            if(kind == GB_DUMP_CONTACT_FORCES && P)
            {
                const size_t        ss = store_size(c->prec);
                std::vector<char> raw(6 * P * ss);
                for(int k = 0; k < 6; ++k)
                    GB_CK(cudaMemcpy(raw.data() + k * P * ss, (const char*)c->d_pf + k * c->cap * ss,
                                     P * ss, cudaMemcpyDeviceToHost));
                ft.resize(6 * P);
                for(int k = 0; k < 6; ++k)
                    for(int64_t p = 0; p < P; ++p)
                        ft[6 * p + k] = ss == 4 ? (double)((const float*)raw.data())[k * P + p]
                                                : ((const double*)raw.data())[k * P + p];
            }
            int64_t w = 0;
            for(int64_t p = 0; p < P; ++p)
            {
                if(b[p] & kObstacleBit) // particle-obstacle records share the list
                    continue;
                if(kind != GB_DUMP_CANDIDATE_PAIRS && !pc[p])
                    continue;
                if(kind == GB_DUMP_CONTACT_INFO)
                {
                    if(out && 7 * w + 7 <= capacity)
                        std::memcpy((double*)out + 7 * w, &info[7 * p], 7 * sizeof(double));
                }
                else if(kind == GB_DUMP_CONTACT_FORCES)
                {
                    if(out && 6 * w + 6 <= capacity)
                        std::memcpy((double*)out + 6 * w, &ft[6 * p], 6 * sizeof(double));
                }
                else if(out && 2 * w + 2 <= capacity)
                {
                    ((uint32_t*)out)[2 * w]     = a[p];
                    ((uint32_t*)out)[2 * w + 1] = b[p];
                }
                ++w;
            }
            *count = kind == GB_DUMP_CONTACT_INFO ? 7 * w : kind == GB_DUMP_CONTACT_FORCES ? 6 * w : 2 * w;
            return GB_OK;
        }
        default:
            return GB_E_INVALID_ARG;
    }
}

int gb_device_pointer(gb_ctx* c, const char* name, void** ptr)
{
    if(!c || !name || !ptr)
        return GB_E_INVALID_ARG;
    const std::string s(name);
    const size_t      n  = c->n;
    const size_t      ss = store_size(c->prec);
    const char*       axes = "xyz";
    for(int k = 0; k < 3; ++k)
    {
        const std::string ax(1, axes[k]);
        if(s == "pos_" + ax)
            return *ptr = c->d_pos + k * n, GB_OK;
        if(s == "vel_" + ax)
            return *ptr = (char*)c->d_vel + k * n * ss, GB_OK;
        if(s == "omega_" + ax)
            return *ptr = (char*)c->d_omg + k * n * ss, GB_OK;
        if(s == "force_" + ax)
            return *ptr = (char*)c->d_frc + k * n * ss, GB_OK;
        if(s == "torque_" + ax)
            return *ptr = (char*)c->d_trq + k * n * ss, GB_OK;
    }
    if(s == "rb_id")
    {
        // written by the caller from now on: the host copy no longer holds
        c->h_rb_id.clear();
        c->fine_planned = false;
        return c->rb_identity = false, *ptr = c->d_rb_id, GB_OK;
    }
    if(s == "rotation")
        return *ptr = c->d_rot, GB_OK;
    return GB_E_INVALID_ARG;
}

} // extern "C"

// ---- RawData writer (gb_rawdata.cuh) ----------------------------------------------
struct gb_rawdata_writer
{
    gb_ctx*      c = nullptr;
    std::string  base;   // directory/root_name
    int          flags = 0;
    FILE*        f[10]  = {}; // position x,y,z; translational x,y,z; angular x,y,z; coordination
    double*      d_snap = nullptr;
    uint32_t*    d_cn   = nullptr;
    double*      h_snap = nullptr; // pinned
    uint32_t*    h_cn   = nullptr; // pinned
    cudaStream_t copy   = nullptr;
    cudaEvent_t  ev_snap = nullptr, ev_copied = nullptr;
    std::thread  worker;
    int          status = GB_OK; // the last save's write status
};

namespace
{
const char* const kRawFiles[10] = {"_position_x",
                                   "_position_y",
                                   "_position_z",
                                   "_translational_velocity_x",
                                   "_translational_velocity_y",
                                   "_translational_velocity_z",
                                   "_angular_velocity_x",
                                   "_angular_velocity_y",
                                   "_angular_velocity_z",
                                   "_coordinationNumber"};

// one save's lines, formatted from the pinned snapshot: component files in
// parallel threads, then the coordination number and particleType files
int raw_write_lines(gb_rawdata_writer* w, int n, double time)
{
    cudaSetDevice(w->c->cfg.device);
    if(cudaEventSynchronize(w->ev_copied) != cudaSuccess)
        return GB_E_CUDA;
    const int    nob = w->c->nob;
    const double* otr = w->c->obs_tr.data();
    char         tbuf[64];
    raw_real(tbuf, sizeof tbuf, time);
    int  bad[9] = {0};
    auto line   = [&](int k) {
        std::string out(tbuf);
        out.reserve((size_t)(n + nob) * 14 + 64);
        char         b[64];
        const double* v = w->h_snap + (size_t)k * n;
        for(int i = 0; i < n; ++i)
        {
            out.push_back(' ');
            out.append(b, (size_t)raw_real(b, sizeof b, v[i]));
        }
        for(int o = 0; o < nob; ++o)
        {
            // obstacles: the origin of their transform, zero velocities
            out.push_back(' ');
            out.append(b, (size_t)raw_real(b, sizeof b, k < 3 ? otr[12 * o + 9 + k] : 0.0));
        }
        out.push_back('\n');
        bad[k] = std::fwrite(out.data(), 1, out.size(), w->f[k]) != out.size()
                 || std::fflush(w->f[k]) != 0;
    };
    std::vector<std::thread> th;
    for(int k = 1; k < 9; ++k)
        th.emplace_back(line, k);
    line(0);
    for(auto& t : th)
        t.join();
    std::string cn;
    if(w->flags & GB_RAW_COORDINATION_NUMBER)
    {
        cn = tbuf;
        for(int i = 0; i < n; ++i)
            cn += " " + std::to_string(w->h_cn[i]);
    }
    cn.push_back('\n');
    int err = std::fwrite(cn.data(), 1, cn.size(), w->f[9]) != cn.size() || std::fflush(w->f[9]);
    // particleType.dat: rewritten at each save with one empty line
    FILE* pt = std::fopen((w->base + "_particleType.dat").c_str(), "w");
    err |= !pt || std::fputc('\n', pt) == EOF;
    if(pt)
        err |= std::fclose(pt) != 0;
    for(int k = 0; k < 9; ++k)
        err |= bad[k];
    return err ? GB_E_INVALID_ARG : GB_OK;
}

int raw_join(gb_rawdata_writer* w)
{
    if(w->worker.joinable())
        w->worker.join();
    return w->status;
}
} // namespace

extern "C" {

int gb_rawdata_open(gb_ctx* c, const char* directory, const char* root_name, int32_t flags,
                    gb_rawdata_writer** out)
{
    if(!c || !directory || !root_name || !out || (flags & ~GB_RAW_COORDINATION_NUMBER))
        return GB_E_INVALID_ARG;
    *out                 = nullptr;
    gb_rawdata_writer* w = new gb_rawdata_writer;
    w->c                 = c;
    w->flags             = flags;
    w->base              = std::string(directory) + "/" + root_name;
    auto fail            = [&](int st) {
        gb_rawdata_close(w);
        return st;
    };
    // PostProcessing_start: the files are created empty (ios::out)
    for(int k = 0; k < 10; ++k)
        if(!(w->f[k] = std::fopen((w->base + kRawFiles[k] + ".dat").c_str(), "w")))
            return fail(GB_E_INVALID_ARG);
    const size_t n = (size_t)std::max(c->n, 1);
    if(dalloc(&w->d_snap, 9 * n) || dalloc(&w->d_cn, n))
        return fail(GB_E_OUT_OF_MEMORY);
    if(cudaMallocHost(&w->h_snap, 9 * n * sizeof(double)) != cudaSuccess
       || cudaMallocHost(&w->h_cn, n * sizeof(uint32_t)) != cudaSuccess)
        return fail(GB_E_OUT_OF_MEMORY);
    if(cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking) != cudaSuccess
       || cudaEventCreateWithFlags(&w->ev_snap, cudaEventDisableTiming) != cudaSuccess
       || cudaEventCreateWithFlags(&w->ev_copied, cudaEventDisableTiming) != cudaSuccess)
        return fail(GB_E_CUDA);
    *out = w;
    return GB_OK;
}

int gb_rawdata_write(gb_rawdata_writer* w, double time)
{
    if(!w)
        return GB_E_INVALID_ARG;
    gb_ctx* c = w->c;
    GB_TRY(ready(c));
    GB_TRY(raw_join(w)); // the previous save has left the pinned buffers
    const int n = c->n;
    if(n > 0)
    {
        const uint32_t* off = c->detect_valid ? c->d_off[c->cur] : nullptr;
        uint32_t*       cn  = (w->flags & GB_RAW_COORDINATION_NUMBER) ? w->d_cn : nullptr;
        if(c->prec == GB_MIXED)
            k_raw_snapshot<float><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
                n, c->d_pos, (const float*)c->d_vel, (const float*)c->d_omg, off, c->d_pc,
                w->d_snap, cn);
        else
            k_raw_snapshot<double><<<blocks(n, kBlock), kBlock, 0, c->stream>>>(
                n, c->d_pos, (const double*)c->d_vel, (const double*)c->d_omg, off, c->d_pc,
                w->d_snap, cn);
        c->launches += 1;
        GB_CK(cudaGetLastError());
    }
    GB_CK(cudaEventRecord(w->ev_snap, c->stream));
    GB_CK(cudaStreamWaitEvent(w->copy, w->ev_snap, 0));
    if(n > 0)
    {
        GB_CK(cudaMemcpyAsync(w->h_snap, w->d_snap, 9 * (size_t)n * sizeof(double),
                              cudaMemcpyDeviceToHost, w->copy));
        if(w->flags & GB_RAW_COORDINATION_NUMBER)
            GB_CK(cudaMemcpyAsync(w->h_cn, w->d_cn, (size_t)n * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, w->copy));
    }
    GB_CK(cudaEventRecord(w->ev_copied, w->copy));
    w->worker = std::thread([w, n, time] { w->status = raw_write_lines(w, n, time); });
    return GB_OK;
}

int gb_rawdata_close(gb_rawdata_writer* w)
{
    if(!w)
        return GB_E_INVALID_ARG;
    int st = raw_join(w);
    for(FILE*& f : w->f)
        if(f)
        {
            if(std::fclose(f) != 0 && st == GB_OK)
                st = GB_E_INVALID_ARG;
            f = nullptr;
        }
    if(w->copy)
        cudaStreamSynchronize(w->copy);
    dfree(w->d_snap);
    dfree(w->d_cn);
    if(w->h_snap)
        cudaFreeHost(w->h_snap);
    if(w->h_cn)
        cudaFreeHost(w->h_cn);
    if(w->ev_snap)
        cudaEventDestroy(w->ev_snap);
    if(w->ev_copied)
        cudaEventDestroy(w->ev_copied);
    if(w->copy)
        cudaStreamDestroy(w->copy);
    delete w;
    return st;
}

} // extern "C"
