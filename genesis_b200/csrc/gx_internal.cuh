// gx_internal.cuh -- shared definitions of the sm_100a hot-path library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "genesis_gpu.h"

namespace gx {

constexpr int kNElem = GX_NELEM;
constexpr int kMaxKinds = 16;          // distinct (element, charge) kinds in the mixed path
constexpr double kFixScale = 4294967296.0;  // 2^32 fixed-point units per force/energy unit
constexpr double kFixInv = 1.0 / 4294967296.0;
constexpr float kFixScaleF = 4294967296.0f;
constexpr double kEpsF64 = 2.220446049250313e-16;  // f64::EPSILON (grid.rs:217)

// Device error word bits (read back by the host after a call).
enum : uint32_t {
    kErrSaturation = 1u,
    kErrNonFinite = 2u,
    kErrCapacity = 4u,
    kErrBinRange = 8u,
    kErrTimeout = 16u,
};

// ---------------------------------------------------------------------------
// Exact FP64: the intrinsics below are never contracted into FMAs, so a chain
// of them rounds exactly like the reference's Rust arithmetic.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }

// f64::rem_euclid: r = a % b (fmod, exact); r < 0 ? r + |b| : r.  When
// |a| < |b|, fmod(a, b) is a itself (the quotient truncates to 0), so the
// division is skipped: every coordinate that is already inside the box takes
// that path, with the same bits.
__device__ __forceinline__ double rem_euclid(double a, double b) {
    double r = fabs(a) < fabs(b) ? a : fmod(a, b);
    return r < 0.0 ? xadd(r, fabs(b)) : r;
}
// min_image, src/physics/grid.rs:300-306 (round = half away from zero).
__device__ __forceinline__ double min_image1(double d, double L) {
    return xsub(d, xmul(L, round(xdiv(d, L))));
}
// min_image1 without the division, for the separation d of two wrapped
// positions (|d| < L): round(d / L) is then 0 or +-1, and the sign test
// below gives the same value except for |d| within rounding of L/2; the
// subtraction is min_image1's, so elsewhere the bits are the same.  Near
// |d| = L/2 both images lie about L/2 from the atom, beyond the cutoff of
// any grid with >= 3 cells per axis (cutoff <= cell <= L/3).
__device__ __forceinline__ double min_image_near(double d, double L, double half_L) {
    const double k = d > half_L ? 1.0 : (d < -half_L ? -1.0 : 0.0);
    return xsub(d, xmul(L, k));
}

// Geometry of one SpatialGrid (src/physics/grid.rs:67-86).
struct GridGeom {
    uint32_t n[3];      // cells per axis
    double cell[3];     // cell edge per axis = L / n
    double L[3];        // world size
    float cellf[3];
    float Lf[3];
    float invLf[3];
    uint32_t ncell;
    int minimg_mask;    // bit k set when axis k has < 3 cells (FP32 min-image needed)
    // Canonical half-shell offsets (grid.rs:275-296): first nonzero +1,
    // zero on degenerate axes.  Up to 13.
    int nhalf;
    int8_t half[13][3];
    // All distinct offsets on non-degenerate axes, excluding 0 (for gather passes).
    int nfull;
    int8_t full[26][3];
};

GridGeom make_grid(const double box[3], double min_cell, int* ok);

__device__ __forceinline__ uint32_t axis_cell(double v, double L, double c, uint32_t n) {
    double u = rem_euclid(xadd(v, xmul(0.5, L)), L);  // grid.rs:230
    double f = floor(xdiv(u, c));                     // grid.rs:231
    uint32_t i = f <= 0.0 ? 0u : (f >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)f);
    return i < n - 1 ? i : n - 1;
}
__device__ __forceinline__ uint32_t encode(const GridGeom& g, uint32_t ix, uint32_t iy, uint32_t iz) {
    return ix + g.n[0] * (iy + g.n[1] * iz);
}
__device__ __forceinline__ void decode(const GridGeom& g, uint32_t idx, uint32_t& ix, uint32_t& iy,
                                       uint32_t& iz) {
    uint32_t nxny = g.n[0] * g.n[1];
    iz = idx / nxny;
    uint32_t rem = idx - iz * nxny;
    iy = rem / g.n[0];
    ix = rem - iy * g.n[0];
}
__device__ __forceinline__ uint32_t wrap_add(uint32_t c, int d, uint32_t n) {
    int v = (int)c + d;
    if (v < 0) v += (int)n;
    if (v >= (int)n) v -= (int)n;
    return (uint32_t)v;
}
__device__ __forceinline__ uint32_t cell_of(const GridGeom& g, double x, double y, double z) {
    return encode(g, axis_cell(x, g.L[0], g.cell[0], g.n[0]), axis_cell(y, g.L[1], g.cell[1], g.n[1]),
                  axis_cell(z, g.L[2], g.cell[2], g.n[2]));
}
// Offset of a coordinate from the origin of its cell (u - i*cell, u as in
// cell_of), exact FP64 so every kernel that stages FP32 positions agrees.
__device__ __forceinline__ double cell_local(double v, double L, double c, uint32_t i) {
    return xsub(rem_euclid(xadd(v, xmul(0.5, L)), L), xmul((double)i, c));
}

// Number of times the reference's neighbors() reports a pair whose members
// sit in cells A != B: the count of offsets o (zero on degenerate axes, o != 0)
// with A + o == B (mod n).  It is > 1 only on axes with exactly two cells.
__device__ __forceinline__ int pair_multiplicity(const GridGeom& g, uint32_t A, uint32_t B) {
    if (A == B) return 1;
    uint32_t a[3], b[3];
    decode(g, A, a[0], a[1], a[2]);
    decode(g, B, b[0], b[1], b[2]);
    int cnt = 0;
    for (int k = 0; k < g.nfull; ++k) {
        bool hit = true;
        for (int ax = 0; ax < 3; ++ax)
            if (wrap_add(a[ax], g.full[k][ax], g.n[ax]) != b[ax]) hit = false;
        cnt += hit;
    }
    return cnt;
}

// Force-law setup (ForceSystem::new, src/systems/forces.rs:100-142).
struct ForceSetup {
    double pair_sigma[kNElem * kNElem];
    double pair_eps[kNElem * kNElem];
    double lj_rc, lj_ron;
    double rc;  // largest enabled cutoff = grid cell
    double coul_rc, coul_ron, grav_rc, grav_ron;
    double bond_k_bind;
    double max_sigma;
    double r_eq_factor;   // 2^(1/6)   (equilibrium_distance, forces.rs:281-283)
    double curv_factor;   // 72 * 2^(-1/3) (well_curvature, forces.rs:194-196)
};

// Mixed-path pair table entry, one per (kind_i, kind_j).
struct PairF {
    float sigma, half_sigma, inv_half_sigma, eps4;
    float eps24, qq, gm, pad1;  // qq = k_e q_i q_j, gm = G m_i m_j
};

// Device buffers of one atom set in cell-sorted order.
struct StateBuf {
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;
    double *charge, *mass, *inv_mass;
    uint8_t* elem;
    uint8_t* kind;
    uint32_t* slot;  // ECS slot of the atom stored at this position
};

// Scratch of one counting sort (cell list).
struct CellList {
    uint32_t* count = nullptr;   // ncell
    uint32_t* start = nullptr;   // ncell + 1
    uint32_t* fill = nullptr;    // ncell
    size_t cap_cells = 0;
    std::vector<uint32_t*> scan_levels;  // block sums per scan level
    std::vector<size_t> scan_sizes;
    uint32_t* tmp = nullptr;     // n: the scatter's order before the per-cell ranking
    size_t cap_tmp = 0;
};
void cells_free(CellList& cl);

struct ProfSlot {
    const char* name;
    uint64_t launches;
    double ms;
    std::vector<cudaEvent_t> ev;  // pairs (start, stop) not yet read
};

}  // namespace gx

struct gx_handle {
    gx_params p;
    gx::ForceSetup fs;
    gx::GridGeom fgrid;  // force grid (cell >= rc)
    cudaStream_t stream = nullptr;
    std::string err;
    int precision = GX_FP64;

    size_t n = 0, cap = 0;
    gx::StateBuf buf[2];
    int cur = 0;
    bool sorted = false;  // buf[cur] is sorted by the force grid and keys are valid

    // per-atom scratch
    uint32_t* key = nullptr;       // cell key per atom (current order)
    uint32_t* key_sorted = nullptr;
    uint32_t* perm = nullptr;      // sorted position -> previous position
    uint32_t* pos_of_slot = nullptr;  // ECS slot -> sorted position
    uint32_t* entity = nullptr;    // EntityId::index per ECS slot
    bool has_entity = false;
    float4* pos4 = nullptr;        // mixed staging: cell-local xyz + kind
    long long* F = nullptr;        // mixed fixed-point forces, 3 * cap (SoA)
    double* host_stage = nullptr;  // device AoS staging for host transfers (3 * cap)
    uint8_t* u8_stage = nullptr;
    gx::CellList cl;

    // reductions and scalars on device
    double* red = nullptr;         // block partials (several rows of kRedCap)
    double* dscal = nullptr;       // [0]=lambda pending, [1]=K, [2]=V, [3]=Vb, [4]=speed, [5]=one
    unsigned long long* dcount = nullptr;  // [0]=pairs, [1..3]=fixed V, Vb, ..., [8]=bond count
    uint32_t* derr = nullptr;      // device error word
    // gx_set_step_async: gx_step returns without waiting; its error word is
    // copied to pinned host memory and reported by the next call that waits
    bool step_async = false;
    bool step_errs_pending = false;
    uint32_t* herr = nullptr;      // pinned copy of derr
    bool lambda_pending = false;

    // mixed kinds
    int nkinds = 0;
    double kind_charge[gx::kMaxKinds];
    double kind_mass[gx::kMaxKinds];  // part of the kind only with gravity
    uint8_t kind_elem[gx::kMaxKinds];
    gx::PairF* d_pairf = nullptr;  // kMaxKinds^2

    // bonds (slot pairs).  The spring kernel reads the count from dcount[8],
    // so a captured tick stays valid while the list changes length in place;
    // only a new buffer (bonds_cap) changes the launch.
    uint32_t* bonds = nullptr;
    size_t nbonds = 0, bonds_cap = 0;

    // gx_tick_host: the column copies run on their own stream beside the tick.
    // io_ev[0..2] order each staged column against its use; io_ev[3] is
    // recorded by every list tick (captured ones too) once the positions are
    // final, so that they can be copied out while the pair pass runs.
    cudaStream_t io_stream = nullptr;
    cudaEvent_t io_ev[4] = {};
    bool io_events = false;
    double* io_stage = nullptr;  // three AoS columns of 3 * io_cap doubles
    size_t io_cap = 0;
    bool last_tick_nl = false;   // the last gx_step tick ran on the neighbour-list path

    // profiling
    bool pass_timing = false;      // events around the pair pass, in captured ticks too
    cudaEvent_t pass_ev[2] = {};
    bool prof_on = false;
    std::vector<gx::ProfSlot> prof;
    std::vector<cudaEvent_t> ev_pool;

    // CUDA graphs of one tick, per buffer parity and with/without records
    cudaGraphExec_t graph_exec[2][2] = {};
    uint64_t graph_key[2][2] = {};
    uint64_t graph_kernels[2][2] = {};
    // list path: kTicksPerGraph ticks captured in one graph, without / with records
    cudaGraphExec_t graph_multi[2] = {};
    uint64_t graph_multi_key[2] = {};
    uint64_t graph_multi_kernels[2] = {};

    // stream-ordered timers and the launch counter
    cudaEvent_t timers[16] = {};
    uint64_t launches = 0;

    // mixed pair-pass variant: 0 = automatic, 1 = thread per atom, 2 = tiled
    int kernel_variant = 0;

    // adjoint (gx_adjoint.cu): checkpoints and work buffers, owned there
    void* adj = nullptr;

    // persistent neighbour list of the mixed pass (gx_nlist.cu), owned there;
    // nl_valid: the list matches buf[cur]'s order and home cells
    void* nl = nullptr;
    bool nl_valid = false;
    // nl_fresh: no position changed since a list-path tick, so the list holds
    // every pair within r_c of the current positions
    bool nl_fresh = false;

    // bond observation (gx_bondtrack.cu): open episodes on the device, owned there
    void* tracker = nullptr;
    void* lens = nullptr;     // analysis staging pool (gx_lens.cu)
    void* coll = nullptr;     // collision pass state (gx_lens.cu)
    void* xport = nullptr;    // XYZ frame buffers (gx_export.cu)
    void* snap = nullptr;     // snapshot encoder buffers (gx_snapshot.cu)
};

// Every kernel launch of the library goes through this macro so the
// handle's launch counter is exact.
#define GX_LAUNCH(h, kern, grid, block, ...)                          \
    do {                                                              \
        kern<<<(grid), (block), 0, (h)->stream>>>(__VA_ARGS__);       \
        ++(h)->launches;                                              \
    } while (0)

namespace gx {

constexpr int kRedCap = 4096;  // max reduction blocks per row

// Error helpers (host).
int set_err(gx_handle* h, int code, const std::string& msg);
int cuda_err(gx_handle* h, cudaError_t e, const char* what);
#define GX_CUDA(h, call)                                        \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return gx::cuda_err(h, e_, #call); \
    } while (0)

// Profiling wrappers around kernel launches.
void prof_begin(gx_handle* h, const char* name);
void prof_end(gx_handle* h, const char* name);

// Launchers implemented in the .cu files.
int ensure_cells(gx_handle* h, CellList& cl, uint32_t ncell);
// The counting sort's per-atom scratch (outside any stream capture).
int ensure_sort_tmp(gx_handle* h, CellList& cl, size_t n);
void cell_scan(gx_handle* h, CellList& cl, uint32_t ncell);
// Counting sort of atoms [0,n) by key into perm (sorted pos -> source index),
// deterministic (ties keep ascending source index).  cl.start gets cell starts.
// `gate` (may be null): a device word; the launches do nothing while it is 0.
int counting_sort(gx_handle* h, CellList& cl, uint32_t ncell, const uint32_t* key, uint32_t n,
                  uint32_t* perm, const uint32_t* gate = nullptr);
void launch_cell_keys(gx_handle* h, const GridGeom& g, const StateBuf& b, uint32_t n, uint32_t* key,
                      const uint32_t* gate = nullptr);
void launch_gather(gx_handle* h, const StateBuf& src, const StateBuf& dst, const uint32_t* perm,
                   const uint32_t* key_in, uint32_t* key_out, uint32_t n, uint32_t* pos_of_slot,
                   const uint32_t* gate = nullptr);
void launch_build_pos4(gx_handle* h, const GridGeom& g, const StateBuf& b, const uint32_t* key,
                       uint32_t n, float4* pos4);

int force_pass(gx_handle* h, bool finalize_acc, double* V, double* Vb, uint64_t* npairs, bool sync_out);
// The observed-bond spring over the device bond list (count in dcount[8])
// into F (mixed) or the accelerations (FP64), and its energy into dscal[3].
// `unit_mult`: every pair within the cutoff occurs once in the reference's
// pair list (a cell grid of at least 3 cells per axis).
int bond_spring(gx_handle* h, bool unit_mult);
// FP64 pair table on the device: sigma_ij then eps_ij, kNElem^2 each (gx_force.cu).
double* d_psig(gx_handle* h);
// out = the sum of part[0..nb) in a fixed order, one block (gx_force.cu).
void launch_sum_rows(gx_handle* h, const double* part, int nb, double* out);
inline bool bonds_on(const gx_handle* h) { return h->p.enable_bond_interaction && h->bonds_cap > 0; }
inline unsigned long long* dnbonds(gx_handle* h) { return h->dcount + 8; }
void adjoint_free(gx_handle* h);

// Neighbour-list path of the mixed pass (gx_nlist.cu).
bool nl_eligible(gx_handle* h);
int nl_prepare(gx_handle* h, bool* graphs_stale);
int nl_tick(gx_handle* h, const double* lambda, double* kpart, double* spart, int* nblocks, bool energy);
int nl_rebuilds(gx_handle* h, uint64_t* out);
int nl_set_skin(gx_handle* h, double skin);
int nl_tune_tpp(gx_handle* h, int reps);
int nl_config(gx_handle* h, double* skin, int* tpp);
int nl_set_tpp(gx_handle* h, int tpp);
int nl_set_slots(gx_handle* h, int slots);
int nl_set_brick(gx_handle* h, int cells);
int nl_set_block(gx_handle* h, int block);
int nl_shape(gx_handle* h, int* tpp, int* block, int* stash, int* brick);
int nl_stats(gx_handle* h, uint64_t* entries, uint64_t* overflowed);
void nl_free(gx_handle* h);
void tracker_free(gx_handle* h);
void lens_free(gx_handle* h);
// CollisionSystem on the device (gx_lens.cu): allocations outside any
// capture, one pass (launches), its counters (synchronises), release.
int collide_prepare(gx_handle* h);
int collide_pass(gx_handle* h);
int collide_read(gx_handle* h, unsigned long long* pass, unsigned long long* total);
void collide_free(gx_handle* h);
void export_free(gx_handle* h);  // gx_export.cu
void snapshot_free(gx_handle* h);  // gx_snapshot.cu
// Applies a pending Berendsen scale to v (any call that reads v commits it).
int commit_pending_lambda(gx_handle* h);
// After a wait on the stream: the error word an asynchronous gx_step left.
int take_step_errors(gx_handle* h);
// Waits for a queued asynchronous gx_step and reports its error word.  Every
// call that clears or consumes the device error word runs this first, so a
// step's error is never cleared before it is reported.
int settle_step_errors(gx_handle* h);

// Read-only view of the persistent neighbour list (gx_nlist.cu) for the
// passes that can take their candidates from it.  Entry e of atom p (sorted
// position) is list[e * stride + p] & idx_mask; atoms whose count exceeds
// cap_nb overflowed and scan the 27 list-grid cells around home[p] instead.
struct NlView {
    const uint32_t* list;
    size_t stride;
    int cap_nb;
    const uint32_t* cnt;
    GridGeom lg;
    const uint32_t* start;
    const uint32_t* home;
    uint32_t idx_mask;
};
// True (and the view) when h->nl_fresh: the list covers every pair within
// r_c of buf[cur], each unordered pair at least once with q > p.
bool nl_view(const gx_handle* h, NlView* v);

void launch_kick(gx_handle* h, const StateBuf& b, uint32_t n, double half_dt, const double* lambda);
void launch_drift(gx_handle* h, const StateBuf& b, uint32_t n, double dt);
void launch_wrap(gx_handle* h, const StateBuf& b, uint32_t n);
void launch_apply_lambda(gx_handle* h, const StateBuf& b, uint32_t n, double* lambda);
void launch_kinetic(gx_handle* h, const StateBuf& b, uint32_t n, const double* lambda, double* partials,
                    double* speed_partials, int* nblocks);
void launch_finalize_sum(gx_handle* h, const double* partials, int nblocks, double* out);
void launch_thermostat_lambda(gx_handle* h, const double* partials, int nblocks, double k, double target,
                              double tau, uint32_t n, double* lambda_out, double* K_out);

}  // namespace gx
