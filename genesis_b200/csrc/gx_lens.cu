// gx_lens.cu -- the observation lenses and the grid parity probes:
//   cell assignment           SpatialGrid::cell_of      src/physics/grid.rs:228-246
//   neighbour pairs           SpatialGrid::neighbors    src/physics/grid.rs:119-153
//   g(r), partial g(r)        radial_distribution(_between) src/analysis/mod.rs:87-201
//   friends-of-friends        clusters                  src/analysis/mod.rs:221-307
//   bound pairs               bound_pairs_with_grid     src/analysis/pairs.rs:132-174
//   elastic collisions        CollisionSystem::run      src/systems/collisions.rs:40-88
//   bond-graph components     bond_components           src/analysis/mod.rs:331-411
//                             + pair_potential_raw      src/physics/forces.rs:355-384
//
// Each lens builds its own grid (cell = the lens cutoff) over the selected
// atoms with the same counting sort as the force pass, then enumerates the
// canonical half shell.  Distance tests use the reference's FP64 operation
// order, so the pair multiset (including the repeats the reference produces
// on axes with exactly two cells) is identical to the reference's.
#include <cmath>
#include <cstring>

#include "gx_internal.cuh"

namespace gx {

struct AuxSet {
    double *x, *y, *z;
    uint8_t* elem;
    uint32_t* slot;
    uint32_t* key;  // aux-grid cell of each sorted aux atom
    const uint32_t* start;
    uint32_t m;
};

}  // namespace gx

using namespace gx;

namespace {

struct AuxPool {
    double* xyz = nullptr;  // 6 * cap: staging xyz + sorted xyz
    uint8_t* elem = nullptr;  // 2 * cap
    uint32_t* u32 = nullptr;  // 6 * cap: slot, slot_sorted, key, key_sorted, perm, sel
    size_t cap = 0;
    CellList cl;
    uint32_t* parent = nullptr;
    uint32_t* size = nullptr;
    uint32_t* entity = nullptr;
    size_t ucap = 0;
    unsigned long long* cnt = nullptr;  // 8 counters
    uint64_t* counts = nullptr;
    size_t ncap = 0;
};

void pool_release(AuxPool* P) {
    if (!P) return;
    void* ps[] = {P->xyz, P->elem, P->u32, P->parent, P->cnt, P->counts};
    for (void* q : ps) cudaFree(q);
    cells_free(P->cl);
    delete P;
}

// The handle's pool for the analysis calls, made on first use.
AuxPool& pool_of(gx_handle* h) {
    if (!h->lens) h->lens = new AuxPool();
    return *static_cast<AuxPool*>(h->lens);
}

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int ensure_pool(gx_handle* h, AuxPool& P, size_t m, size_t natoms) {
    if (m > P.cap) {
        cudaFree(P.xyz);
        cudaFree(P.elem);
        cudaFree(P.u32);
        size_t cap = m < 1024 ? 1024 : m;
        GX_CUDA(h, cudaMalloc(&P.xyz, 6 * cap * sizeof(double)));
        GX_CUDA(h, cudaMalloc(&P.elem, 2 * cap));
        GX_CUDA(h, cudaMalloc(&P.u32, 6 * cap * sizeof(uint32_t)));
        P.cap = cap;
    }
    if (natoms > P.ucap) {
        cudaFree(P.parent);
        size_t cap = natoms < 1024 ? 1024 : natoms;
        GX_CUDA(h, cudaMalloc(&P.parent, 3 * cap * sizeof(uint32_t)));
        P.size = P.parent + cap;
        P.entity = P.parent + 2 * cap;
        P.ucap = cap;
    }
    if (!P.cnt) GX_CUDA(h, cudaMalloc(&P.cnt, 8 * sizeof(unsigned long long)));
    return GX_OK;
}

__global__ void k_sample(const uint32_t* __restrict__ pos_of_slot, uint32_t count, uint32_t step,
                         uint32_t* __restrict__ sel) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < count) sel[q] = pos_of_slot[q * step];
}

__global__ void k_select(GridGeom g, StateBuf b, const uint32_t* __restrict__ sel, uint32_t m, double* tx, double* ty,
                         double* tz, uint8_t* te, uint32_t* tslot, uint32_t* key) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    uint32_t p = sel ? sel[q] : q;
    double x = b.x[p], y = b.y[p], z = b.z[p];
    tx[q] = x;
    ty[q] = y;
    tz[q] = z;
    te[q] = b.elem[p];
    tslot[q] = b.slot[p];
    key[q] = cell_of(g, x, y, z);
}

__global__ void k_aux_gather(const uint32_t* __restrict__ perm, uint32_t m, const double* tx, const double* ty,
                             const double* tz, const uint8_t* te, const uint32_t* tslot, const uint32_t* key,
                             AuxSet a) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    uint32_t q = perm[p];
    a.x[p] = tx[q];
    a.y[p] = ty[q];
    a.z[p] = tz[q];
    a.elem[p] = te[q];
    a.slot[p] = tslot[q];
    a.key[p] = key[q];
}

// The bond grid for the observation: every atom's cell, counted as it is
// found (count holds ncell + 1 entries), then placed straight into the
// sorted copy.  The order inside a cell is the order of the placing
// atomics, which the half-shell enumeration does not depend on: each pair
// of a cell is visited once (j > i) whatever the order, and pairs across
// cells by their cells alone.
__global__ void k_select_count(GridGeom g, StateBuf b, uint32_t m, uint32_t* __restrict__ key,
                               uint32_t* __restrict__ count) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    const uint32_t c = cell_of(g, b.x[q], b.y[q], b.z[q]);
    key[q] = c;
    atomicAdd(&count[c], 1u);
}

__global__ void k_place(StateBuf b, uint32_t m, const uint32_t* __restrict__ key, const uint32_t* __restrict__ start,
                        uint32_t* __restrict__ fill, AuxSet a) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    const uint32_t c = key[q];
    const uint32_t p = start[c] + atomicAdd(&fill[c], 1u);
    a.x[p] = b.x[q];
    a.y[p] = b.y[q];
    a.z[p] = b.z[q];
    a.elem[p] = b.elem[q];
    a.slot[p] = b.slot[q];
    a.key[p] = c;
}

// Canonical half-shell enumeration with the exact check_pair test
// (src/physics/grid.rs:201-225).  V::operator()(i, j, d) sees aux indices.
// min_image1 for a difference of which only the length is used: within
// 0.49 L the rounded quotient is below one half, round() gives zero and the
// reference's d - L * 0 is d itself (up to the sign of a zero).
__device__ __forceinline__ double near_image1(double d, double L) {
    return fabs(d) <= xmul(0.49, L) ? d : min_image1(d, L);
}

template <class V>
__global__ void k_pairs(GridGeom g, AuxSet a, double box0, double box1, double box2, double cd2, V visit) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    visit.begin();
    if (i < a.m) {
        uint32_t c = a.key[i];
        uint32_t cx, cy, cz;
        decode(g, c, cx, cy, cz);
        double xi = a.x[i], yi = a.y[i], zi = a.z[i];
        for (int k = -1; k < g.nhalf; ++k) {
            uint32_t B, lo;
            if (k < 0) {
                B = c;
                lo = i + 1;
            } else {
                B = encode(g, wrap_add(cx, g.half[k][0], g.n[0]), wrap_add(cy, g.half[k][1], g.n[1]),
                           wrap_add(cz, g.half[k][2], g.n[2]));
                lo = a.start[B];
            }
            uint32_t hi = a.start[B + 1];
            for (uint32_t j = lo; j < hi; ++j) {
                double dx = near_image1(xsub(xi, a.x[j]), box0);
                double dy = near_image1(xsub(yi, a.y[j]), box1);
                double dz = near_image1(xsub(zi, a.z[j]), box2);
                double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                if (d2 >= cd2) continue;
                double d = xsqrt(d2);
                if (d <= kEpsF64) continue;
                visit(a, i, j, d);
            }
        }
    }
    visit.end();
}

struct NeighborsVisit {
    uint32_t* out;
    size_t cap;
    unsigned long long* cnt;
    __device__ void begin() const {}
    __device__ void end() const {}
    __device__ void operator()(const AuxSet& a, uint32_t i, uint32_t j, double) const {
        unsigned long long k = atomicAdd(cnt, 1ull);
        if (k < cap) {
            out[2 * k] = a.slot[i];
            out[2 * k + 1] = a.slot[j];
        }
    }
};

// Up to this many bins, each block counts in shared memory and adds its
// nonzero bins to the global counts once (integer sums: the same result).
constexpr uint32_t kGrLocalBins = 1024;

struct GrVisit {
    double r_max, dr;
    unsigned long long* counts;
    uint32_t nbins;
    int ta, tb;
    uint32_t* err;
    __device__ unsigned* local() const {
        __shared__ unsigned hist[kGrLocalBins];
        return hist;
    }
    __device__ void begin() const {
        if (nbins > kGrLocalBins) return;
        unsigned* h = local();
        for (uint32_t k = threadIdx.x; k < nbins; k += blockDim.x) h[k] = 0u;
        __syncthreads();
    }
    __device__ void end() const {
        if (nbins > kGrLocalBins) return;
        __syncthreads();
        const unsigned* h = local();
        for (uint32_t k = threadIdx.x; k < nbins; k += blockDim.x)
            if (h[k]) atomicAdd(&counts[k], (unsigned long long)h[k]);
    }
    __device__ void operator()(const AuxSet& a, uint32_t i, uint32_t j, double d) const {
        if (ta >= 0) {
            int x = a.elem[i], y = a.elem[j];
            if (!((x == ta && y == tb) || (x == tb && y == ta))) return;
        }
        if (d >= r_max) return;  // analysis/mod.rs:113-115
        double f = xdiv(d, dr);  // (d / dr) as usize
        uint32_t bi = f >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)f;
        if (bi >= nbins) {
            atomicOr(err, kErrBinRange);
            return;
        }
        if (nbins <= kGrLocalBins)
            atomicAdd(&local()[bi], 1u);
        else
            atomicAdd(&counts[bi], 1ull);
    }
};

__device__ __forceinline__ uint32_t uf_root(uint32_t* par, uint32_t x) {
    uint32_t cur = par[x];
    if (cur != x) {
        uint32_t next, prev = x;
        while (cur > (next = par[cur])) {
            par[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}
__device__ __forceinline__ void uf_unite(uint32_t* par, uint32_t a, uint32_t b) {
    uint32_t ra = uf_root(par, a), rb = uf_root(par, b);
    while (ra != rb) {
        if (ra < rb) {
            uint32_t t = ra;
            ra = rb;
            rb = t;
        }
        uint32_t old = atomicCAS(&par[ra], ra, rb);
        if (old == ra) break;
        ra = uf_root(par, old);
        rb = uf_root(par, rb);
    }
}

struct FofVisit {
    double bond_factor;
    double sig[kNElem];
    uint32_t* parent;
    unsigned long long* bound;
    __device__ void begin() const {}
    __device__ void end() const {}
    __device__ void operator()(const AuxSet& a, uint32_t i, uint32_t j, double d) const {
        // bond = bond_factor * 0.5 * (sigma_a + sigma_b), analysis/mod.rs:250
        double bond = xmul(xmul(bond_factor, 0.5), xadd(sig[a.elem[i]], sig[a.elem[j]]));
        if (d < bond) {
            uf_unite(parent, a.slot[i], a.slot[j]);
            atomicAdd(bound, 1ull);
        }
    }
};

struct BoundVisit {
    double k_bind;
    double sig[kNElem];
    const uint32_t* entity;
    uint32_t* out;
    size_t cap;
    unsigned long long* cnt;
    __device__ void begin() const {}
    __device__ void end() const {}
    __device__ void operator()(const AuxSet& a, uint32_t i, uint32_t j, double d) const {
        // threshold = k_bind * mix_sigma, analysis/pairs.rs:163
        double threshold = xmul(k_bind, xmul(0.5, xadd(sig[a.elem[i]], sig[a.elem[j]])));
        if (!(d < threshold)) return;
        // entity ids (EntityId::index), or slot numbers when entity is null
        uint32_t ea = entity ? entity[a.slot[i]] : a.slot[i], eb = entity ? entity[a.slot[j]] : a.slot[j];
        if (eb < ea) {
            uint32_t t = ea;
            ea = eb;
            eb = t;
        }
        unsigned long long k = atomicAdd(cnt, 1ull);
        if (k < cap) {
            out[2 * k] = ea;
            out[2 * k + 1] = eb;
        }
    }
};

// CollisionSystem (src/systems/collisions.rs:40-88) on the collision grid
// (cell >= 2r): one thread per atom visits its own cell and every offset,
// as the FP64 force pass does, so a pair is seen as often as the reference's
// pair list holds it.  The impulse of elastic_pair
// (src/physics/collision.rs:16-32) is computed from the velocities before
// the pass; the atom's own half of it is exactly the negation of what its
// partner computes (the displacement, the relative velocity and the normal
// all flip sign exactly), so each thread sums its own velocity change with
// no atomics.  A collision is counted once per pair-list entry (through the
// canonical half shell, or j > i in the own cell).
__global__ void __launch_bounds__(128) k_collide(GridGeom g, AuxSet a, StateBuf b,
                                                 const uint32_t* __restrict__ pos_of_slot, double box0, double box1,
                                                 double box2, double cd2, double* __restrict__ dv, size_t stride,
                                                 unsigned long long* __restrict__ count) {
    __shared__ unsigned int sc;
    if (threadIdx.x == 0) sc = 0u;
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.m) {
        const uint32_t c = a.key[i];
        uint32_t cx, cy, cz;
        decode(g, c, cx, cy, cz);
        const double xi = a.x[i], yi = a.y[i], zi = a.z[i];
        const uint32_t si = a.slot[i], pi = pos_of_slot[si];
        const double vxi = b.vx[pi], vyi = b.vy[pi], vzi = b.vz[pi], mi = b.mass[pi];
        double dvx = 0.0, dvy = 0.0, dvz = 0.0;
        unsigned int cnt = 0u;
        for (int k = -1; k < g.nfull; ++k) {
            const uint32_t B = k < 0 ? c
                                     : encode(g, wrap_add(cx, g.full[k][0], g.n[0]), wrap_add(cy, g.full[k][1], g.n[1]),
                                              wrap_add(cz, g.full[k][2], g.n[2]));
            for (uint32_t j = a.start[B], hi = a.start[B + 1]; j < hi; ++j) {
                if (j == i) continue;
                const double dx = min_image1(xsub(xi, a.x[j]), box0);
                const double dy = min_image1(xsub(yi, a.y[j]), box1);
                const double dz = min_image1(xsub(zi, a.z[j]), box2);
                const double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                if (d2 >= cd2) continue;
                const double d = xsqrt(d2);
                if (d <= kEpsF64) continue;  // check_pair, grid.rs:201-225
                const uint32_t pj = pos_of_slot[a.slot[j]];
                const double mj = b.mass[pj];
                if (mi <= 0.0 || mj <= 0.0) continue;
                const double inv = xdiv(1.0, d);
                const double nx = xmul(dx, inv), ny = xmul(dy, inv), nz = xmul(dz, inv);
                const double rx = xsub(vxi, b.vx[pj]), ry = xsub(vyi, b.vy[pj]), rz = xsub(vzi, b.vz[pj]);
                const double vn = xadd(xadd(xmul(rx, nx), xmul(ry, ny)), xmul(rz, nz));
                if (vn >= 0.0) continue;  // separating: no impulse
                const double jj = xdiv(xmul(-2.0, vn), xadd(xdiv(1.0, mi), xdiv(1.0, mj)));
                const double im = xdiv(1.0, mi);
                const double ax = xmul(xmul(nx, jj), im), ay = xmul(xmul(ny, jj), im), az = xmul(xmul(nz, jj), im);
                if (ax == 0.0 && ay == 0.0 && az == 0.0) continue;
                dvx = xadd(dvx, ax);
                dvy = xadd(dvy, ay);
                dvz = xadd(dvz, az);
                if (k < 0 ? j > i : k < g.nhalf) ++cnt;
            }
        }
        dv[si] = dvx;
        dv[stride + si] = dvy;
        dv[2 * stride + si] = dvz;
        if (cnt) atomicAdd(&sc, cnt);
    }
    __syncthreads();
    if (threadIdx.x == 0 && sc) atomicAdd(count, (unsigned long long)sc);
}

// vel += dv for every atom once any pair collided (collisions.rs:80-84).
__global__ void k_apply_dv(StateBuf b, const uint32_t* __restrict__ pos_of_slot, const double* __restrict__ dv,
                           size_t stride, uint32_t n, const unsigned long long* __restrict__ count) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || *count == 0ull) return;
    const uint32_t p = pos_of_slot[s];
    b.vx[p] = xadd(b.vx[p], dv[s]);
    b.vy[p] = xadd(b.vy[p], dv[stride + s]);
    b.vz[p] = xadd(b.vz[p], dv[2 * stride + s]);
}

__global__ void k_add_total(unsigned long long* c) { c[1] += c[0]; }

// Components of the bond list (bond_components, src/analysis/mod.rs:331-411):
// union-find over the bonds, the label of a bonded slot is its root (the
// smallest slot of the component), an atom in no bond gets 0xFFFFFFFF.
__global__ void k_bond_unite(const uint32_t* __restrict__ bonds, size_t nb, uint32_t n, uint32_t* par,
                             uint32_t* __restrict__ mark) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const uint32_t a = bonds[2 * k], b = bonds[2 * k + 1];
    if (a >= n || b >= n) return;
    mark[a] = 1u;
    mark[b] = 1u;
    if (a != b) uf_unite(par, a, b);
}

__global__ void k_bond_labels(uint32_t* par, const uint32_t* __restrict__ mark, uint32_t n,
                              uint32_t* __restrict__ label) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) label[i] = mark[i] ? uf_root(par, i) : 0xFFFFFFFFu;
}

// pair_potential_raw (src/physics/forces.rs:360-384) of each bond at the
// current positions, in the reference's operation order: r = max(|min
// image of pa - pb|, 1e-9) (bond_structure.rs:113), unswitched LJ without
// the core clamp (lj_raw, forces.rs:346-353), + k_e q_a q_b / r, + the
// harmonic term 0.5 k (r - r_eq)^2 with k = well_curvature, r_eq =
// equilibrium_distance (forces.rs:193-195, 281-283).
struct RawLaw {
    double sig[kNElem * kNElem], eps[kNElem * kNElem], qq[kNElem * kNElem];
    double curv_factor, r_eq_factor;
    double box[3];
    int coulomb, bond;
};

__global__ void k_bond_energy(const uint32_t* __restrict__ bonds, size_t nb, StateBuf b,
                              const uint32_t* __restrict__ pos_of_slot, RawLaw L, double* __restrict__ energy) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const uint32_t ia = pos_of_slot[bonds[2 * k]], ib = pos_of_slot[bonds[2 * k + 1]];
    const double dx = min_image1(xsub(b.x[ia], b.x[ib]), L.box[0]);
    const double dy = min_image1(xsub(b.y[ia], b.y[ib]), L.box[1]);
    const double dz = min_image1(xsub(b.z[ia], b.z[ib]), L.box[2]);
    const double r = fmax(xsqrt(xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz))), 1e-9);
    const int t = b.elem[ia] * kNElem + b.elem[ib];
    const double sg = L.sig[t], ep = L.eps[t];
    const double s = xdiv(sg, r);
    const double s6 = xmul(xmul(xmul(xmul(xmul(s, s), s), s), s), s);
    const double s12 = xmul(s6, s6);
    double v = xmul(xmul(4.0, ep), xsub(s12, s6));
    if (L.coulomb) v = xadd(v, xdiv(L.qq[t], r));
    if (L.bond) {
        const double kk = xdiv(xmul(L.curv_factor, ep), xmul(sg, sg));
        const double dr = xsub(r, xmul(sg, L.r_eq_factor));
        v = xadd(v, xmul(xmul(xmul(0.5, kk), dr), dr));
    }
    energy[k] = v;
}

// Bound pairs routed to their owner: the pair (slot a < slot b) is appended
// to a's bucket [k * stride + a] (k < depth; the count runs on past the
// depth, so an overflow shows, and the counts sum to the number of pairs
// found, duplicates of a 2-cell axis included).  The enumeration is
// k_pairs' (the same cells, candidates and exact test), with 16 lanes per
// atom: lane 0 scans the atom's own cell, lane k + 1 the half-shell
// neighbour k, so that the chains of dependent loads run side by side.
constexpr int kBucketLanes = 16;

static_assert(kBucketLanes >= 14, "one lane per half-shell cell and the own cell");

struct BucketArgs {
    double k_bind;
    double sig[kNElem];
    uint32_t* bucket;
    uint32_t* bcnt;
    uint32_t depth;
    size_t stride;
};

// One candidate of bound_pairs_with_grid (pairs.rs:150-170): the exact
// test, then (lower slot, higher slot) appended to the lower slot's bucket.
__device__ __forceinline__ void bound_candidate(double xi, double yi, double zi, double si, uint32_t slot_i, double xj,
                                                double yj, double zj, double sj, uint32_t slot_j, double box0,
                                                double box1, double box2, double cd2, const BucketArgs& v) {
    double dx = near_image1(xsub(xi, xj), box0);
    double dy = near_image1(xsub(yi, yj), box1);
    double dz = near_image1(xsub(zi, zj), box2);
    double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
    if (d2 >= cd2) return;
    double threshold = xmul(v.k_bind, xmul(0.5, xadd(si, sj)));  // pairs.rs:163
    // d = sqrt(d2) (correctly rounded) against the threshold, decided
    // on d2 away from the boundary: beyond 1e-12 relative either way
    // the rounded root cannot fall on the other side
    const double t2 = xmul(threshold, threshold);
    if (d2 >= xmul(t2, 1.0 + 1e-12)) return;
    if (d2 > xmul(t2, 1.0 - 1e-12) || d2 <= 1e-30) {
        double d = xsqrt(d2);
        if (d <= kEpsF64) return;  // check_pair, grid.rs:201-225
        if (!(d < threshold)) return;
    }
    uint32_t sa = slot_i, sb = slot_j;
    if (sb < sa) {
        uint32_t q = sa;
        sa = sb;
        sb = q;
    }
    uint32_t r = atomicAdd(&v.bcnt[sa], 1u);
    if (r < v.depth) v.bucket[(size_t)r * v.stride + sa] = sb;
}

__global__ void __launch_bounds__(256) k_bound_buckets(GridGeom g, AuxSet a, double box0, double box1, double box2,
                                                       double cd2, BucketArgs v) {
    // the offsets and sigmas, indexed per lane and per atom, from shared
    // memory (constant-index copies: no per-thread copy of the parameters)
    __shared__ int8_t half[13][3];
    __shared__ double sig[kNElem];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 13; ++q) {
            half[q][0] = g.half[q][0];
            half[q][1] = g.half[q][1];
            half[q][2] = g.half[q][2];
        }
#pragma unroll
        for (int q = 0; q < kNElem; ++q) sig[q] = v.sig[q];
    }
    __syncthreads();
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / kBucketLanes;
    const int k = (int)(t % kBucketLanes) - 1;
    if (i < a.m && k < g.nhalf) {
        const uint32_t c = a.key[i];
        uint32_t B, lo;
        if (k < 0) {
            B = c;
            lo = i + 1;
        } else {
            uint32_t cx, cy, cz;
            decode(g, c, cx, cy, cz);
            B = encode(g, wrap_add(cx, half[k][0], g.n[0]), wrap_add(cy, half[k][1], g.n[1]),
                       wrap_add(cz, half[k][2], g.n[2]));
            lo = a.start[B];
        }
        const uint32_t hi = a.start[B + 1];
        const double xi = a.x[i], yi = a.y[i], zi = a.z[i];
        const double si = sig[a.elem[i]];
        const uint32_t slot_i = a.slot[i];
        for (uint32_t j = lo; j < hi; ++j)
            bound_candidate(xi, yi, zi, si, slot_i, a.x[j], a.y[j], a.z[j], sig[a.elem[j]], a.slot[j], box0, box1,
                            box2, cd2, v);
    }
}

// The same decisions with the candidates taken from the persistent neighbour
// list, which holds every pair within r_c (> the bond cutoff) of the current
// positions: each unordered pair once, from its lower sorted position.  No
// bond grid is binned.  kListBoundLanes lanes per atom take its entries in
// turn (short chains of dependent gathers side by side).
constexpr int kListBoundLanes = 8;
__global__ void __launch_bounds__(256) k_bound_from_list(StateBuf b, uint32_t n, NlView nv, double box0, double box1,
                                                         double box2, double cd2, BucketArgs v) {
    __shared__ double sig[kNElem];
    if (threadIdx.x < kNElem) sig[threadIdx.x] = v.sig[threadIdx.x];
    __syncthreads();
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t p = (uint32_t)(t / kListBoundLanes);
    const uint32_t lane = (uint32_t)(t % kListBoundLanes);
    if (p >= n) return;
    const double xi = b.x[p], yi = b.y[p], zi = b.z[p];
    const double si = sig[b.elem[p]];
    const uint32_t slot_i = b.slot[p];
    const uint32_t m = nv.cnt[p];
    if (m <= (uint32_t)nv.cap_nb) {
        for (uint32_t e = lane; e < m; e += kListBoundLanes) {
            const uint32_t q = __ldg(nv.list + (size_t)e * nv.stride + p) & nv.idx_mask;
            if (q > p)
                bound_candidate(xi, yi, zi, si, slot_i, b.x[q], b.y[q], b.z[q], sig[b.elem[q]], b.slot[q], box0, box1,
                                box2, cd2, v);
        }
    } else {  // overflowed list: the list-grid cells from the home cell on (sorted by cell: q > p)
        const uint32_t c = nv.home[p];
        uint32_t cx, cy, cz;
        decode(nv.lg, c, cx, cy, cz);
        for (uint32_t code = lane; code < 27; code += kListBoundLanes) {
            const int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
            const uint32_t B = encode(nv.lg, wrap_add(cx, ox, nv.lg.n[0]), wrap_add(cy, oy, nv.lg.n[1]),
                                      wrap_add(cz, oz, nv.lg.n[2]));
            if (B < c) continue;
            for (uint32_t q = nv.start[B], hi = nv.start[B + 1]; q < hi; ++q)
                if (q > p)
                    bound_candidate(xi, yi, zi, si, slot_i, b.x[q], b.y[q], b.z[q], sig[b.elem[q]], b.slot[q], box0,
                                    box1, box2, cd2, v);
        }
    }
}

__global__ void k_iota(uint32_t* p, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}
__global__ void k_fof_finish(uint32_t* par, uint32_t* size, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t r = uf_root(par, i);
    atomicAdd(&size[r], 1u);
}
__global__ void k_fof_labels(uint32_t* par, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    par[i] = uf_root(par, i);
}
// cnt[0] monomers, [1] aggregates, [2] largest, [3] components
__global__ void k_fof_stats(const uint32_t* size, const uint32_t* par, uint32_t n, unsigned long long* cnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || par[i] != i) return;
    uint32_t s = size[i];
    atomicAdd(&cnt[3], 1ull);
    if (s == 1) atomicAdd(&cnt[0], 1ull);
    else atomicAdd(&cnt[1], 1ull);
    atomicMax(&cnt[2], (unsigned long long)s);
}
__global__ void k_cell_assign(GridGeom g, StateBuf b, uint32_t n, uint32_t* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[b.slot[i]] = cell_of(g, b.x[i], b.y[i], b.z[i]);
}

// Builds the aux grid over m selected atoms (sel = sorted positions, or
// nullptr for all atoms).
int build_aux(gx_handle* h, AuxPool& P, const GridGeom& g, const uint32_t* sel, uint32_t m, AuxSet& a) {
    size_t cap = P.cap;
    double* tx = P.xyz;
    double* ty = tx + cap;
    double* tz = ty + cap;
    a.x = P.xyz + 3 * cap;
    a.y = a.x + cap;
    a.z = a.y + cap;
    uint8_t* te = P.elem;
    a.elem = P.elem + cap;
    uint32_t* tslot = P.u32;
    a.slot = P.u32 + cap;
    uint32_t* key = P.u32 + 2 * cap;
    a.key = P.u32 + 3 * cap;
    uint32_t* perm = P.u32 + 4 * cap;
    a.m = m;
    if (m) GX_LAUNCH(h, k_select, nblk(m, 256), 256, g, h->buf[h->cur], sel, m, tx, ty, tz, te, tslot, key);
    int rc = counting_sort(h, P.cl, g.ncell, key, m, perm);
    if (rc) return rc;
    if (m) GX_LAUNCH(h, k_aux_gather, nblk(m, 256), 256, perm, m, tx, ty, tz, te, tslot, key, a);
    a.start = P.cl.start;
    return GX_OK;
}

int require(gx_handle* h) {
    if (!h) return GX_ERR_ARG;
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    return GX_OK;
}

int gr_common(gx_handle* h, int ta, int tb, double r_max_in, size_t nbins_in, size_t sample_cap, uint64_t* counts,
              double* bins, double* rmo, double* dro) {
    int rc = require(h);
    if (rc) return rc;
    if (!counts) return GX_ERR_ARG;
    if ((rc = settle_step_errors(h))) return rc;  // this call clears the error word below
    size_t nbins = nbins_in < 1 ? 1 : (nbins_in > 65536 ? 65536 : nbins_in);
    const double* box = h->p.box;
    double half_min = std::fmin(std::fmin(box[0], box[1]), box[2]) * 0.5;
    double r_max = std::fmin(std::fmax(r_max_in, 1e-9), half_min);
    double dr = r_max / (double)nbins;
    double vol = box[0] * box[1] * box[2];
    size_t n = h->n;
    // g_subsample (analysis/mod.rs:32-46)
    size_t step = 1, m = n;
    if (sample_cap && n > sample_cap) {
        step = n / sample_cap + 1;
        m = n / step;
    }
    AuxPool& P = pool_of(h);
    if ((rc = ensure_pool(h, P, m, n))) return rc;
    if (nbins > P.ncap) {
        cudaFree(P.counts);
        GX_CUDA(h, cudaMalloc(&P.counts, nbins * sizeof(uint64_t)));
        P.ncap = nbins;
    }
    uint32_t* sel = nullptr;
    if (step > 1) {
        sel = P.u32 + 5 * P.cap;
        GX_LAUNCH(h, k_sample, nblk(m, 256), 256, h->pos_of_slot, (uint32_t)m, (uint32_t)step, sel);
    }
    int ok = 0;
    GridGeom g = make_grid(box, r_max, &ok);
    if (!ok) return set_err(h, GX_ERR_UNSUPPORTED, "g(r) grid too large");
    AuxSet a;
    if ((rc = build_aux(h, P, g, sel, (uint32_t)m, a))) return rc;
    GX_CUDA(h, cudaMemsetAsync(P.counts, 0, nbins * sizeof(uint64_t), h->stream));
    GX_CUDA(h, cudaMemsetAsync(h->derr, 0, sizeof(uint32_t), h->stream));
    GrVisit v{r_max, dr, (unsigned long long*)P.counts, (uint32_t)nbins, ta, tb, h->derr};
    prof_begin(h, "gr_pairs");
    if (m) GX_LAUNCH(h, k_pairs, nblk(m, 128), 128, g, a, box[0], box[1], box[2], r_max * r_max, v);
    prof_end(h, "gr_pairs");
    uint32_t e = 0;
    GX_CUDA(h, cudaMemcpyAsync(counts, P.counts, nbins * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaMemcpyAsync(&e, h->derr, sizeof e, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    if (rmo) *rmo = r_max;
    if (dro) *dro = dr;
    // normalisation on the host (analysis/mod.rs:119-132, 184-199)
    if (bins) {
        for (size_t i = 0; i < nbins; ++i) bins[i] = 0.0;
        double pair_count = 0.0;
        bool partial = ta >= 0;
        if (partial) {
            // species counts of the sample come from the counts kernel-free path:
            // recount on the host from the element column of the sample.
            std::vector<uint8_t> el(m);
            GX_CUDA(h, cudaMemcpy(el.data(), a.elem, m, cudaMemcpyDeviceToHost));
            size_t na = 0, nb = 0;
            for (uint8_t t : el) {
                na += t == ta;
                nb += t == tb;
            }
            pair_count = ta == tb ? (double)na * (double)(na == 0 ? 0 : na - 1) * 0.5 : (double)na * (double)nb;
        }
        bool skip = partial ? !(pair_count > 0.0) : m < 2;
        if (!skip) {
            const double pi = 3.141592653589793;
            for (size_t i = 0; i < nbins; ++i) {
                double r_lo = (double)i * dr;
                double r_hi = r_lo + dr;
                double shell = 4.0 / 3.0 * pi * (r_hi * r_hi * r_hi - r_lo * r_lo * r_lo);
                double expected = partial ? pair_count * shell / vol : (double)(m * (m - 1)) * 0.5 * shell / vol;
                bins[i] = (double)counts[i] / std::fmax(expected, 2.2250738585072014e-308);
            }
        }
    }
    if (e & kErrBinRange) return set_err(h, GX_ERR_CAPACITY, "a distance rounded into bin nbins (the reference panics here)");
    return GX_OK;
}

}  // namespace

extern "C" {

int gx_cell_assign(gx_handle* h, double min_cell, uint32_t* cells) {
    int rc = require(h);
    if (rc) return rc;
    if (!cells) return GX_ERR_ARG;
    int ok = 0;
    GridGeom g = make_grid(h->p.box, min_cell, &ok);
    if (!ok) return set_err(h, GX_ERR_ARG, "invalid grid");
    AuxPool& P = pool_of(h);
    if ((rc = ensure_pool(h, P, h->n, h->n))) return rc;
    uint32_t n = (uint32_t)h->n;
    if (n) GX_LAUNCH(h, k_cell_assign, nblk(n, 256), 256, g, h->buf[h->cur], n, P.u32);
    if (n) GX_CUDA(h, cudaMemcpyAsync(cells, P.u32, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_neighbors(gx_handle* h, double min_cell, double cutoff, uint32_t* pairs, size_t cap, size_t* npairs) {
    int rc = require(h);
    if (rc) return rc;
    if (cap && !pairs) return GX_ERR_ARG;
    int ok = 0;
    GridGeom g = make_grid(h->p.box, min_cell, &ok);
    if (!ok) return set_err(h, GX_ERR_ARG, "invalid grid");
    AuxPool& P = pool_of(h);
    uint32_t n = (uint32_t)h->n;
    if ((rc = ensure_pool(h, P, n, n))) return rc;
    AuxSet a;
    if ((rc = build_aux(h, P, g, nullptr, n, a))) return rc;
    uint32_t* dout = nullptr;
    if (cap) GX_CUDA(h, cudaMalloc(&dout, 2 * cap * sizeof(uint32_t)));
    GX_CUDA(h, cudaMemsetAsync(P.cnt, 0, sizeof(unsigned long long), h->stream));
    NeighborsVisit v{dout, cap, P.cnt};
    if (n) GX_LAUNCH(h, k_pairs, nblk(n, 128), 128, g, a, h->p.box[0], h->p.box[1], h->p.box[2], cutoff * cutoff, v);
    unsigned long long total = 0;
    GX_CUDA(h, cudaMemcpyAsync(&total, P.cnt, sizeof total, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    size_t w = total < cap ? (size_t)total : cap;
    if (w) GX_CUDA(h, cudaMemcpy(pairs, dout, 2 * w * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    cudaFree(dout);
    if (npairs) *npairs = (size_t)total;
    GX_CUDA(h, cudaGetLastError());
    return total > cap ? set_err(h, GX_ERR_CAPACITY, "pair buffer too small") : GX_OK;
}

int gx_radial_distribution(gx_handle* h, double r_max, size_t nbins, size_t sample_cap, uint64_t* counts,
                           double* bins, double* r_max_out, double* dr_out) {
    return gr_common(h, -1, -1, r_max, nbins, sample_cap, counts, bins, r_max_out, dr_out);
}

int gx_radial_distribution_between(gx_handle* h, uint8_t ta, uint8_t tb, double r_max, size_t nbins,
                                   size_t sample_cap, uint64_t* counts, double* bins, double* r_max_out,
                                   double* dr_out) {
    if (ta >= kNElem || tb >= kNElem) return GX_ERR_ARG;
    return gr_common(h, ta, tb, r_max, nbins, sample_cap, counts, bins, r_max_out, dr_out);
}

int gx_collision_count(gx_handle* h, uint64_t* total) {
    if (!h || !total) return GX_ERR_ARG;
    unsigned long long pass = 0, all = 0;
    int rc = collide_read(h, &pass, &all);
    *total = all;
    return rc;
}

int gx_bond_components(gx_handle* h, uint32_t* labels, double* edge_energy, size_t energy_cap, size_t* nbonds) {
    int rc = require(h);
    if (rc) return rc;
    const uint32_t n = (uint32_t)h->n;
    const size_t nb = h->bonds ? h->nbonds : 0;
    if (nbonds) *nbonds = nb;
    if (edge_energy && energy_cap < nb) return set_err(h, GX_ERR_CAPACITY, "edge_energy holds fewer than nbonds");
    if (n == 0) return GX_OK;
    AuxPool& P = pool_of(h);
    if ((rc = ensure_pool(h, P, n, n))) return rc;
    const StateBuf& b = h->buf[h->cur];
    if (labels) {
        GX_LAUNCH(h, k_iota, nblk(n, 256), 256, P.parent, n);
        GX_CUDA(h, cudaMemsetAsync(P.size, 0, n * sizeof(uint32_t), h->stream));
        if (nb) GX_LAUNCH(h, k_bond_unite, nblk(nb, 256), 256, h->bonds, nb, n, P.parent, P.size);
        GX_LAUNCH(h, k_bond_labels, nblk(n, 256), 256, P.parent, P.size, n, P.entity);
        GX_CUDA(h, cudaMemcpyAsync(labels, P.entity, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    }
    double* tmp = nullptr;
    if (edge_energy && nb) {
        RawLaw L;
        for (int a = 0; a < kNElem; ++a)
            for (int c = 0; c < kNElem; ++c) {  // mix_sigma, mix_epsilon (forces.rs:127-134)
                L.sig[a * kNElem + c] = 0.5 * (h->p.sigma[a] + h->p.sigma[c]);
                L.eps[a * kNElem + c] = h->p.thermal_constant * std::sqrt(h->p.epsilon_k[a] * h->p.epsilon_k[c]);
                L.qq[a * kNElem + c] = h->p.coulomb_constant * h->p.charge[a] * h->p.charge[c];
            }
        L.curv_factor = 72.0 * std::pow(2.0, -1.0 / 3.0);
        L.r_eq_factor = std::pow(2.0, 1.0 / 6.0);
        for (int k = 0; k < 3; ++k) L.box[k] = h->p.box[k];
        L.coulomb = h->p.enable_electrostatics ? 1 : 0;
        L.bond = h->p.enable_bond_interaction ? 1 : 0;
        double* dst = P.xyz;
        if (nb > 6 * P.cap) {
            GX_CUDA(h, cudaMalloc(&tmp, nb * sizeof(double)));
            dst = tmp;
        }
        GX_LAUNCH(h, k_bond_energy, nblk(nb, 256), 256, h->bonds, nb, b, h->pos_of_slot, L, dst);
        cudaError_t e = cudaMemcpyAsync(edge_energy, dst, nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) return cuda_err(h, e, "gx_bond_components");
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}

int gx_clusters(gx_handle* h, double bond_factor, uint32_t* labels, uint64_t stats[4], double* mean_size) {
    int rc = require(h);
    if (rc) return rc;
    if (!stats) return GX_ERR_ARG;
    stats[0] = stats[1] = stats[2] = stats[3] = 0;
    if (mean_size) *mean_size = 0.0;
    uint32_t n = (uint32_t)h->n;
    if (n == 0) return GX_OK;  // analysis/mod.rs:230-232
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    AuxPool& P = pool_of(h);
    if ((rc = ensure_pool(h, P, n, n))) return rc;
    // max sigma over the particles present (analysis/mod.rs:236-238): the
    // kind table of gx_set_state lists every element present, unless it
    // overflowed, when the element column is read back
    double max_sigma = 0.0;
    if (h->nkinds <= kMaxKinds) {
        for (int k = 0; k < h->nkinds; ++k) max_sigma = std::fmax(max_sigma, h->p.sigma[h->kind_elem[k]]);
    } else {
        std::vector<uint8_t> el(n);
        GX_CUDA(h, cudaMemcpy(el.data(), h->buf[h->cur].elem, n, cudaMemcpyDeviceToHost));
        for (uint8_t t : el) max_sigma = std::fmax(max_sigma, h->p.sigma[t]);
    }
    double cutoff = std::fmax(std::fmax(bond_factor, 0.1) * max_sigma, 1e-9);
    int ok = 0;
    GridGeom g = make_grid(h->p.box, cutoff, &ok);
    if (!ok) return set_err(h, GX_ERR_UNSUPPORTED, "FoF grid too large");
    AuxSet a;
    if ((rc = build_aux(h, P, g, nullptr, n, a))) return rc;
    GX_LAUNCH(h, k_iota, nblk(n, 256), 256, P.parent, n);
    GX_CUDA(h, cudaMemsetAsync(P.size, 0, n * sizeof(uint32_t), h->stream));
    GX_CUDA(h, cudaMemsetAsync(P.cnt, 0, 8 * sizeof(unsigned long long), h->stream));
    FofVisit v;
    v.bond_factor = bond_factor;
    for (int k = 0; k < kNElem; ++k) v.sig[k] = h->p.sigma[k];
    v.parent = P.parent;
    v.bound = P.cnt + 4;
    prof_begin(h, "fof_pairs");
    GX_LAUNCH(h, k_pairs, nblk(n, 128), 128, g, a, h->p.box[0], h->p.box[1], h->p.box[2], cutoff * cutoff, v);
    prof_end(h, "fof_pairs");
    GX_LAUNCH(h, k_fof_finish, nblk(n, 256), 256, P.parent, P.size, n);
    GX_LAUNCH(h, k_fof_labels, nblk(n, 256), 256, P.parent, n);
    GX_LAUNCH(h, k_fof_stats, nblk(n, 256), 256, P.size, P.parent, n, P.cnt);
    unsigned long long c[8];
    GX_CUDA(h, cudaMemcpyAsync(c, P.cnt, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    if (labels) GX_CUDA(h, cudaMemcpyAsync(labels, P.parent, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    stats[0] = c[0];
    stats[1] = c[1];
    stats[2] = c[2];
    stats[3] = c[4];
    if (mean_size) *mean_size = (double)n / (double)(c[3] > 0 ? c[3] : 1);
    return GX_OK;
}

}  // extern "C"

namespace gx {

void lens_free(gx_handle* h) {
    pool_release(static_cast<AuxPool*>(h->lens));
    h->lens = nullptr;
}

// The collision pass's own staging, so that a captured tick holds fixed
// addresses: the binned copy of the atoms, the velocity changes (3 x cap by
// slot) and the counters ([0] this pass, [1] cumulative).
struct CollideState {
    AuxPool* pool = nullptr;
    double* dv = nullptr;
    size_t cap = 0;
    unsigned long long* cnt = nullptr;
};

void collide_free(gx_handle* h) {
    CollideState* c = static_cast<CollideState*>(h->coll);
    if (!c) return;
    pool_release(c->pool);
    cudaFree(c->dv);
    cudaFree(c->cnt);
    delete c;
    h->coll = nullptr;
}

static GridGeom collide_grid(gx_handle* h, int* ok) {
    return make_grid(h->p.box, 2.0 * h->p.particle_radius, ok);  // CollisionSystem::new, collisions.rs:16-21
}

// Allocations of the pass, outside any capture.
int collide_prepare(gx_handle* h) {
    if (!(h->p.particle_radius > 0.0)) return set_err(h, GX_ERR_ARG, "particle_radius must be positive");
    int ok = 0;
    GridGeom g = collide_grid(h, &ok);
    if (!ok) return set_err(h, GX_ERR_ARG, "collision grid is empty or too large");
    if (!h->coll) h->coll = new CollideState();
    CollideState* c = static_cast<CollideState*>(h->coll);
    if (!c->pool) c->pool = new AuxPool();
    int rc = ensure_pool(h, *c->pool, h->n, h->n);
    if (!rc) rc = ensure_cells(h, c->pool->cl, g.ncell);
    if (!rc) rc = ensure_sort_tmp(h, c->pool->cl, h->cap);  // the pass runs inside captured ticks
    if (rc) return rc;
    if (c->cap < h->cap) {
        cudaFree(c->dv);
        c->dv = nullptr;
        GX_CUDA(h, cudaMalloc(&c->dv, 3 * h->cap * sizeof(double)));
        c->cap = h->cap;
    }
    if (!c->cnt) {
        GX_CUDA(h, cudaMalloc(&c->cnt, 2 * sizeof(unsigned long long)));
        GX_CUDA(h, cudaMemsetAsync(c->cnt, 0, 2 * sizeof(unsigned long long), h->stream));
    }
    return GX_OK;
}

// The counters of the last pass and of all passes (synchronises).
int collide_read(gx_handle* h, unsigned long long* pass, unsigned long long* total) {
    *pass = *total = 0;
    CollideState* c = static_cast<CollideState*>(h->coll);
    if (!c || !c->cnt) return GX_OK;
    unsigned long long v[2] = {0, 0};
    GX_CUDA(h, cudaMemcpyAsync(v, c->cnt, sizeof v, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    *pass = v[0];
    *total = v[1];
    return GX_OK;
}

// One pass on the handle's stream (launches only; collide_prepare first).
int collide_pass(gx_handle* h) {
    const uint32_t n = (uint32_t)h->n;
    if (!n) return GX_OK;
    CollideState* c = static_cast<CollideState*>(h->coll);
    int ok = 0;
    GridGeom g = collide_grid(h, &ok);
    AuxSet a;
    int rc = build_aux(h, *c->pool, g, nullptr, n, a);
    if (rc) return rc;
    const double contact = 2.0 * h->p.particle_radius;
    prof_begin(h, "collisions");
    GX_CUDA(h, cudaMemsetAsync(c->cnt, 0, sizeof(unsigned long long), h->stream));
    GX_LAUNCH(h, k_collide, nblk(n, 128), 128, g, a, h->buf[h->cur], h->pos_of_slot, h->p.box[0], h->p.box[1],
              h->p.box[2], contact * contact, c->dv, c->cap, c->cnt);
    GX_LAUNCH(h, k_apply_dv, nblk(n, 256), 256, h->buf[h->cur], h->pos_of_slot, c->dv, c->cap, n, c->cnt);
    GX_LAUNCH(h, k_add_total, 1, 1, c->cnt);
    prof_end(h, "collisions");
    return GX_OK;
}

void aux_pool_free(void* pool) { pool_release(static_cast<AuxPool*>(pool)); }

// The neighbour list can stand in for the bond grid when it holds every pair
// within the bond cutoff (positions unchanged since a list tick, cutoff
// below r_c) and the bond grid has at least 3 cells per axis, where the
// reference's grid reports each pair exactly once.
bool bound_from_list(const gx_handle* h, double cutoff, const GridGeom& bond_grid, NlView* nv) {
    if (!(cutoff < 0.99 * h->fs.rc)) return false;
    for (int k = 0; k < 3; ++k)
        if (bond_grid.n[k] < 3) return false;
    return nl_view(h, nv);
}

// What a captured observation depends on when it takes the list path: the
// list and its cell starts (null on the bond-grid path).
void bound_list_key(const gx_handle* h, double k_bind, const void** list, const void** start) {
    *list = *start = nullptr;
    double ms = 0.0;
    for (int k = 0; k < kNElem; ++k) ms = std::fmax(ms, h->p.sigma[k]);
    int ok = 0;
    GridGeom g = make_grid(h->p.box, k_bind * ms, &ok);
    NlView nv;
    if (ok && bound_from_list(h, k_bind * ms, g, &nv)) {
        *list = nv.list;
        *start = nv.start;
    }
}

// bound_pairs_with_grid (src/analysis/pairs.rs:132-174) with the pairs left on
// the device in their owners' buckets (k_bound_buckets).  The staging lives
// in the caller's pool (*pool, made on first use), so that its addresses
// stay fixed for a captured observation.  Launches only; the caller zeroes
// bcnt.
int bound_buckets_device(gx_handle* h, void** pool, double k_bind, uint32_t* bucket, uint32_t* bcnt, uint32_t depth,
                         size_t stride) {
    uint32_t n = (uint32_t)h->n;
    if (!*pool) *pool = new AuxPool();
    AuxPool& P = *static_cast<AuxPool*>(*pool);
    int rc = ensure_pool(h, P, n, n);
    if (rc) return rc;
    double ms = 0.0;  // bind_cutoff, analysis/pairs.rs:112-114
    for (int k = 0; k < kNElem; ++k) ms = std::fmax(ms, h->p.sigma[k]);
    double cutoff = k_bind * ms;
    int ok = 0;
    GridGeom g = make_grid(h->p.box, cutoff, &ok);
    if (!ok) return set_err(h, GX_ERR_ARG, "invalid bond grid");
    BucketArgs v;
    v.k_bind = k_bind;
    for (int k = 0; k < kNElem; ++k) v.sig[k] = h->p.sigma[k];
    v.bucket = bucket;
    v.bcnt = bcnt;
    v.depth = depth;
    v.stride = stride;
    NlView nv;
    if (bound_from_list(h, cutoff, g, &nv)) {
        prof_begin(h, "bound_pairs");
        if (n)
            GX_LAUNCH(h, k_bound_from_list, nblk((size_t)n * kListBoundLanes, 256), 256, h->buf[h->cur], n, nv,
                      h->p.box[0], h->p.box[1], h->p.box[2], cutoff * cutoff, v);
        prof_end(h, "bound_pairs");
        return GX_OK;
    }
    if ((rc = ensure_cells(h, P.cl, g.ncell))) return rc;
    AuxSet a;
    a.x = P.xyz + 3 * P.cap;
    a.y = a.x + P.cap;
    a.z = a.y + P.cap;
    a.elem = P.elem + P.cap;
    a.slot = P.u32 + P.cap;
    a.key = P.u32 + 3 * P.cap;
    a.start = P.cl.start;
    a.m = n;
    uint32_t* key = P.u32 + 2 * P.cap;
    const StateBuf& b = h->buf[h->cur];
    prof_begin(h, "bond_grid");
    GX_CUDA(h, cudaMemsetAsync(P.cl.count, 0, ((size_t)g.ncell + 1) * sizeof(uint32_t), h->stream));
    GX_CUDA(h, cudaMemsetAsync(P.cl.fill, 0, (size_t)g.ncell * sizeof(uint32_t), h->stream));
    if (n) GX_LAUNCH(h, k_select_count, nblk(n, 256), 256, g, b, n, key, P.cl.count);
    cell_scan(h, P.cl, g.ncell);
    if (n) GX_LAUNCH(h, k_place, nblk(n, 256), 256, b, n, key, P.cl.start, P.cl.fill, a);
    prof_end(h, "bond_grid");
    prof_begin(h, "bound_pairs");
    if (n)
        GX_LAUNCH(h, k_bound_buckets, nblk((size_t)n * kBucketLanes, 256), 256, g, a, h->p.box[0], h->p.box[1],
                  h->p.box[2], cutoff * cutoff, v);
    prof_end(h, "bound_pairs");
    return GX_OK;
}

}  // namespace gx

extern "C" {

int gx_bound_pairs(gx_handle* h, double k_bind, uint32_t* pairs, size_t cap, size_t* npairs) {
    int rc = require(h);
    if (rc) return rc;
    if (cap && !pairs) return GX_ERR_ARG;
    uint32_t n = (uint32_t)h->n;
    AuxPool& P = pool_of(h);
    if ((rc = ensure_pool(h, P, n, n))) return rc;
    double ms = 0.0;  // bind_cutoff, analysis/pairs.rs:112-114
    for (int k = 0; k < kNElem; ++k) ms = std::fmax(ms, h->p.sigma[k]);
    double cutoff = k_bind * ms;
    int ok = 0;
    GridGeom g = make_grid(h->p.box, cutoff, &ok);
    if (!ok) return set_err(h, GX_ERR_ARG, "invalid bond grid");
    AuxSet a;
    if ((rc = build_aux(h, P, g, nullptr, n, a))) return rc;
    if (h->has_entity) GX_CUDA(h, cudaMemcpyAsync(P.entity, h->entity, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
    else GX_LAUNCH(h, k_iota, nblk(n, 256), 256, P.entity, n);
    uint32_t* dout = nullptr;
    if (cap) GX_CUDA(h, cudaMalloc(&dout, 2 * cap * sizeof(uint32_t)));
    GX_CUDA(h, cudaMemsetAsync(P.cnt, 0, sizeof(unsigned long long), h->stream));
    BoundVisit v;
    v.k_bind = k_bind;
    for (int k = 0; k < kNElem; ++k) v.sig[k] = h->p.sigma[k];
    v.entity = P.entity;
    v.out = dout;
    v.cap = cap;
    v.cnt = P.cnt;
    prof_begin(h, "bound_pairs");
    if (n) GX_LAUNCH(h, k_pairs, nblk(n, 128), 128, g, a, h->p.box[0], h->p.box[1], h->p.box[2], cutoff * cutoff, v);
    prof_end(h, "bound_pairs");
    unsigned long long total = 0;
    GX_CUDA(h, cudaMemcpyAsync(&total, P.cnt, sizeof total, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    size_t w = total < cap ? (size_t)total : cap;
    if (w) GX_CUDA(h, cudaMemcpy(pairs, dout, 2 * w * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    cudaFree(dout);
    if (npairs) *npairs = (size_t)total;
    GX_CUDA(h, cudaGetLastError());
    return total > cap ? set_err(h, GX_ERR_CAPACITY, "pair buffer too small") : GX_OK;
}

}  // extern "C"
