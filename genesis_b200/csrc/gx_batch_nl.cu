// gx_batch_nl.cu -- batch mode 4: the all-replica tick of mode 2 over
// persistent half neighbour lists (the single-universe list path, variant
// 6, applied to every replica at once).
//
// Every replica gets a list grid of cells >= r_c + skin; the grids share one
// global cell index (cell_base[r] + local cell).  At a rebuild all atoms are
// sorted by that index (slot s = sorted position, perm[s] = atom), each
// slot's atom keeps its home cell, and each slot gets the list of its pairs
// within r_c + skin (half list: the partner at a later slot of the same
// cell, or in a later cell of the replica).  Between rebuilds the state
// stays in its concatenated order and nothing is sorted:
//
//   k_bn_advance  kick (the replica's pending Berendsen scale), drift, wrap
//                 (the reference's exact FP64 steps, as k_fb_advance), then
//                 the slot's FP32 position in its home-cell frame of the
//                 last rebuild and the displacement test against it; zero
//                 forces
//   [rebuild]     only when some atom moved more than skin/2: list-grid
//                 keys, the shared counting sort, home frames, lists -- the
//                 body of a conditional graph node, so a tick without a
//                 rebuild launches none of it
//   k_bn_force    one lane per slot over its half list (nl_pair, the
//                 single-universe list pass's per-pair operations), far ends
//                 through 64-bit integer atomics, potential and pair count
//                 per replica on the tick that reports them
//   k_bn_finish   a = F 2^-32 / m and the second kick per slot (k_fb_finish's
//                 steps) with the kinetic energy summed per block
//   k_bn_thermo   per replica: the kinetic energy from its blocks' sums, in
//                 block order, and the Berendsen scale (k_fb_thermo's)
//
// The wrap of the reference (boundary.rs:28-34) translates each replica by
// half its box every tick; as in the single-universe path, a parity of those
// translations since the rebuild (one for all replicas: they tick together)
// is undone when the frame is staged.  Forces are order-independent integer
// sums of the same per-pair arithmetic as the single-universe list path, in
// the frame of the list grid, so they match mode 2 (whose frame is the force
// grid) to the last FP32 bits of the positions, within the same error bound.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gx_batch.cuh"
#include "gx_pair_f32.cuh"

namespace gx {

struct BnGeo {
    GridGeom g;          // the replica's list grid
    uint32_t cell_base;  // its first cell in the global index
};

struct BatchNl {
    size_t cap = 0;
    int nrep = 0;
    uint32_t ncell = 0;
    double skin = 0.0;
    int cap_nb = 0;
    BnGeo* geo = nullptr;
    float4* shift = nullptr;    // [nrep][27] periodic shift of neighbour-cell code k
    uint32_t* perm = nullptr;   // slot -> atom
    uint32_t* slot_of = nullptr;// atom -> slot
    uint32_t* home = nullptr;   // slot -> local home cell at the last rebuild
    uint32_t* srep = nullptr;   // slot -> replica
    float4* ref = nullptr;      // slot -> home-frame position at the last rebuild
    uint32_t* list = nullptr;   // entry e of slot s at list[e * cap + s], partner | code << 27
    uint32_t* cnt = nullptr;    // entries per slot (> cap_nb: overflowed, scans its cells)
    uint32_t* flag = nullptr;   // [0] rebuild requested, [1] rebuilds, [2] half-box parity, [3] body runs
    double* kpart = nullptr;    // per finishing block: kinetic energy of its (at most two) replicas
    uint64_t version = ~0ull;   // the batch's state version the lists follow
    gx_handle* ctx = nullptr;   // launch context: stream, counter, the list grid's counting sort
    cudaStream_t side = nullptr;
    cudaGraphExec_t graph[2] = {};
    uint64_t graph_kernels = 0, body_kernels = 0;
    uint32_t body_runs_seen = 0;
};

void batch_nl_free(BatchNl* s) {
    if (!s) return;
    for (cudaGraphExec_t g : s->graph)
        if (g) cudaGraphExecDestroy(g);
    cudaFree(s->geo);
    cudaFree(s->shift);
    cudaFree(s->perm);
    cudaFree(s->slot_of);
    cudaFree(s->home);
    cudaFree(s->srep);
    cudaFree(s->ref);
    cudaFree(s->list);
    cudaFree(s->cnt);
    cudaFree(s->flag);
    cudaFree(s->kpart);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->ctx) {
        cells_free(s->ctx->cl);
        s->ctx->stream = nullptr;  // owned by the batch
        delete s->ctx;
    }
    delete s;
}

namespace {

constexpr int kBnThreads = 128;  // slots per block of the pair pass; a replica holds at least this many
constexpr uint32_t kBnIdxMask = (1u << 27) - 1u;

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ __forceinline__ bool gated_off(const uint32_t* gate) { return gate && *gate == 0u; }

// Offset of a coordinate from its home cell's origin in the frame of the
// last rebuild (`shift`: the half-box translation to undo, 0 or L/2),
// unwrapped across the periodic boundary (the single-universe path's).
__device__ __forceinline__ double bn_home_local(double v, double L, double c, uint32_t i, double shift) {
    double u = xsub(rem_euclid(xadd(xadd(v, xmul(0.5, L)), shift), L), xmul((double)i, c));
    if (u > 0.5 * L) u = xsub(u, L);
    else if (u < -0.5 * L) u = xadd(u, L);
    return u;
}

__device__ __forceinline__ float4 bn_stage(const GridGeom& g, uint32_t home, double x, double y, double z, uint8_t kind,
                                           bool half) {
    uint32_t ix, iy, iz;
    decode(g, home, ix, iy, iz);
    return make_float4((float)bn_home_local(x, g.L[0], g.cell[0], ix, half ? xmul(0.5, g.L[0]) : 0.0),
                       (float)bn_home_local(y, g.L[1], g.cell[1], iy, half ? xmul(0.5, g.L[1]) : 0.0),
                       (float)bn_home_local(z, g.L[2], g.cell[2], iz, half ? xmul(0.5, g.L[2]) : 0.0),
                       __int_as_float((int)kind));
}

// Kick, drift, wrap (k_fb_advance's FP64 steps), the slot's home-frame
// position with this tick's wrap included in the parity, the displacement
// test, and the slot's force sums zeroed for the half-list pass.
__global__ void __launch_bounds__(256) k_bn_advance(const BnGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of,
                                                     BatchArrays A, const double* __restrict__ lam, double half_dt,
                                                     double dt, int wrap, const uint32_t* __restrict__ slot_of,
                                                     const uint32_t* __restrict__ home, const float4* __restrict__ ref,
                                                     float lim2, uint32_t* __restrict__ flag, uint32_t total,
                                                     uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool over = false;
    const bool half = ((flag[2] + (wrap ? 1u : 0u)) & 1u) != 0u;
    if (i < total) {
        const uint32_t r = rep_of[i];
        const double l = lam[r];
        double vx = xadd(xmul(A.vx[i], l), xmul(A.ax[i], half_dt));
        double vy = xadd(xmul(A.vy[i], l), xmul(A.ay[i], half_dt));
        double vz = xadd(xmul(A.vz[i], l), xmul(A.az[i], half_dt));
        double x = xadd(A.x[i], xmul(vx, dt)), y = xadd(A.y[i], xmul(vy, dt)), z = xadd(A.z[i], xmul(vz, dt));
        const GridGeom& g = geo[r].g;
        if (wrap) {  // half the box: exact, the same value as the replica's half_box
            const double hx = xmul(0.5, g.L[0]), hy = xmul(0.5, g.L[1]), hz = xmul(0.5, g.L[2]);
            x = xsub(rem_euclid(x, xmul(2.0, hx)), hx);
            y = xsub(rem_euclid(y, xmul(2.0, hy)), hy);
            z = xsub(rem_euclid(z, xmul(2.0, hz)), hz);
        }
        A.vx[i] = vx;
        A.vy[i] = vy;
        A.vz[i] = vz;
        A.x[i] = x;
        A.y[i] = y;
        A.z[i] = z;
        const uint32_t s = slot_of[i];
        const size_t fs = A.total;
        A.F[s] = 0;
        A.F[fs + s] = 0;
        A.F[2 * fs + s] = 0;
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            atomicOr(err, kErrNonFinite);
            over = true;
        } else {
            const float4 p = bn_stage(g, home[s], x, y, z, A.kind[i], half);
            A.pos4[s] = p;
            const float4 q = ref[s];
            const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
            over = !(dx * dx + dy * dy + dz * dz <= lim2);
        }
    }
    if (__any_sync(0xffffffffu, over) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// The rebuild body's condition: the flag k_bn_advance raised.
__global__ void k_bn_set_cond(cudaGraphConditionalHandle hc, const uint32_t* __restrict__ flag) {
    cudaGraphSetConditional(hc, flag[0] != 0u ? 1u : 0u);
}

__global__ void k_bn_keys(const BnGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of, BatchArrays A,
                          uint32_t total, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const BnGeo& G = geo[rep_of[i]];
    A.key[i] = G.cell_base + cell_of(G.g, A.x[i], A.y[i], A.z[i]);
}

// Slots after the sort: each slot's atom, home cell, replica and home-frame
// position (the reference frame of the displacement test).
__global__ void k_bn_stage(const BnGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of, BatchArrays A,
                           const uint32_t* __restrict__ perm, uint32_t* __restrict__ slot_of,
                           uint32_t* __restrict__ home, uint32_t* __restrict__ srep, float4* __restrict__ ref,
                           uint32_t total, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
    const uint32_t i = perm[s], r = rep_of[i];
    const BnGeo& G = geo[r];
    const uint32_t c = A.key[i] - G.cell_base;
    slot_of[i] = s;
    home[s] = c;
    srep[s] = r;
    const float4 p = bn_stage(G.g, c, A.x[i], A.y[i], A.z[i], A.kind[i], false);
    A.pos4[s] = p;
    ref[s] = p;
}

__device__ __forceinline__ uint32_t bn_cell_at(const GridGeom& g, uint32_t cx, uint32_t cy, uint32_t cz, uint32_t code) {
    const int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
    return encode(g, wrap_add(cx, ox, g.n[0]), wrap_add(cy, oy, g.n[1]), wrap_add(cz, oz, g.n[2]));
}

// Half lists of the pairs within r_l (r_l^2 = rl2) over the 27 home-grid
// cells of the slot's replica, each pair once: a later slot of the same cell
// or any slot of a later cell (slots are sorted by cell, so those are the
// later slots).  A cell whose nearest point is out of reach is skipped whole
// (k_nl_build's test and slack).
__global__ void __launch_bounds__(kBnThreads) k_bn_build(const BnGeo* __restrict__ geo,
                                                          const uint32_t* __restrict__ srep,
                                                          const uint32_t* __restrict__ home,
                                                          const float4* __restrict__ pos4,
                                                          const uint32_t* __restrict__ start, uint32_t total, float rl2,
                                                          uint32_t* __restrict__ list, size_t stride, int cap_nb,
                                                          uint32_t* __restrict__ cnt, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    const uint32_t s = blockIdx.x * kBnThreads + threadIdx.x;
    if (s >= total) return;
    const BnGeo& G = geo[srep[s]];
    const GridGeom& g = G.g;
    const uint32_t base = G.cell_base;
    const float4 pi = pos4[s];
    const uint32_t c = home[s];
    uint32_t cx, cy, cz;
    decode(g, c, cx, cy, cz);
    const float slack = 1e-3f;
    uint32_t m = 0;
    for (uint32_t code = 0; code < 27; ++code) {
        const int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
        const uint32_t B = bn_cell_at(g, cx, cy, cz, code);
        if (B < c) continue;
        const float mx = fmaxf((ox > 0 ? g.cellf[0] - pi.x : (ox < 0 ? pi.x : 0.f)) - slack, 0.f);
        const float my = fmaxf((oy > 0 ? g.cellf[1] - pi.y : (oy < 0 ? pi.y : 0.f)) - slack, 0.f);
        const float mz = fmaxf((oz > 0 ? g.cellf[2] - pi.z : (oz < 0 ? pi.z : 0.f)) - slack, 0.f);
        if (dist2(mx, my, mz) >= rl2) continue;
        const float qx = fadd(pi.x, -(float)ox * g.cellf[0]), qy = fadd(pi.y, -(float)oy * g.cellf[1]),
                    qz = fadd(pi.z, -(float)oz * g.cellf[2]);
        uint32_t lo = start[base + B];
        const uint32_t hi = start[base + B + 1];
        if (B == c) lo = s + 1;
#pragma unroll 4
        for (uint32_t q = lo; q < hi; ++q) {
            const float4 pj = pos4[q];
            if (dist2(fsub(qx, pj.x), fsub(qy, pj.y), fsub(qz, pj.z)) < rl2) {
                if (m < (uint32_t)cap_nb) list[(size_t)m * stride + s] = q | (code << 27);
                ++m;
            }
        }
    }
    cnt[s] = m;
}

// Periodic shift of neighbour-cell code k of every replica's list grid.
__global__ void k_bn_shifts(const BnGeo* __restrict__ geo, int nrep, float4* __restrict__ shift) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 27 * nrep) return;
    const GridGeom& g = geo[t / 27].g;
    const int code = t % 27;
    const int ox = code % 3 - 1, oy = (code / 3) % 3 - 1, oz = code / 9 - 1;
    shift[t] = make_float4(-(float)ox * g.cellf[0], -(float)oy * g.cellf[1], -(float)oz * g.cellf[2], 0.f);
}

// The pair pass: one lane per slot over its half list, the far end's force
// through 64-bit integer atomics (k_nl_force's loop and nl_pair).  A block
// of kBnThreads slots spans at most two replicas (each holds at least that
// many atoms), whose shift tables it keeps in shared memory.  An overflowed
// list scans the slot's 27 home-grid cells directly.  With ENERGY the
// replicas' potentials and pair counts go to racc (mode 2's warp sums).
template <bool ENERGY>
__global__ void __launch_bounds__(kBnThreads) k_bn_force(const BnGeo* __restrict__ geo,
                                                          const float4* __restrict__ shift_tab,
                                                          const float4* __restrict__ pos4,
                                                          const uint32_t* __restrict__ home,
                                                          const uint32_t* __restrict__ srep,
                                                          const uint32_t* __restrict__ start, uint32_t total, LawF32 L,
                                                          const PairF* __restrict__ tab,
                                                          const uint32_t* __restrict__ list, size_t stride,
                                                          int cap_nb, const uint32_t* __restrict__ cnt,
                                                          long long* __restrict__ F, size_t fstride,
                                                          unsigned long long* __restrict__ racc,
                                                          uint32_t* __restrict__ err) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ float4 s_shift[2][27];
    const int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kBnThreads) st[t] = tab[t];
    const uint32_t first = blockIdx.x * kBnThreads;
    const uint32_t last = min(first + (uint32_t)kBnThreads, total) - 1u;
    const uint32_t r0 = srep[first], r1 = srep[last];
    if (threadIdx.x < 54) {
        const uint32_t w = threadIdx.x / 27, k = threadIdx.x % 27;
        s_shift[w][k] = shift_tab[(size_t)(w ? r1 : r0) * 27 + k];
    }
    __syncthreads();
    const uint32_t s = first + threadIdx.x;
    PairAcc a;
    uint32_t r = 0xFFFFFFFFu;
    if (s < total) {
        r = srep[s];
        const float4* sh_tab = s_shift[r == r0 ? 0 : 1];
        const float4 pi = pos4[s];
        const int ki = __float_as_int(pi.w);
        const uint32_t m = cnt[s];
        if (m <= (uint32_t)cap_nb) {
            const uint32_t* lp = list + s;
            uint32_t e = 0;
            for (; e + 4 <= m; e += 4) {  // four entries per round, every load before any pair math
                uint32_t w[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] = __ldg(lp + (size_t)(e + k) * stride);
                float4 pj[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) pj[k] = __ldg(pos4 + (w[k] & kBnIdxMask));
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float4 sh = sh_tab[w[k] >> 27];
                    const uint32_t q = w[k] & kBnIdxMask;
                    nl_pair(L, st, ki, pi, pj[k], sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);  // half list: q > s
                }
            }
            for (; e < m; ++e) {
                const uint32_t w = __ldg(lp + (size_t)e * stride);
                const float4 sh = sh_tab[w >> 27];
                const uint32_t q = w & kBnIdxMask;
                nl_pair(L, st, ki, pi, __ldg(pos4 + q), sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);  // half list: q > s
            }
        } else {  // overflowed list: the later slots of the home-grid cells
            const BnGeo& G = geo[r];
            const uint32_t c = home[s];
            uint32_t cx, cy, cz;
            decode(G.g, c, cx, cy, cz);
            for (uint32_t code = 0; code < 27; ++code) {
                const uint32_t B = bn_cell_at(G.g, cx, cy, cz, code);
                if (B < c) continue;
                const float4 sh = sh_tab[code];
                for (uint32_t q = start[G.cell_base + B], hi = start[G.cell_base + B + 1]; q < hi; ++q)
                    if (q > s) nl_pair(L, st, ki, pi, pos4[q], sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);
            }
        }
        atomicAdd((unsigned long long*)&F[s], (unsigned long long)a.fx);
        atomicAdd((unsigned long long*)&F[fstride + s], (unsigned long long)a.fy);
        atomicAdd((unsigned long long*)&F[2 * fstride + s], (unsigned long long)a.fz);
    }
    if (!ENERGY) return;
    // per-replica potential and pair count: one atomic per warp when the warp
    // lies in one replica, else one per lane
    const uint32_t rw = __shfl_sync(0xffffffffu, r, 0);
    if (__all_sync(0xffffffffu, r == rw) && rw != 0xFFFFFFFFu) {
        unsigned long long x = (unsigned long long)a.vq, y = a.np;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_down_sync(0xffffffffu, x, o);
            y += __shfl_down_sync(0xffffffffu, y, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&racc[2 * rw], x);
            atomicAdd(&racc[2 * rw + 1], y);
        }
    } else if (r != 0xFFFFFFFFu) {
        atomicAdd(&racc[2 * r], (unsigned long long)a.vq);
        atomicAdd(&racc[2 * r + 1], (unsigned long long)a.np);
    }
}

// a = F 2^-32 / m and the second kick (k_fb_finish's FP64 steps) per slot,
// with the new kinetic energy summed per block in a fixed order.  A
// replica's atoms hold exactly the slots [base, base + n) (the slots are
// sorted by a global cell index grouped by replica), and every replica holds
// at least kBnThreads >= kBnRed atoms, so a block of kBnRed slots holds at
// most two replicas: kpart[2b] is the sum over the block's first replica,
// kpart[2b + 1] over its second.
constexpr int kBnRed = 128;
static_assert(kBnRed <= kBnThreads, "two replicas per reduction block at most");

__global__ void __launch_bounds__(kBnRed) k_bn_finish(BatchArrays A, const uint32_t* __restrict__ perm,
                                                       const uint32_t* __restrict__ srep, uint32_t total,
                                                       double half_dt, double* __restrict__ kpart) {
    __shared__ double sh[2][kBnRed / 32];
    const uint32_t first = blockIdx.x * kBnRed, s = first + threadIdx.x;
    const uint32_t r0 = srep[first];
    double k0 = 0.0, k1 = 0.0;
    if (s < total) {
        const size_t fs = A.total;
        const uint32_t i = perm[s];
        const double im = A.inv_mass[i];
        const double ax = xmul(xmul(__ll2double_rn(A.F[s]), kFixInv), im);
        const double ay = xmul(xmul(__ll2double_rn(A.F[fs + s]), kFixInv), im);
        const double az = xmul(xmul(__ll2double_rn(A.F[2 * fs + s]), kFixInv), im);
        A.ax[i] = ax;
        A.ay[i] = ay;
        A.az[i] = az;
        const double vx = xadd(A.vx[i], xmul(ax, half_dt));
        const double vy = xadd(A.vy[i], xmul(ay, half_dt));
        const double vz = xadd(A.vz[i], xmul(az, half_dt));
        A.vx[i] = vx;
        A.vy[i] = vy;
        A.vz[i] = vz;
        const double ke = xmul(xmul(0.5, A.mass[i]), xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz)));
        if (srep[s] == r0) k0 = ke;
        else k1 = ke;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        k0 = xadd(k0, __shfl_down_sync(0xffffffffu, k0, o));
        k1 = xadd(k1, __shfl_down_sync(0xffffffffu, k1, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][w] = k0;
        sh[1][w] = k1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < kBnRed / 32; ++k) {
            t0 = xadd(t0, sh[0][k]);
            t1 = xadd(t1, sh[1][k]);
        }
        kpart[2 * blockIdx.x] = t0;
        kpart[2 * blockIdx.x + 1] = t1;
    }
}

// One warp per replica: its kinetic energy from the partials of the blocks
// over its slots, in block order, and the Berendsen scale of
// ThermostatSystem::run (thermostat.rs:52-71) as fb_thermo_one computes it;
// the potential and pair count of the reporting tick to `out`.
__global__ void k_bn_thermo(const RepThermo* __restrict__ th, const uint32_t* __restrict__ srep,
                            const double* __restrict__ kpart, double* __restrict__ lam,
                            unsigned long long* __restrict__ racc, double k_thermal, double* __restrict__ out) {
    const int r = blockIdx.x;
    const RepThermo T = th[r];
    if (threadIdx.x != 0) return;
    double ks = 0.0;
    if (T.n) {
        const uint32_t b0 = T.base / kBnRed, b1 = (T.base + T.n - 1) / kBnRed;
        for (uint32_t b = b0; b <= b1; ++b) ks = xadd(ks, kpart[2 * b + (srep[b * kBnRed] == (uint32_t)r ? 0 : 1)]);
    }
    double l = 1.0;
    if (T.thermo && T.n > 0) {
        const double t = xdiv(xmul(2.0 / 3.0, xdiv(ks, (double)T.n)), k_thermal);
        if (isfinite(t) && t > 0.0) {
            const double l2 = xadd(1.0, xmul(xdiv(1.0, T.tau), xsub(xdiv(T.target, t), 1.0)));
            l = xsqrt(fmax(l2, 0.0));
        }
    }
    lam[r] = l;
    out[4 * r + 1] = xmul(__ll2double_rn((long long)racc[2 * r]), kFixInv);
    out[4 * r + 2] = l;
    out[4 * r + 3] = (double)racc[2 * r + 1];
    racc[2 * r] = 0;
    racc[2 * r + 1] = 0;
}

__global__ void k_bn_body_done(uint32_t* flag) { flag[3] += 1u; }

// After the (conditional) rebuild: count it and restart the parity, or
// toggle the parity with this tick's wrap.
__global__ void k_bn_end(uint32_t* flag, int wrap) {
    if (flag[0]) {
        flag[1] += 1u;
        flag[0] = 0u;
        flag[2] = 0u;
    } else if (wrap) {
        flag[2] ^= 1u;
    }
}

__global__ void k_bn_stats(const uint32_t* __restrict__ cnt, uint32_t n, int cap_nb, unsigned long long* __restrict__ out) {
    unsigned long long e = 0, o = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t m = cnt[i];
        e += m;
        o += m > (uint32_t)cap_nb ? 1ull : 0ull;
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        e += __shfl_down_sync(0xffffffffu, e, k);
        o += __shfl_down_sync(0xffffffffu, o, k);
    }
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicAdd(out, e);
        if (o) atomicAdd(out + 1, o);
    }
}

__global__ void k_bn_init_slots(uint32_t* __restrict__ slot_of, uint32_t* __restrict__ perm, uint32_t total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total) slot_of[i] = perm[i] = i;
}

int bnerr(gx_batch* b, int code, const std::string& m) {
    b->err = m;
    return code;
}
#define GXN_CUDA(b, call)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return bnerr(b, GX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// The default skin is larger than the single universe's 0.1 r_c: the first
// atom of any replica to move skin/2 rebuilds every replica's lists, so the
// rebuilds come more often (256 sweep replicas: every 4 ticks at 0.1 r_c,
// every 6 at 0.15 r_c, 0.58 against 0.56 ms per tick).
double skin_of(const gx_batch* b) { return b->nl_skin >= 0.0 ? b->nl_skin : 0.15 * b->rc; }

// Allocates the lists (outside any capture) for the batch's current atoms.
int bn_prepare(gx_batch* b) {
    const double skin = skin_of(b);
    BatchNl* s = b->nl;
    if (s && s->cap == b->total && s->nrep == b->nrep && s->skin == skin) return GX_OK;
    batch_nl_free(s);
    s = b->nl = new BatchNl();
    s->cap = b->total;
    s->nrep = b->nrep;
    s->skin = skin;
    const double rl = b->rc + skin;
    std::vector<BnGeo> geo(b->nrep);
    uint32_t cells = 0;
    double rho = 0.0;
    for (int r = 0; r < b->nrep; ++r) {
        const RepDesc& d = b->reps[r];
        int ok = 0;
        geo[r].g = make_grid(d.g.L, rl, &ok);
        if (!ok) return bnerr(b, GX_ERR_ARG, "a replica's neighbour-list grid is empty or too large");
        geo[r].cell_base = cells;
        if ((uint64_t)cells + geo[r].g.ncell > 0xFFFFFFF0ull) return bnerr(b, GX_ERR_CAPACITY, "too many list cells");
        cells += geo[r].g.ncell;
        rho = std::max(rho, (double)d.n / (d.g.L[0] * d.g.L[1] * d.g.L[2]));
    }
    s->ncell = cells;
    const double expect = rho * (4.0 / 3.0) * 3.14159265358979 * rl * rl * rl;
    int cap_nb = (int)std::ceil(2.0 * expect) + 32;
    cap_nb = std::min((cap_nb + 7) & ~7, 1024);
    s->cap_nb = cap_nb;
    const size_t n = b->total;
    GXN_CUDA(b, cudaMalloc(&s->geo, b->nrep * sizeof(BnGeo)));
    GXN_CUDA(b, cudaMalloc(&s->shift, (size_t)b->nrep * 27 * sizeof(float4)));
    GXN_CUDA(b, cudaMalloc(&s->perm, n * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->slot_of, n * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->home, n * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->srep, n * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->ref, n * sizeof(float4)));
    GXN_CUDA(b, cudaMalloc(&s->list, (size_t)cap_nb * n * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->cnt, n * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->flag, 4 * sizeof(uint32_t)));
    GXN_CUDA(b, cudaMalloc(&s->kpart, 2 * (size_t)nblk(n, kBnRed) * sizeof(double)));
    GXN_CUDA(b, cudaMemcpy(s->geo, geo.data(), b->nrep * sizeof(BnGeo), cudaMemcpyHostToDevice));
    GXN_CUDA(b, cudaMemsetAsync(s->home, 0, n * sizeof(uint32_t), b->stream));
    GXN_CUDA(b, cudaMemsetAsync(s->srep, 0, n * sizeof(uint32_t), b->stream));
    GXN_CUDA(b, cudaMemsetAsync(s->ref, 0, n * sizeof(float4), b->stream));
    GXN_CUDA(b, cudaMemsetAsync(s->cnt, 0, n * sizeof(uint32_t), b->stream));
    GXN_CUDA(b, cudaMemsetAsync(s->flag, 0, 4 * sizeof(uint32_t), b->stream));
    // before the first rebuild every atom writes its own slot
    k_bn_init_slots<<<nblk(n, 256), 256, 0, b->stream>>>(s->slot_of, s->perm, (uint32_t)n);
    k_bn_shifts<<<nblk(27 * (size_t)b->nrep, 256), 256, 0, b->stream>>>(s->geo, b->nrep, s->shift);
    GXN_CUDA(b, cudaGetLastError());
    GXN_CUDA(b, cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    s->ctx = new gx_handle();
    s->ctx->stream = b->stream;
    if (ensure_cells(s->ctx, s->ctx->cl, s->ncell)) return bnerr(b, GX_ERR_OOM, s->ctx->err);
    if (ensure_sort_tmp(s->ctx, s->ctx->cl, n)) return bnerr(b, GX_ERR_OOM, s->ctx->err);  // before capture
    return GX_OK;
}

// One tick of every replica (launches only: captured).  The rebuild goes
// into the body of a conditional (IF) node, captured from a second stream.
int bn_tick(gx_batch* b, const FlatShared& fsh, bool energy) {
    BatchNl* s = b->nl;
    gx_handle* h = s->ctx;
    const uint32_t n = (uint32_t)b->total;
    const BatchArrays A = b->A;
    const int wrap = b->p.enable_boundaries ? 1 : 0;
    const float lim = (float)(0.5 * s->skin * (1.0 - 1e-4));
    GX_LAUNCH(h, k_bn_advance, nblk(n, 256), 256, s->geo, fsh.rep_of, A, fsh.lam, 0.5 * b->p.dt, b->p.dt, wrap,
              s->slot_of, s->home, s->ref, lim * lim, s->flag, n, b->d_err);
    cudaStreamCaptureStatus st;
    unsigned long long id = 0;
    cudaGraph_t gr = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    GXN_CUDA(b, cudaStreamGetCaptureInfo(h->stream, &st, &id, &gr, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) return bnerr(b, GX_ERR_STATE, "the mode-4 tick is built only by capture");
    cudaGraphConditionalHandle hc;
    GXN_CUDA(b, cudaGraphConditionalHandleCreate(&hc, gr, 0, cudaGraphCondAssignDefault));
    GX_LAUNCH(h, k_bn_set_cond, 1, 1, hc, s->flag);
    GXN_CUDA(b, cudaStreamGetCaptureInfo(h->stream, &st, &id, &gr, &deps, &nd));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    GXN_CUDA(b, cudaGraphAddNode(&node, gr, deps, nd, &cp));
    GXN_CUDA(b, cudaStreamUpdateCaptureDependencies(h->stream, &node, 1, cudaStreamSetCaptureDependencies));
    GXN_CUDA(b, cudaStreamBeginCaptureToGraph(s->side, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed));
    cudaStream_t main_stream = h->stream;
    h->stream = s->side;
    const uint64_t l0 = h->launches;
    const float rl = (float)((b->rc + s->skin) * (1.0 + 1e-6));
    GX_LAUNCH(h, k_bn_keys, nblk(n, 256), 256, s->geo, fsh.rep_of, A, n, s->flag);
    int rc = counting_sort(h, h->cl, s->ncell, A.key, n, s->perm, s->flag);
    if (!rc) {
        GX_LAUNCH(h, k_bn_stage, nblk(n, 256), 256, s->geo, fsh.rep_of, A, s->perm, s->slot_of, s->home, s->srep,
                  s->ref, n, s->flag);
        GX_LAUNCH(h, k_bn_build, nblk(n, kBnThreads), kBnThreads, s->geo, s->srep, s->home, A.pos4, h->cl.start, n,
                  rl * rl, s->list, s->cap, s->cap_nb, s->cnt, s->flag);
        GX_LAUNCH(h, k_bn_body_done, 1, 1, s->flag);
    }
    s->body_kernels = h->launches - l0;
    h->launches = l0;  // counted when a body runs
    cudaGraph_t body = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s->side, &body);
    h->stream = main_stream;
    if (rc) return bnerr(b, rc, h->err);
    if (ce != cudaSuccess) return bnerr(b, GX_ERR_CUDA, std::string("rebuild body: ") + cudaGetErrorString(ce));
    GX_LAUNCH(h, k_bn_end, 1, 1, s->flag, wrap);
    auto kf = energy ? k_bn_force<true> : k_bn_force<false>;
    GX_LAUNCH(h, kf, nblk(n, kBnThreads), kBnThreads, s->geo, s->shift, A.pos4, s->home, s->srep, h->cl.start, n, b->L,
              b->d_tab, s->list, s->cap, s->cap_nb, s->cnt, A.F, A.total, fsh.acc, b->d_err);
    GX_LAUNCH(h, k_bn_finish, nblk(n, kBnRed), kBnRed, A, s->perm, s->srep, n, 0.5 * b->p.dt, s->kpart);
    GX_LAUNCH(h, k_bn_thermo, b->nrep, 32, fsh.th, s->srep, s->kpart, fsh.lam, fsh.acc, b->p.thermal_constant,
              b->d_out);
    return GX_OK;
}

}  // namespace

bool batch_nl_eligible(const gx_batch* b) {
    if (!b->has_state || !b->total) return false;
    const double rl = b->rc + skin_of(b);
    for (const RepDesc& d : b->reps) {
        if (d.n < (uint32_t)kBnThreads) return false;
        int ok = 0;
        const GridGeom g = make_grid(d.g.L, rl, &ok);
        if (!ok || g.n[0] < 3 || g.n[1] < 3 || g.n[2] < 3) return false;
    }
    return true;
}

// Mode 4: nsteps ticks of every replica, each a replay of one captured tick;
// the lists are rebuilt on the first tick after any change of the state that
// they did not follow (a new state, another mode's ticks, a restored
// snapshot) and whenever an atom has moved more than skin/2.
int batch_nl_step(gx_batch* b, int nsteps, uint64_t* launches) {
    if (launches) *launches = 0;
    if (!b->total || nsteps <= 0) return GX_OK;
    if (!batch_nl_eligible(b))
        return bnerr(b, GX_ERR_UNSUPPORTED,
                     "batch mode 4 needs every replica to hold >= 128 atoms and >= 3 list-grid cells per axis");
    FlatShared fsh;
    int rc = flat_shared(b, &fsh);
    if (rc) return rc;
    if ((rc = bn_prepare(b))) return rc;
    BatchNl* s = b->nl;
    gx_handle* h = s->ctx;
    if (s->version != b->version) {
        const uint32_t one = 1u;
        GXN_CUDA(b, cudaMemcpyAsync(s->flag, &one, sizeof one, cudaMemcpyHostToDevice, b->stream));
        s->version = b->version;
    }
    for (int e = 0; e < 2; ++e) {
        if (s->graph[e]) continue;
        cudaGraph_t g = nullptr;
        GXN_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const uint64_t c0 = h->launches;
        int trc = bn_tick(b, fsh, e == 1);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (trc || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return trc ? trc : bnerr(b, GX_ERR_CUDA, cudaGetErrorString(ce));
        }
        ce = cudaGraphInstantiate(&s->graph[e], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return bnerr(b, GX_ERR_CUDA, cudaGetErrorString(ce));
        s->graph_kernels = h->launches - c0;
        h->launches = c0;
    }
    const uint64_t l0 = h->launches;
    for (int t = 0; t < nsteps; ++t) {
        GXN_CUDA(b, cudaGraphLaunch(s->graph[t == nsteps - 1], b->stream));
        h->launches += s->graph_kernels;
    }
    flat_commit(b, h);
    GXN_CUDA(b, cudaGetLastError());
    if (launches) *launches = h->launches - l0;
    return GX_OK;
}

// Entries of mode 4's current lists (an overflowed slot counts the entries
// it found) and the slots whose list overflowed (synchronises).
int batch_nl_stats(gx_batch* b, uint64_t* entries, uint64_t* overflowed) {
    *entries = *overflowed = 0;
    BatchNl* s = b->nl;
    if (!s || !s->cnt || !b->total) return GX_OK;
    unsigned long long* d = nullptr;
    GXN_CUDA(b, cudaMalloc(&d, 2 * sizeof(unsigned long long)));
    unsigned long long v[2] = {0, 0};
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof v, b->stream);
    if (e == cudaSuccess) {
        k_bn_stats<<<256, 256, 0, b->stream>>>(s->cnt, (uint32_t)b->total, s->cap_nb, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(v, d, sizeof v, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(d);
    if (e != cudaSuccess) return bnerr(b, GX_ERR_CUDA, cudaGetErrorString(e));
    *entries = v[0];
    *overflowed = v[1];
    return GX_OK;
}

// Rebuilds done by mode 4 so far (synchronises).
int batch_nl_rebuilds(gx_batch* b, uint64_t* out) {
    *out = 0;
    if (!b->nl || !b->nl->flag) return GX_OK;
    uint32_t f[4] = {0, 0, 0, 0};
    GXN_CUDA(b, cudaMemcpyAsync(f, b->nl->flag, sizeof f, cudaMemcpyDeviceToHost, b->stream));
    GXN_CUDA(b, cudaStreamSynchronize(b->stream));
    *out = f[1];
    return GX_OK;
}

}  // namespace gx
