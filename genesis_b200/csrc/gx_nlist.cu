// gx_nlist.cu -- the mixed pair pass over a persistent neighbour list
// (kernel variants 5 and 6).
//
// The reference rebuilds its cell list and pair list every tick
// (ForceSystem::run, src/systems/forces.rs:228-232).  The pair SET it
// evaluates is {pairs with d < r_c} at this tick, and the mixed path's sums
// are order-independent integers, so any enumeration that yields exactly
// that set gives the same forces.  Here a list of all pairs within
// r_c + skin is built on a grid whose cells are at least r_c + skin wide and
// reused while no atom has moved more than skin/2 since the build: then every
// pair now within r_c was within r_c + skin at the build.  Between rebuilds
// the atoms keep their sorted positions and their home cell, so the FP32
// cell-local frame (offsets from the home cell's origin, |offset| below a
// cell plus skin/2) keeps the same precision as the per-tick frame.
//
// The reference's wrap, x <- rem_euclid(x, 2h) - h (boundary.rs:28-34,
// reproduced bit for bit), translates the whole periodic system by h = L/2
// on every tick.  The list frame therefore co-moves: a device parity counts
// those half-box translations since the last rebuild and the staging adds
// them back, so only physical motion enters the displacement test (a wrong
// parity reads as an L/2 jump, which forces a rebuild).
//
// One tick (all launches captured in one CUDA graph; the rebuild launches
// read a device flag and do nothing when it is clear):
//   k_nl_advance   kick (with the pending Berendsen scale), drift, wrap,
//                  home-frame FP32 staging, displacement check -> flag;
//                  zeroes the force sums of the half-list pass
//   [rebuild]      cell keys, counting sort, gather, copy back, staging,
//                  list build
//   k_nl_end       rebuild count, frame parity, zeroed energy counters
//   k_nl_force     one thread per atom over its full list: FP32 pair law,
//                  fixed-point sums in registers, plain stores (no atomics);
//                  the potential and pair count take each pair once (q > p)
//   k_nl_finish    a = F 2^-32 / m, second kick, kinetic-energy partials
// An atom whose list overflowed scans its 27 home-grid cells directly, so
// the pair set stays exact whatever the local density.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "gx_law64.cuh"
#include "gx_pair_f32.cuh"

namespace gx {

struct NlState {
    GridGeom lg{};            // list grid: cells >= r_c + skin
    double skin = -1.0;       // < 0: default (0.1 r_c)
    double skin_used = 0.0;
    int half = -1;            // list kind built: 0 full, 1 half (variant 6)
    int tpp = 1;              // threads per atom in the list pass (1, 2, 4, 8)
    int slots = 16;           // variant 7: stash slots per thread (8 or 16)
    int brick = 1;            // variant 8: 0 = bricks of 4 cells (1024 staged atoms), 1 = 8 cells (2048)
    int block = 0;            // variant 6, one lane per atom: 0 = far ends always global, 128 or 256 = far
                              // ends inside a block of that many atoms summed in shared memory
    int cap_nb = 0;           // list entries per atom
    size_t cap = 0;           // atoms the buffers hold
    uint32_t* list = nullptr; // entry e of atom p at list[e * cap + p]
    uint32_t* cnt = nullptr;  // entries per atom (> cap_nb: overflowed)
    float4* ref = nullptr;    // home-frame positions at the last rebuild
    uint32_t* flag = nullptr; // [0] rebuild requested, [1] rebuilds done, [2] half-box translations since (mod 2),
                              // [3] runs of a captured rebuild body
    CellList cl;
    // A captured tick puts the rebuild in the body of a conditional (IF)
    // graph node, set from flag[0], so that a tick without a rebuild does
    // not launch it at all.  The body is captured from a second stream.
    cudaStream_t side = nullptr;
    uint64_t body_kernels = 0;  // kernels in the body (counted when it runs)
    uint32_t body_runs_seen = 0;
};

namespace {

constexpr int kNlThreads = 128;
constexpr int kNlBuildThreads = 128;
constexpr int kNlBuildUnroll = 4;
constexpr int kRedThreads = 256;
constexpr uint32_t kIdxMask = (1u << 27) - 1u;

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ __forceinline__ bool gated_off(const uint32_t* gate) { return gate && *gate == 0u; }

// Offset of a coordinate from its home cell's origin in the frame of the
// last rebuild (`shift` = the translation to undo, 0 or L/2), unwrapped
// across the periodic boundary (the atom may have left its home cell).
__device__ __forceinline__ double home_local(double v, double L, double c, uint32_t i, double shift) {
    double u = xsub(rem_euclid(xadd(xadd(v, xmul(0.5, L)), shift), L), xmul((double)i, c));
    if (u > 0.5 * L) u = xsub(u, L);
    else if (u < -0.5 * L) u = xadd(u, L);
    return u;
}

__device__ __forceinline__ float4 stage_one(const GridGeom& g, const StateBuf& b, uint32_t home, uint32_t i,
                                            double x, double y, double z, bool half) {
    uint32_t ix, iy, iz;
    decode(g, home, ix, iy, iz);
    return make_float4((float)home_local(x, g.L[0], g.cell[0], ix, half ? xmul(0.5, g.L[0]) : 0.0),
                       (float)home_local(y, g.L[1], g.cell[1], iy, half ? xmul(0.5, g.L[1]) : 0.0),
                       (float)home_local(z, g.L[2], g.cell[2], iz, half ? xmul(0.5, g.L[2]) : 0.0),
                       __int_as_float((int)b.kind[i]));
}

// Neighbour-cell code: (ox+1) + 3(oy+1) + 9(oz+1); 13 is the home cell.
__device__ __forceinline__ void code_shift(const GridGeom& g, uint32_t code, float& sx, float& sy, float& sz) {
    int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
    sx = -(float)ox * g.cellf[0];
    sy = -(float)oy * g.cellf[1];
    sz = -(float)oz * g.cellf[2];
}

__device__ __forceinline__ uint32_t cell_at(const GridGeom& g, uint32_t cx, uint32_t cy, uint32_t cz, uint32_t code) {
    int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
    return encode(g, wrap_add(cx, ox, g.n[0]), wrap_add(cy, oy, g.n[1]), wrap_add(cz, oz, g.n[2]));
}

// Kick (integrate.rs:38-45, with the pending scale of thermostat.rs:68-70),
// drift (integrate.rs:62-66), wrap (boundary.rs:28-34) with the same exact
// FP64 operations as k_kick/k_drift/k_wrap; then the home-frame staging and
// the displacement test against the last rebuild.
__global__ void __launch_bounds__(256) k_nl_advance(StateBuf b, uint32_t n, const double* __restrict__ lambda,
                                                     double half_dt, double dt, double hx, double hy, double hz,
                                                     int wrap, GridGeom g, const uint32_t* __restrict__ home,
                                                     float4* __restrict__ pos4, const float4* __restrict__ ref,
                                                     float lim2, uint32_t* __restrict__ flag,
                                                     uint32_t* __restrict__ err, long long* __restrict__ F,
                                                     size_t fstride) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool over = false;
    if (F && i < n) {  // the half-list pass accumulates into F: zero it here, not in a separate memset
        F[i] = 0;
        F[fstride + i] = 0;
        F[2 * fstride + i] = 0;
    }
    // translations since the rebuild, this tick's wrap included
    const bool half = ((flag[2] + (wrap ? 1u : 0u)) & 1u) != 0u;
    if (i < n) {
        double vx = b.vx[i], vy = b.vy[i], vz = b.vz[i];
        if (lambda) {
            double l = *lambda;
            vx = xmul(vx, l);
            vy = xmul(vy, l);
            vz = xmul(vz, l);
        }
        vx = xadd(vx, xmul(b.ax[i], half_dt));
        vy = xadd(vy, xmul(b.ay[i], half_dt));
        vz = xadd(vz, xmul(b.az[i], half_dt));
        double x = xadd(b.x[i], xmul(vx, dt)), y = xadd(b.y[i], xmul(vy, dt)), z = xadd(b.z[i], xmul(vz, dt));
        if (wrap) {
            x = xsub(rem_euclid(x, xmul(2.0, hx)), hx);
            y = xsub(rem_euclid(y, xmul(2.0, hy)), hy);
            z = xsub(rem_euclid(z, xmul(2.0, hz)), hz);
        }
        b.vx[i] = vx;
        b.vy[i] = vy;
        b.vz[i] = vz;
        b.x[i] = x;
        b.y[i] = y;
        b.z[i] = z;
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            atomicOr(err, kErrNonFinite);
            over = true;
        } else {
            float4 p = stage_one(g, b, home[i], i, x, y, z, half);
            pos4[i] = p;
            float4 r = ref[i];
            float dx = p.x - r.x, dy = p.y - r.y, dz = p.z - r.z;
            over = !(dx * dx + dy * dy + dz * dz <= lim2);
        }
    }
    if (__any_sync(0xffffffffu, over) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// buf[cur ^ 1] (just gathered) back into buf[cur], so the live state never
// changes buffers and the captured tick does not depend on a parity.
__global__ void k_nl_copy(StateBuf s, StateBuf d, uint32_t n, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    d.x[p] = s.x[p];
    d.y[p] = s.y[p];
    d.z[p] = s.z[p];
    d.vx[p] = s.vx[p];
    d.vy[p] = s.vy[p];
    d.vz[p] = s.vz[p];
    d.ax[p] = s.ax[p];
    d.ay[p] = s.ay[p];
    d.az[p] = s.az[p];
    d.charge[p] = s.charge[p];
    d.mass[p] = s.mass[p];
    d.inv_mass[p] = s.inv_mass[p];
    d.elem[p] = s.elem[p];
    d.kind[p] = s.kind[p];
    d.slot[p] = s.slot[p];
}

__global__ void k_nl_stage(GridGeom g, StateBuf b, const uint32_t* __restrict__ home, uint32_t n,
                           float4* __restrict__ pos4, float4* __restrict__ ref, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = stage_one(g, b, home[i], i, b.x[i], b.y[i], b.z[i], false);
    pos4[i] = p;
    ref[i] = p;
}

// List of the pairs within r_l (r_l^2 = rl2) over the 27 home-grid cells:
// every neighbour (full list), or with HALF only those at a later sorted
// position (each pair once).  A neighbour cell whose nearest point is out of
// reach of the atom is skipped whole, and the cell's periodic shift is added
// to the atom once per cell; the resulting rounding differences (an ulp of
// a cell length) lie well inside the 1e-6 relative margin of r_l, so the
// list still holds every pair within r_c + skin.
template <bool HALF>
__global__ void __launch_bounds__(kNlBuildThreads) k_nl_build(GridGeom g, const float4* __restrict__ pos4,
                                                          const uint32_t* __restrict__ home,
                                                          const uint32_t* __restrict__ start, uint32_t n, float rl2,
                                                          uint32_t* __restrict__ list, size_t stride, int cap_nb,
                                                          uint32_t* __restrict__ cnt, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t p = blockIdx.x * kNlBuildThreads + threadIdx.x;
    if (p >= n) return;
    const float4 pi = pos4[p];
    const uint32_t c = home[p];
    uint32_t cx, cy, cz;
    decode(g, c, cx, cy, cz);
    // atoms of a cell sit within [0, cell) of its frame up to staging rounding
    const float slack = 1e-3f;
    uint32_t m = 0;
    for (uint32_t code = 0; code < 27; ++code) {
        const int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
        const uint32_t B = cell_at(g, cx, cy, cz, code);
        // atoms are sorted by cell: a lower cell index means every q < p
        if (HALF && B < c) continue;
        const float mx = fmaxf((ox > 0 ? g.cellf[0] - pi.x : (ox < 0 ? pi.x : 0.f)) - slack, 0.f);
        const float my = fmaxf((oy > 0 ? g.cellf[1] - pi.y : (oy < 0 ? pi.y : 0.f)) - slack, 0.f);
        const float mz = fmaxf((oz > 0 ? g.cellf[2] - pi.z : (oz < 0 ? pi.z : 0.f)) - slack, 0.f);
        if (dist2(mx, my, mz) >= rl2) continue;  // the whole cell is out of reach
        float sx, sy, sz;
        code_shift(g, code, sx, sy, sz);
        const float qx = fadd(pi.x, sx), qy = fadd(pi.y, sy), qz = fadd(pi.z, sz);
        uint32_t lo = start[B];
        const uint32_t hi = start[B + 1];
        if (HALF && B == c) lo = p + 1;  // HALF: every candidate lies after p
#pragma unroll(kNlBuildUnroll)
        for (uint32_t q = lo; q < hi; ++q) {
            if (!HALF && q == p) continue;
            const float4 pj = pos4[q];
            if (dist2(fsub(qx, pj.x), fsub(qy, pj.y), fsub(qz, pj.z)) < rl2) {
                if (m < (uint32_t)cap_nb) list[(size_t)m * stride + p] = q | (code << 27);
                ++m;
            }
        }
    }
    cnt[p] = m;
}

// The rebuild body's condition: the flag k_nl_advance raised.
__global__ void k_nl_set_cond(cudaGraphConditionalHandle hc, const uint32_t* __restrict__ flag) {
    cudaGraphSetConditional(hc, flag[0] != 0u ? 1u : 0u);
}

__global__ void k_nl_body_done(uint32_t* flag) { flag[3] += 1u; }

__global__ void k_nl_end(uint32_t* flag, int wrap, unsigned long long* __restrict__ counts) {
    // the force pass's potential, pair and bond-energy counters start at zero
    counts[0] = counts[1] = counts[2] = counts[3] = 0ull;
    if (flag[0]) {
        flag[1] += 1u;
        flag[0] = 0u;
        flag[2] = 0u;
    } else if (wrap) {
        flag[2] ^= 1u;
    }
}

template <int BS>
__device__ __forceinline__ unsigned long long block_sum_u(unsigned long long v, unsigned long long* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < BS / 32) ? sh[threadIdx.x] : 0ull;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

// The half-list pass with one lane per atom and the far end's force kept in
// the block where it can be.  Atoms are sorted by cell, so a block of BS
// consecutive atoms covers whole runs of cells along x, and for about half
// of the pairs within r_c the far end q lies in the same block (a numpy
// count on the quench lattice: 47 % at 128 atoms, 56 % at 256).  Those far
// ends go into 64-bit sums in shared memory, each kept as two 32-bit words
// added with the low word's carry (two native 32-bit shared atomics, where a
// 64-bit shared atomic is several times slower); the others go to global
// memory as in k_nl_force.  At the end each thread adds its atom's shared
// sum to its own and writes one global atomic per component.  Integer sums
// modulo 2^64, so the forces are the same bits as k_nl_force's.
template <bool ENERGY, int BS>
__global__ void __launch_bounds__(BS) k_nl_force_local(GridGeom g, const float4* __restrict__ pos4,
                                                        const uint32_t* __restrict__ home,
                                                        const uint32_t* __restrict__ start, uint32_t n, LawF32 L,
                                                        const PairF* __restrict__ tab,
                                                        const uint32_t* __restrict__ list, size_t stride,
                                                        int cap_nb, const uint32_t* __restrict__ cnt,
                                                        long long* __restrict__ F, size_t fstride,
                                                        unsigned long long* __restrict__ vacc,
                                                        unsigned long long* __restrict__ npairs,
                                                        uint32_t* __restrict__ err) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ float4 s_shift[27];
    __shared__ unsigned long long shu[BS / 32];
    __shared__ uint32_t s_lo[3][BS], s_hi[3][BS];
    const int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += BS) st[t] = tab[t];
    if (threadIdx.x < 27) {
        float sx, sy, sz;
        code_shift(g, threadIdx.x, sx, sy, sz);
        s_shift[threadIdx.x] = make_float4(sx, sy, sz, 0.f);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        s_lo[c][threadIdx.x] = 0u;
        s_hi[c][threadIdx.x] = 0u;
    }
    __syncthreads();
    const uint32_t b0 = blockIdx.x * BS;
    const uint32_t p = b0 + threadIdx.x;
    PairAcc a;
    // the far end's share of one pair: shared memory inside the block, else global
    auto far = [&](uint32_t q, long long fx, long long fy, long long fz) {
        const uint32_t lq = q - b0;
        if (lq < (uint32_t)BS) {
            const long long v[3] = {-fx, -fy, -fz};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const unsigned long long u = (unsigned long long)v[c];
                const uint32_t lo = (uint32_t)u, old = atomicAdd(&s_lo[c][lq], lo);
                atomicAdd(&s_hi[c][lq], (uint32_t)(u >> 32) + (old + lo < old ? 1u : 0u));
            }
        } else {
            atomicAdd((unsigned long long*)&F[q], (unsigned long long)(-fx));
            atomicAdd((unsigned long long*)&F[fstride + q], (unsigned long long)(-fy));
            atomicAdd((unsigned long long*)&F[2 * fstride + q], (unsigned long long)(-fz));
        }
    };
    auto pair = [&](const float4& pi, int ki, const float4& pj, const float4& sh, uint32_t q) {
        const float dx = delta1(pi.x, pj.x, sh.x), dy = delta1(pi.y, pj.y, sh.y), dz = delta1(pi.z, pj.z, sh.z);
        const float d2 = dist2(dx, dy, dz);
        if (!(d2 < L.rc2) || d2 == 0.f) return;
        float fs, v;
        pair_f32(L, st[ki * L.nkinds + __float_as_int(pj.w)], d2, fs, v);
        long long qx, qy, qz;
                quant3(fmul(dx, fs), fmul(dy, fs), fmul(dz, fs), qx, qy, qz, err);
        a.fx += qx;
        a.fy += qy;
        a.fz += qz;
        far(q, qx, qy, qz);
        if (ENERGY && q > p) {
            a.vq += quant(v, err);
            ++a.np;
        }
    };
    if (p < n) {
        const float4 pi = pos4[p];
        const int ki = __float_as_int(pi.w);
        const uint32_t m = cnt[p];
        if (m <= (uint32_t)cap_nb) {
            const uint32_t* lp = list + p;
            uint32_t e = 0;
            for (; e + 4 <= m; e += 4) {  // four entries per round, every load issued before any pair math
                uint32_t w[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] = __ldg(lp + (size_t)(e + k) * stride);
                float4 pj[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) pj[k] = __ldg(pos4 + (w[k] & kIdxMask));
#pragma unroll
                for (int k = 0; k < 4; ++k) pair(pi, ki, pj[k], s_shift[w[k] >> 27], w[k] & kIdxMask);
            }
            for (; e < m; ++e) {
                const uint32_t w = __ldg(lp + (size_t)e * stride);
                pair(pi, ki, __ldg(pos4 + (w & kIdxMask)), s_shift[w >> 27], w & kIdxMask);
            }
        } else {  // overflowed list: scan the home-grid cells directly
            uint32_t cx, cy, cz;
            const uint32_t c = home[p];
            decode(g, c, cx, cy, cz);
            for (uint32_t code = 0; code < 27; ++code) {
                const uint32_t B = cell_at(g, cx, cy, cz, code);
                if (B < c) continue;
                for (uint32_t q = start[B], hi = start[B + 1]; q < hi; ++q)
                    if (q > p) pair(pi, ki, pos4[q], s_shift[code], q);
            }
        }
    }
    __syncthreads();
    if (p < n) {
        const long long sx = (long long)(((unsigned long long)s_hi[0][threadIdx.x] << 32) | s_lo[0][threadIdx.x]);
        const long long sy = (long long)(((unsigned long long)s_hi[1][threadIdx.x] << 32) | s_lo[1][threadIdx.x]);
        const long long sz = (long long)(((unsigned long long)s_hi[2][threadIdx.x] << 32) | s_lo[2][threadIdx.x]);
        atomicAdd((unsigned long long*)&F[p], (unsigned long long)(a.fx + sx));
        atomicAdd((unsigned long long*)&F[fstride + p], (unsigned long long)(a.fy + sy));
        atomicAdd((unsigned long long*)&F[2 * fstride + p], (unsigned long long)(a.fz + sz));
    }
    if (ENERGY) {
        unsigned long long sv = block_sum_u<BS>((unsigned long long)a.vq, shu);
        unsigned long long np = block_sum_u<BS>(a.np, shu);
        if (threadIdx.x == 0) {
            if (sv) atomicAdd(vacc, sv);
            if (np) atomicAdd(npairs, np);
        }
    }
}

// Full list: each thread sums its own atom's forces and stores them.  HALF:
// each pair once, the far end's force through 64-bit integer atomics (F must
// be zero on entry); both give the same fixed-point sums.  Without ENERGY
// (ticks that record nothing) the potential and the pair count are left
// out: the forces are the same bits.
template <bool HALF, bool ENERGY>
__global__ void __launch_bounds__(kNlThreads) k_nl_force(GridGeom g, const float4* __restrict__ pos4,
                                                          const uint32_t* __restrict__ home,
                                                          const uint32_t* __restrict__ start, uint32_t n, LawF32 L,
                                                          const PairF* __restrict__ tab,
                                                          const uint32_t* __restrict__ list, size_t stride,
                                                          int cap_nb, const uint32_t* __restrict__ cnt,
                                                          long long* __restrict__ F, size_t fstride,
                                                          unsigned long long* __restrict__ vacc,
                                                          unsigned long long* __restrict__ npairs,
                                                          uint32_t* __restrict__ err) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ float4 s_shift[27];
    __shared__ unsigned long long shu[kNlThreads / 32];
    int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kNlThreads) st[t] = tab[t];
    if (threadIdx.x < 27) {
        float sx, sy, sz;
        code_shift(g, threadIdx.x, sx, sy, sz);
        s_shift[threadIdx.x] = make_float4(sx, sy, sz, 0.f);
    }
    __syncthreads();
    uint32_t p = blockIdx.x * kNlThreads + threadIdx.x;
    PairAcc a;
    if (p < n) {
        float4 pi = pos4[p];
        int ki = __float_as_int(pi.w);
        uint32_t m = cnt[p];
        if (m <= (uint32_t)cap_nb) {
            // four entries per round, every load issued before any pair math
            const uint32_t* lp = list + p;
            uint32_t e = 0;
            for (; e + 4 <= m; e += 4) {
                uint32_t w[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k] = __ldg(lp + (size_t)(e + k) * stride);
                float4 pj[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) pj[k] = __ldg(pos4 + (w[k] & kIdxMask));
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    float4 sh = s_shift[w[k] >> 27];
                    uint32_t q = w[k] & kIdxMask;
                    nl_pair(L, st, ki, pi, pj[k], sh.x, sh.y, sh.z, ENERGY && (HALF || q > p), a, err, HALF ? F : nullptr, q,
                            fstride);
                }
            }
            for (; e < m; ++e) {
                uint32_t w = __ldg(lp + (size_t)e * stride);
                float4 sh = s_shift[w >> 27];
                uint32_t q = w & kIdxMask;
                nl_pair(L, st, ki, pi, __ldg(pos4 + q), sh.x, sh.y, sh.z, ENERGY && (HALF || q > p), a, err,
                        HALF ? F : nullptr, q, fstride);
            }
        } else {  // overflowed list: scan the home-grid cells directly
            uint32_t cx, cy, cz;
            decode(g, home[p], cx, cy, cz);
            const uint32_t c = home[p];
            for (uint32_t code = 0; code < 27; ++code) {
                uint32_t B = cell_at(g, cx, cy, cz, code);
                if (HALF && B < c) continue;
                float sx, sy, sz;
                code_shift(g, code, sx, sy, sz);
                for (uint32_t q = start[B], hi = start[B + 1]; q < hi; ++q)
                    if (HALF ? q > p : q != p)
                        nl_pair(L, st, ki, pi, pos4[q], sx, sy, sz, ENERGY && q > p, a, err, HALF ? F : nullptr, q, fstride);
            }
        }
        if (HALF) {
            atomicAdd((unsigned long long*)&F[p], (unsigned long long)a.fx);
            atomicAdd((unsigned long long*)&F[fstride + p], (unsigned long long)a.fy);
            atomicAdd((unsigned long long*)&F[2 * fstride + p], (unsigned long long)a.fz);
        } else {
            F[p] = a.fx;
            F[fstride + p] = a.fy;
            F[2 * fstride + p] = a.fz;
        }
    }
    if (ENERGY) {
        unsigned long long s = block_sum_u<kNlThreads>((unsigned long long)a.vq, shu);
        unsigned long long np = block_sum_u<kNlThreads>(a.np, shu);
        if (threadIdx.x == 0) {
            if (s) atomicAdd(vacc, s);
            if (np) atomicAdd(npairs, np);
        }
    }
}

// TPP lanes per atom: lane k of an atom's group takes list entries k,
// k + TPP, ... (more independent gathers in flight, less divergence between
// list lengths); the group's integer partial sums are combined with
// shuffles, so every TPP gives the same bits.
template <bool HALF, int TPP, bool ENERGY>
__global__ void __launch_bounds__(kNlThreads) k_nl_force_tpp(GridGeom g, const float4* __restrict__ pos4,
                                                              const uint32_t* __restrict__ home,
                                                              const uint32_t* __restrict__ start, uint32_t n,
                                                              LawF32 L, const PairF* __restrict__ tab,
                                                              const uint32_t* __restrict__ list, size_t stride,
                                                              int cap_nb, const uint32_t* __restrict__ cnt,
                                                              long long* __restrict__ F, size_t fstride,
                                                              unsigned long long* __restrict__ vacc,
                                                              unsigned long long* __restrict__ npairs,
                                                              uint32_t* __restrict__ err) {
    static_assert(kNlThreads % TPP == 0 && 32 % TPP == 0, "TPP must divide the warp");
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ float4 s_shift[27];
    __shared__ unsigned long long shu[kNlThreads / 32];
    int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kNlThreads) st[t] = tab[t];
    if (threadIdx.x < 27) {
        float sx, sy, sz;
        code_shift(g, threadIdx.x, sx, sy, sz);
        s_shift[threadIdx.x] = make_float4(sx, sy, sz, 0.f);
    }
    __syncthreads();
    const uint32_t gid = blockIdx.x * kNlThreads + threadIdx.x;
    const uint32_t p = gid / TPP;
    const uint32_t sub = threadIdx.x % TPP;
    PairAcc a;
    if (p < n) {
        float4 pi = pos4[p];
        int ki = __float_as_int(pi.w);
        uint32_t m = cnt[p];
        if (m <= (uint32_t)cap_nb) {
            const uint32_t* lp = list + p;
            uint32_t e = sub;
            for (; e + TPP < m; e += 2 * TPP) {  // two entries per round, loads first
                uint32_t w0 = __ldg(lp + (size_t)e * stride), w1 = __ldg(lp + (size_t)(e + TPP) * stride);
                float4 p0 = __ldg(pos4 + (w0 & kIdxMask)), p1 = __ldg(pos4 + (w1 & kIdxMask));
                float4 s0 = s_shift[w0 >> 27], s1 = s_shift[w1 >> 27];
                uint32_t q0 = w0 & kIdxMask, q1 = w1 & kIdxMask;
                nl_pair(L, st, ki, pi, p0, s0.x, s0.y, s0.z, ENERGY && (HALF || q0 > p), a, err, HALF ? F : nullptr, q0,
                        fstride);
                nl_pair(L, st, ki, pi, p1, s1.x, s1.y, s1.z, ENERGY && (HALF || q1 > p), a, err, HALF ? F : nullptr, q1,
                        fstride);
            }
            if (e < m) {
                uint32_t w = __ldg(lp + (size_t)e * stride);
                float4 sh = s_shift[w >> 27];
                uint32_t q = w & kIdxMask;
                nl_pair(L, st, ki, pi, __ldg(pos4 + q), sh.x, sh.y, sh.z, ENERGY && (HALF || q > p), a, err,
                        HALF ? F : nullptr, q, fstride);
            }
        } else {  // overflowed list: the group splits the 27 home-grid cells
            uint32_t cx, cy, cz;
            decode(g, home[p], cx, cy, cz);
            const uint32_t c = home[p];
            for (uint32_t code = sub; code < 27; code += TPP) {
                uint32_t B = cell_at(g, cx, cy, cz, code);
                if (HALF && B < c) continue;
                float sx, sy, sz;
                code_shift(g, code, sx, sy, sz);
                for (uint32_t q = start[B], hi = start[B + 1]; q < hi; ++q)
                    if (HALF ? q > p : q != p)
                        nl_pair(L, st, ki, pi, pos4[q], sx, sy, sz, ENERGY && q > p, a, err, HALF ? F : nullptr, q, fstride);
            }
        }
    }
#pragma unroll
    for (int o = TPP / 2; o > 0; o >>= 1) {
        a.fx += __shfl_down_sync(0xffffffffu, a.fx, o, TPP);
        a.fy += __shfl_down_sync(0xffffffffu, a.fy, o, TPP);
        a.fz += __shfl_down_sync(0xffffffffu, a.fz, o, TPP);
    }
    if (p < n && sub == 0) {
        if (HALF) {
            atomicAdd((unsigned long long*)&F[p], (unsigned long long)a.fx);
            atomicAdd((unsigned long long*)&F[fstride + p], (unsigned long long)a.fy);
            atomicAdd((unsigned long long*)&F[2 * fstride + p], (unsigned long long)a.fz);
        } else {
            F[p] = a.fx;
            F[fstride + p] = a.fy;
            F[2 * fstride + p] = a.fz;
        }
    }
    if (ENERGY) {
        unsigned long long s = block_sum_u<kNlThreads>((unsigned long long)a.vq, shu);
        unsigned long long np = block_sum_u<kNlThreads>(a.np, shu);
        if (threadIdx.x == 0) {
            if (s) atomicAdd(vacc, s);
            if (np) atomicAdd(npairs, np);
        }
    }
}

// Variant 7: the half list of variant 6, evaluated in two phases per round.
// Each thread first walks its list and keeps the entries that lie within the
// cutoff (their displacement and the packed partner index and kind) in a
// shared-memory stash of S slots; then the warp runs the pair law over the
// stashed entries together.  The lanes whose atoms have fewer pairs in range
// wait only in the short collection loop, not in the pair law, which keeps
// more of the warp busy in the arithmetic.  Same pairs, same per-pair
// operations, same integer sums: the forces are bit-identical to variant 6.
template <bool ENERGY, int S>
__global__ void __launch_bounds__(kNlThreads) k_nl_force_cmp(GridGeom g, const float4* __restrict__ pos4,
                                                              const uint32_t* __restrict__ home,
                                                              const uint32_t* __restrict__ start, uint32_t n,
                                                              LawF32 L, const PairF* __restrict__ tab,
                                                              const uint32_t* __restrict__ list, size_t stride,
                                                              int cap_nb, const uint32_t* __restrict__ cnt,
                                                              long long* __restrict__ F, size_t fstride,
                                                              unsigned long long* __restrict__ vacc,
                                                              unsigned long long* __restrict__ npairs,
                                                              uint32_t* __restrict__ err) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ float4 s_shift[27];
    __shared__ unsigned long long shu[kNlThreads / 32];
    __shared__ float4 stash[S * kNlThreads];  // slot k of thread t at [k * kNlThreads + t]
    int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kNlThreads) st[t] = tab[t];
    if (threadIdx.x < 27) {
        float sx, sy, sz;
        code_shift(g, threadIdx.x, sx, sy, sz);
        s_shift[threadIdx.x] = make_float4(sx, sy, sz, 0.f);
    }
    __syncthreads();
    const uint32_t p = blockIdx.x * kNlThreads + threadIdx.x;
    PairAcc a;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int ki = 0;
    uint32_t m = 0;
    if (p < n) {
        pi = pos4[p];
        ki = __float_as_int(pi.w);
        m = cnt[p];
        if (m > (uint32_t)cap_nb) {  // overflowed list: scan the home-grid cells directly
            uint32_t cx, cy, cz;
            const uint32_t c = home[p];
            decode(g, c, cx, cy, cz);
            for (uint32_t code = 0; code < 27; ++code) {
                uint32_t B = cell_at(g, cx, cy, cz, code);
                if (B < c) continue;
                float4 sh = s_shift[code];
                for (uint32_t q = start[B], hi = start[B + 1]; q < hi; ++q)
                    if (q > p) nl_pair(L, st, ki, pi, pos4[q], sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);
            }
            m = 0;
        }
    }
    const uint32_t* lp = list + p;
    float4* my = stash + threadIdx.x;
    uint32_t e = 0;
    while (__any_sync(0xffffffffu, e < m)) {
        // collect: up to S in-range entries, four list entries per round with every load issued first
        int k = 0;
        for (; e + 4 <= m && k <= S - 4; e += 4) {
            uint32_t w[4];
            float4 pj[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) w[u] = __ldg(lp + (size_t)(e + u) * stride);
#pragma unroll
            for (int u = 0; u < 4; ++u) pj[u] = __ldg(pos4 + (w[u] & kIdxMask));
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float4 sh = s_shift[w[u] >> 27];
                const float dx = delta1(pi.x, pj[u].x, sh.x), dy = delta1(pi.y, pj[u].y, sh.y),
                            dz = delta1(pi.z, pj[u].z, sh.z);
                const float d2 = dist2(dx, dy, dz);
                if (d2 < L.rc2 && d2 != 0.f) {
                    my[k * kNlThreads] = make_float4(
                        dx, dy, dz, __uint_as_float((w[u] & kIdxMask) | ((uint32_t)__float_as_int(pj[u].w) << 27)));
                    ++k;
                }
            }
        }
        for (; e < m && k < S; ++e) {
            const uint32_t w = __ldg(lp + (size_t)e * stride);
            const float4 pj = __ldg(pos4 + (w & kIdxMask));
            const float4 sh = s_shift[w >> 27];
            const float dx = delta1(pi.x, pj.x, sh.x), dy = delta1(pi.y, pj.y, sh.y), dz = delta1(pi.z, pj.z, sh.z);
            const float d2 = dist2(dx, dy, dz);
            if (d2 < L.rc2 && d2 != 0.f) {
                my[k * kNlThreads] =
                    make_float4(dx, dy, dz, __uint_as_float((w & kIdxMask) | ((uint32_t)__float_as_int(pj.w) << 27)));
                ++k;
            }
        }
        int kmax = k;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
        // evaluate: the warp runs the pair law over the stashed entries together
        for (int t = 0; t < kmax; ++t) {
            if (t < k) {
                const float4 sv = my[t * kNlThreads];
                const uint32_t qk = __float_as_uint(sv.w);
                const uint32_t q = qk & kIdxMask;
                float fs, v;
                pair_f32(L, st[ki * L.nkinds + (int)(qk >> 27)], dist2(sv.x, sv.y, sv.z), fs, v);
                long long qx, qy, qz;
                    quant3(fmul(sv.x, fs), fmul(sv.y, fs), fmul(sv.z, fs), qx, qy, qz, err);
                a.fx += qx;
                a.fy += qy;
                a.fz += qz;
                atomicAdd((unsigned long long*)&F[q], (unsigned long long)(-qx));
                atomicAdd((unsigned long long*)&F[fstride + q], (unsigned long long)(-qy));
                atomicAdd((unsigned long long*)&F[2 * fstride + q], (unsigned long long)(-qz));
                if (ENERGY && q > p) {
                    a.vq += quant(v, err);
                    ++a.np;
                }
            }
        }
    }
    if (p < n) {
        atomicAdd((unsigned long long*)&F[p], (unsigned long long)a.fx);
        atomicAdd((unsigned long long*)&F[fstride + p], (unsigned long long)a.fy);
        atomicAdd((unsigned long long*)&F[2 * fstride + p], (unsigned long long)a.fz);
    }
    if (ENERGY) {
        unsigned long long s = block_sum_u<kNlThreads>((unsigned long long)a.vq, shu);
        unsigned long long np = block_sum_u<kNlThreads>(a.np, shu);
        if (threadIdx.x == 0) {
            if (s) atomicAdd(vacc, s);
            if (np) atomicAdd(npairs, np);
        }
    }
}

// Bricks.  A brick is K consecutive list-grid cells of one x-row; atoms are
// sorted by cell, so its home atoms are one contiguous range, and the
// neighbour cells of every home cell lie in the 9 rows (y +- 1, z +- 1) over
// x0 - 1 .. x0 + K, each at most two contiguous ranges of sorted atoms (two
// where the x-range wraps).  brick_stage copies those ranges of the float4
// staging into shared memory as TMA bulk copies (cp.async.bulk: every range
// starts on a 16-byte boundary and is a whole number of float4s; no
// multicast, the source is this GPU's memory) completing on one mbarrier,
// and every thread polls it a bounded number of times.  A partner in
// neighbour-cell code c lies in row c / 3 (code = (ox+1) + 3 (oy+1) +
// 9 (oz+1)), whose ranges give its shared-memory slot.  A brick whose
// neighbourhood exceeds CAP atoms reads global memory instead.
constexpr uint32_t kBrickWaitLimit = 1u << 20;  // polls of the staging mbarrier before giving up

template <int CAP>
struct BrickSmem {
    float4 pos[CAP];
    uint32_t gA[9], eA[9], oA[9], gB[9], eB[9], oB[9];
    uint32_t total;
    unsigned long long mbar;
};

// Stages the brick's neighbourhood; [hlo, hhi) = its home atoms.  Returns
// false (on every thread, after the copies in flight have landed and
// kErrTimeout is set) when the staging wait gave up.
template <int CAP>
__device__ bool brick_stage(const GridGeom& g, const uint32_t* __restrict__ start, const float4* __restrict__ pos4,
                            uint32_t K, uint32_t nchunks, BrickSmem<CAP>& S, uint32_t* __restrict__ err,
                            uint32_t& hlo, uint32_t& hhi) {
    const uint32_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const uint32_t row = blockIdx.x / nchunks, chunk = blockIdx.x - row * nchunks;
    const uint32_t cy = row % ny, cz = row / ny;
    const uint32_t x0 = chunk * K, x1 = min(x0 + K, nx);  // home cells x0 .. x1 - 1
    if (threadIdx.x < 9) {
        const int dy = (int)(threadIdx.x % 3) - 1, dz = (int)(threadIdx.x / 3) - 1;
        const uint32_t rb = nx * (wrap_add(cy, dy, ny) + ny * wrap_add(cz, dz, nz));  // cell x = 0 of the row
        uint32_t gA, eA, gB = 0, eB = 0;
        if (x1 - x0 + 2 >= nx) {  // cells x0 - 1 .. x1 cover the whole row
            gA = start[rb];
            eA = start[rb + nx];
        } else if (x0 == 0) {  // cell nx - 1, then 0 .. x1
            gA = start[rb + nx - 1];
            eA = start[rb + nx];
            gB = start[rb];
            eB = start[rb + x1 + 1];
        } else if (x1 == nx) {  // x0 - 1 .. nx - 1, then cell 0
            gA = start[rb + x0 - 1];
            eA = start[rb + nx];
            gB = start[rb];
            eB = start[rb + 1];
        } else {
            gA = start[rb + x0 - 1];
            eA = start[rb + x1 + 1];
        }
        S.gA[threadIdx.x] = gA;
        S.eA[threadIdx.x] = eA;
        S.gB[threadIdx.x] = gB;
        S.eB[threadIdx.x] = eB;
    }
    const uint32_t hb = nx * (cy + ny * cz);
    hlo = start[hb + x0];
    hhi = start[hb + x1];
    __syncthreads();
    const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&S.mbar);
    if (threadIdx.x == 0) {
        uint32_t off = 0;
        for (int r = 0; r < 9; ++r) {
            S.oA[r] = off;
            off += S.eA[r] - S.gA[r];
            S.oB[r] = off;
            off += S.eB[r] - S.gB[r];
        }
        S.total = off;
        if (off && off <= (uint32_t)CAP) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(off * 16u)
                         : "memory");
            for (int r = 0; r < 9; ++r) {
                const uint32_t gs[2] = {S.gA[r], S.gB[r]}, ln[2] = {S.eA[r] - S.gA[r], S.eB[r] - S.gB[r]},
                               os[2] = {S.oA[r], S.oB[r]};
                for (int k = 0; k < 2; ++k) {
                    if (!ln[k]) continue;
                    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(S.pos + os[k]);
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                            dst),
                        "l"(pos4 + gs[k]), "r"(ln[k] * 16u), "r"(mbar)
                        : "memory");
                }
            }
        }
    }
    __syncthreads();
    if (S.total && S.total <= (uint32_t)CAP) {
        auto wait = [&](uint32_t limit) -> bool {
            for (uint32_t it = 0; it < limit; ++it) {
                uint32_t done = 0;
                asm volatile(
                    "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                    : "=r"(done)
                    : "r"(mbar), "r"(0u)
                    : "memory");
                if (done) return true;
            }
            return false;
        };
        const bool ok = wait(kBrickWaitLimit);
        if (__syncthreads_or(!ok)) {  // every thread leaves together
            if (!ok) wait(kBrickWaitLimit);  // let copies still in flight land before the block exits
            if (threadIdx.x == 0) atomicOr(err, kErrTimeout);
            return false;
        }
    }
    return true;
}

// Shared-memory slot of the atom at sorted position q seen through
// neighbour-cell code `code`; >= S.total when not staged (not expected for a
// list partner; the caller then reads global memory).
template <int CAP>
__device__ __forceinline__ uint32_t brick_slot(const BrickSmem<CAP>& S, uint32_t q, uint32_t code) {
    const uint32_t r = code / 3u;
    return q - S.gA[r] < S.eA[r] - S.gA[r] ? S.oA[r] + (q - S.gA[r]) : S.oB[r] + (q - S.gB[r]);
}

template <int CAP>
__device__ __forceinline__ float4 brick_pos(const BrickSmem<CAP>& S, bool staged, uint32_t w,
                                            const float4* __restrict__ pos4) {
    const uint32_t q = w & kIdxMask;
    if (!staged) return __ldg(pos4 + q);
    const uint32_t idx = brick_slot(S, q, w >> 27);
    return idx < S.total ? S.pos[idx] : __ldg(pos4 + q);
}

// Variant 8: the half list of variant 6, evaluated brick by brick, each
// partner read from the staged neighbourhood.  Same pairs and per-pair
// operations as variant 6: bit-identical forces.
template <bool ENERGY, int CAP>
__global__ void __launch_bounds__(kNlThreads) k_nl_force_brick(GridGeom g, const float4* __restrict__ pos4,
                                                                const uint32_t* __restrict__ home,
                                                                const uint32_t* __restrict__ start, uint32_t n,
                                                                LawF32 L, const PairF* __restrict__ tab,
                                                                const uint32_t* __restrict__ list, size_t stride,
                                                                int cap_nb, const uint32_t* __restrict__ cnt,
                                                                long long* __restrict__ F, size_t fstride,
                                                                unsigned long long* __restrict__ vacc,
                                                                unsigned long long* __restrict__ npairs,
                                                                uint32_t* __restrict__ err, uint32_t K,
                                                                uint32_t nchunks) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ float4 s_shift[27];
    __shared__ unsigned long long shu[kNlThreads / 32];
    __shared__ __align__(16) BrickSmem<CAP> S;
    const int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kNlThreads) st[t] = tab[t];
    if (threadIdx.x < 27) {
        float sx, sy, sz;
        code_shift(g, threadIdx.x, sx, sy, sz);
        s_shift[threadIdx.x] = make_float4(sx, sy, sz, 0.f);
    }
    uint32_t hlo, hhi;
    if (!brick_stage<CAP>(g, start, pos4, K, nchunks, S, err, hlo, hhi)) return;
    const bool staged = S.total <= (uint32_t)CAP;
    PairAcc a;
    for (uint32_t p = hlo + threadIdx.x; p < hhi; p += kNlThreads) {
        const float4 pi = pos4[p];
        const int ki = __float_as_int(pi.w);
        const uint32_t m = cnt[p];
        a.fx = a.fy = a.fz = 0;  // this atom's own sums (the potential and pair count run on)
        if (m <= (uint32_t)cap_nb) {
            const uint32_t* lp = list + p;
            uint32_t e = 0;
            for (; e + 4 <= m; e += 4) {
                uint32_t w[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) w[u] = __ldg(lp + (size_t)(e + u) * stride);
                float4 pj[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) pj[u] = brick_pos(S, staged, w[u], pos4);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float4 sh = s_shift[w[u] >> 27];
                    const uint32_t q = w[u] & kIdxMask;
                    nl_pair(L, st, ki, pi, pj[u], sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);  // half list: q > p
                }
            }
            for (; e < m; ++e) {
                const uint32_t w = __ldg(lp + (size_t)e * stride);
                const uint32_t q = w & kIdxMask;
                const float4 pj = brick_pos(S, staged, w, pos4);
                const float4 sh = s_shift[w >> 27];
                nl_pair(L, st, ki, pi, pj, sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);  // half list: q > p
            }
        } else {  // overflowed list: scan the home-grid cells directly
            uint32_t cx, ccy, ccz;
            const uint32_t c = home[p];
            decode(g, c, cx, ccy, ccz);
            for (uint32_t code = 0; code < 27; ++code) {
                const uint32_t B = cell_at(g, cx, ccy, ccz, code);
                if (B < c) continue;
                const float4 sh = s_shift[code];
                for (uint32_t q = start[B], hi = start[B + 1]; q < hi; ++q)
                    if (q > p) nl_pair(L, st, ki, pi, pos4[q], sh.x, sh.y, sh.z, ENERGY, a, err, F, q, fstride);
            }
        }
        atomicAdd((unsigned long long*)&F[p], (unsigned long long)a.fx);
        atomicAdd((unsigned long long*)&F[fstride + p], (unsigned long long)a.fy);
        atomicAdd((unsigned long long*)&F[2 * fstride + p], (unsigned long long)a.fz);
    }
    if (ENERGY) {
        unsigned long long sv = block_sum_u<kNlThreads>((unsigned long long)a.vq, shu);
        unsigned long long np = block_sum_u<kNlThreads>(a.np, shu);
        if (threadIdx.x == 0) {
            if (sv) atomicAdd(vacc, sv);
            if (np) atomicAdd(npairs, np);
        }
    }
}

// The list build of k_nl_build brick by brick: the candidates are read from
// the staged neighbourhood; the cells, the reach test, the candidate order
// and the distance test are k_nl_build's, so the lists are the same words.
template <bool HALF, int CAP>
__global__ void __launch_bounds__(kNlBuildThreads) k_nl_build_brick(GridGeom g, const float4* __restrict__ pos4,
                                                                    const uint32_t* __restrict__ home,
                                                                    const uint32_t* __restrict__ start, float rl2,
                                                                    uint32_t* __restrict__ list, size_t stride,
                                                                    int cap_nb, uint32_t* __restrict__ cnt,
                                                                    uint32_t* __restrict__ err, uint32_t K,
                                                                    uint32_t nchunks,
                                                                    const uint32_t* __restrict__ gate) {
    __shared__ __align__(16) BrickSmem<CAP> S;
    if (gated_off(gate)) return;
    uint32_t hlo, hhi;
    if (!brick_stage<CAP>(g, start, pos4, K, nchunks, S, err, hlo, hhi)) return;
    const bool staged = S.total <= (uint32_t)CAP;
    const float slack = 1e-3f;  // atoms of a cell sit within [0, cell) of its frame up to staging rounding
    for (uint32_t p = hlo + threadIdx.x; p < hhi; p += kNlBuildThreads) {
        const float4 pi = pos4[p];
        const uint32_t c = home[p];
        uint32_t cx, cy, cz;
        decode(g, c, cx, cy, cz);
        uint32_t m = 0;
        for (uint32_t code = 0; code < 27; ++code) {
            const int ox = (int)(code % 3u) - 1, oy = (int)((code / 3u) % 3u) - 1, oz = (int)(code / 9u) - 1;
            const uint32_t B = cell_at(g, cx, cy, cz, code);
            if (HALF && B < c) continue;  // atoms are sorted by cell: a lower cell index means every q < p
            const float mx = fmaxf((ox > 0 ? g.cellf[0] - pi.x : (ox < 0 ? pi.x : 0.f)) - slack, 0.f);
            const float my = fmaxf((oy > 0 ? g.cellf[1] - pi.y : (oy < 0 ? pi.y : 0.f)) - slack, 0.f);
            const float mz = fmaxf((oz > 0 ? g.cellf[2] - pi.z : (oz < 0 ? pi.z : 0.f)) - slack, 0.f);
            if (dist2(mx, my, mz) >= rl2) continue;  // the whole cell is out of reach
            float sx, sy, sz;
            code_shift(g, code, sx, sy, sz);
            const float qx = fadd(pi.x, sx), qy = fadd(pi.y, sy), qz = fadd(pi.z, sz);
            uint32_t lo = start[B];
            const uint32_t hi = start[B + 1];
            if (HALF && B == c) lo = p + 1;  // HALF: every candidate lies after p
            // the cell is one contiguous run of its row's staged range
            const uint32_t s0 = staged ? brick_slot(S, lo, code) : 0u;
            const bool in_smem = staged && lo < hi && s0 + (hi - lo) <= S.total;
#pragma unroll(kNlBuildUnroll)
            for (uint32_t q = lo; q < hi; ++q) {
                if (!HALF && q == p) continue;
                const float4 pj = in_smem ? S.pos[s0 + (q - lo)] : pos4[q];
                if (dist2(fsub(qx, pj.x), fsub(qy, pj.y), fsub(qz, pj.z)) < rl2) {
                    if (m < (uint32_t)cap_nb) list[(size_t)m * stride + p] = q | (code << 27);
                    ++m;
                }
            }
        }
        cnt[p] = m;
    }
}

template <bool HALF>
void launch_nl_force(gx_handle* h, int tpp, const GridGeom& g, const NlState* s, uint32_t n, const LawF32& L,
                     bool energy) {
    const float4* pos4 = h->pos4;
    const uint32_t* home = h->key_sorted;
    const uint32_t* start = s->cl.start;
    if (HALF && h->kernel_variant == 8) {
        const uint32_t K = s->brick == 0 ? 4u : 8u;
        const uint32_t nchunks = (g.n[0] + K - 1) / K;
        const unsigned nb = nchunks * g.n[1] * g.n[2];
        auto kb = s->brick == 0 ? (energy ? k_nl_force_brick<true, 1024> : k_nl_force_brick<false, 1024>)
                                : (energy ? k_nl_force_brick<true, 2048> : k_nl_force_brick<false, 2048>);
        GX_LAUNCH(h, kb, nb, kNlThreads, g, pos4, home, start, n, L, h->d_pairf, s->list, s->cap, s->cap_nb, s->cnt,
                  h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr, K, nchunks);
        return;
    }
    if (HALF && h->kernel_variant == 7) {
        auto kc = s->slots == 8 ? (energy ? k_nl_force_cmp<true, 8> : k_nl_force_cmp<false, 8>)
                                : (energy ? k_nl_force_cmp<true, 16> : k_nl_force_cmp<false, 16>);
        GX_LAUNCH(h, kc, nblk(n, kNlThreads), kNlThreads, g, pos4, home, start, n, L, h->d_pairf, s->list, s->cap,
                  s->cap_nb, s->cnt, h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr);
        return;
    }
    if (HALF && tpp <= 1 && s->block > 0) {  // far ends inside the block summed in shared memory
        if (s->block == 256) {
            auto kl = energy ? k_nl_force_local<true, 256> : k_nl_force_local<false, 256>;
            GX_LAUNCH(h, kl, nblk(n, 256), 256, g, pos4, home, start, n, L, h->d_pairf, s->list, s->cap, s->cap_nb,
                      s->cnt, h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr);
        } else {
            auto kl = energy ? k_nl_force_local<true, 128> : k_nl_force_local<false, 128>;
            GX_LAUNCH(h, kl, nblk(n, 128), 128, g, pos4, home, start, n, L, h->d_pairf, s->list, s->cap, s->cap_nb,
                      s->cnt, h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr);
        }
        return;
    }
    if (tpp <= 1) {
        auto k1 = energy ? k_nl_force<HALF, true> : k_nl_force<HALF, false>;
        GX_LAUNCH(h, k1, nblk(n, kNlThreads), kNlThreads, g, pos4, home, start, n, L, h->d_pairf, s->list, s->cap,
                  s->cap_nb, s->cnt, h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr);
        return;
    }
    const size_t threads = (size_t)n * tpp;
    auto k = energy ? (tpp == 2 ? k_nl_force_tpp<HALF, 2, true>
                                : (tpp == 4 ? k_nl_force_tpp<HALF, 4, true> : k_nl_force_tpp<HALF, 8, true>))
                    : (tpp == 2 ? k_nl_force_tpp<HALF, 2, false>
                                : (tpp == 4 ? k_nl_force_tpp<HALF, 4, false> : k_nl_force_tpp<HALF, 8, false>));
    GX_LAUNCH(h, k, nblk(threads, kNlThreads), kNlThreads, g, pos4, home, start, n, L, h->d_pairf, s->list, s->cap,
              s->cap_nb, s->cnt, h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr);
}

__global__ void k_nl_fix_to_double(const unsigned long long* __restrict__ v, double* out, double* zero) {
    *out = xmul(__ll2double_rn((long long)*v), kFixInv);
    *zero = 0.0;
}

template <int BS>
__device__ __forceinline__ double block_sum_d(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < BS / 32) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

// a = F 2^-32 (1/m) (as k_fix_to_acc), v += a dt/2 (as k_kick), and with
// THERMO >= 1 the kinetic-energy partials of the new v with k_kinetic's block
// mapping and operation order, so lambda is bit-identical to the unfused tick;
// THERMO = 2 also the speed partials (sum of |v|) for the tick's record.
// With vsum: also k_nl_fix_to_double's conversion of the potential (ticks
// without a bond spring, which would write the bond-energy slot after it).
template <int THERMO>
__global__ void __launch_bounds__(kRedThreads) k_nl_finish(StateBuf b, const long long* __restrict__ F,
                                                           size_t fstride, uint32_t n, double half_dt,
                                                           double* __restrict__ kpart, double* __restrict__ spart,
                                                           const unsigned long long* __restrict__ vsum,
                                                           double* __restrict__ vout, double* __restrict__ bzero) {
    __shared__ double sh[kRedThreads / 32];
    if (vsum && blockIdx.x == 0 && threadIdx.x == 0) {
        *vout = xmul(__ll2double_rn((long long)*vsum), kFixInv);
        *bzero = 0.0;
    }
    double ks = 0.0, ss = 0.0;
    for (uint32_t i = blockIdx.x * kRedThreads + threadIdx.x; i < n; i += gridDim.x * kRedThreads) {
        double im = b.inv_mass[i];
        double ax = xmul(xmul(__ll2double_rn(F[i]), kFixInv), im);
        double ay = xmul(xmul(__ll2double_rn(F[fstride + i]), kFixInv), im);
        double az = xmul(xmul(__ll2double_rn(F[2 * fstride + i]), kFixInv), im);
        b.ax[i] = ax;
        b.ay[i] = ay;
        b.az[i] = az;
        double vx = xadd(b.vx[i], xmul(ax, half_dt));
        double vy = xadd(b.vy[i], xmul(ay, half_dt));
        double vz = xadd(b.vz[i], xmul(az, half_dt));
        b.vx[i] = vx;
        b.vy[i] = vy;
        b.vz[i] = vz;
        if (THERMO) {
            double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
            ks = xadd(ks, xmul(xmul(0.5, b.mass[i]), l2));
            if (THERMO == 2) ss = xadd(ss, xsqrt(l2));
        }
    }
    if (THERMO) {
        ks = block_sum_d<kRedThreads>(ks, sh);
        if (threadIdx.x == 0) kpart[blockIdx.x] = ks;
    }
    if (THERMO == 2) {
        ss = block_sum_d<kRedThreads>(ss, sh);
        if (threadIdx.x == 0) spart[blockIdx.x] = ss;
    }
}

// Plain FP64 pass over the full list: one thread per atom visits every
// neighbour of its list (within r_c + skin at the last rebuild) in the
// build's order with the reference's exact per-pair arithmetic (the
// minimum image of the FP64 positions, pair_f64) and sums its acceleration
// in that order: no atomics, deterministic.  The list build used the FP32
// staging; its radius exceeds r_c + skin by 1e-6 relative and the staging
// error is ~1e-6 absolute, both far inside the skin/2 margin, so every pair
// with d < r_c in FP64 is in the list.  V and the pair count take each
// unordered pair once (q > p).
__global__ void __launch_bounds__(kNlThreads) k_nl_force64(GridGeom g, StateBuf b, const uint32_t* __restrict__ home,
                                                            const uint32_t* __restrict__ start, uint32_t n, LawF64 L,
                                                            const double* __restrict__ psig,
                                                            const double* __restrict__ peps,
                                                            const uint32_t* __restrict__ list, size_t stride,
                                                            int cap_nb, const uint32_t* __restrict__ cnt,
                                                            double* __restrict__ vpart,
                                                            unsigned long long* __restrict__ npairs) {
    __shared__ double shd[kNlThreads / 32];
    __shared__ unsigned long long shu[kNlThreads / 32];
    const uint32_t i = blockIdx.x * kNlThreads + threadIdx.x;
    double V = 0.0;
    unsigned long long np = 0;
    if (i < n) {
        const double xi = b.x[i], yi = b.y[i], zi = b.z[i];
        const int ti = b.elem[i];
        const double qi = b.charge[i], mi = b.mass[i], inv_mi = b.inv_mass[i];
        double ax = 0.0, ay = 0.0, az = 0.0;
        // the list grid has >= 3 cells per axis (min_image_near)
        const double hx = xmul(0.5, L.box[0]), hy = xmul(0.5, L.box[1]), hz = xmul(0.5, L.box[2]);
        auto visit = [&](uint32_t j) {
            const double dx = min_image_near(xsub(xi, b.x[j]), L.box[0], hx);
            const double dy = min_image_near(xsub(yi, b.y[j]), L.box[1], hy);
            const double dz = min_image_near(xsub(zi, b.z[j]), L.box[2], hz);
            const double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
            if (d2 >= L.rc2) return;
            const double d = xsqrt(d2);
            if (d <= kEpsF64) return;
            const int tj = b.elem[j];
            double fmag, Vij = 0.0;
            const int tt = ti * kNElem + tj;  // psig, then peps, then (24 eps) / sigma, each kNElem^2
            pair_f64_e24(L, d, psig[tt], peps[tt], peps[kNElem * kNElem + tt], qi, b.charge[j], mi, b.mass[j], fmag,
                         Vij);
            if (j > i) {
                V = xadd(V, Vij);
                ++np;
            }
            if (fmag != 0.0) {
                const double inv = xdiv(1.0, d);
                ax = xadd(ax, xmul(xmul(xmul(dx, inv), fmag), inv_mi));
                ay = xadd(ay, xmul(xmul(xmul(dy, inv), fmag), inv_mi));
                az = xadd(az, xmul(xmul(xmul(dz, inv), fmag), inv_mi));
            }
        };
        const uint32_t m = cnt[i];
        if (m <= (uint32_t)cap_nb) {
            const uint32_t* lp = list + i;
            for (uint32_t e = 0; e < m; ++e) visit(__ldg(lp + (size_t)e * stride) & kIdxMask);
        } else {  // overflowed list: every atom of the 27 home-grid cells
            uint32_t cx, cy, cz;
            decode(g, home[i], cx, cy, cz);
            for (uint32_t code = 0; code < 27; ++code) {
                const uint32_t B = cell_at(g, cx, cy, cz, code);
                for (uint32_t q = start[B], hi = start[B + 1]; q < hi; ++q)
                    if (q != i) visit(q);
            }
        }
        b.ax[i] = ax;
        b.ay[i] = ay;
        b.az[i] = az;
    }
    V = block_sum_d<kNlThreads>(V, shd);
    np = block_sum_u<kNlThreads>(np, shu);
    if (threadIdx.x == 0) {
        vpart[blockIdx.x] = V;
        if (np) atomicAdd(npairs, np);
    }
}

// FP64 second kick (as k_kick) and, with THERMO, the kinetic-energy partials
// with k_nl_finish's block mapping and operation order.
template <int THERMO>
__global__ void __launch_bounds__(kRedThreads) k_nl_finish64(StateBuf b, uint32_t n, double half_dt,
                                                             double* __restrict__ kpart, double* __restrict__ spart) {
    __shared__ double sh[kRedThreads / 32];
    double ks = 0.0, ss = 0.0;
    for (uint32_t i = blockIdx.x * kRedThreads + threadIdx.x; i < n; i += gridDim.x * kRedThreads) {
        const double vx = xadd(b.vx[i], xmul(b.ax[i], half_dt));
        const double vy = xadd(b.vy[i], xmul(b.ay[i], half_dt));
        const double vz = xadd(b.vz[i], xmul(b.az[i], half_dt));
        b.vx[i] = vx;
        b.vy[i] = vy;
        b.vz[i] = vz;
        if (THERMO) {
            double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
            ks = xadd(ks, xmul(xmul(0.5, b.mass[i]), l2));
            if (THERMO == 2) ss = xadd(ss, xsqrt(l2));
        }
    }
    if (THERMO) {
        ks = block_sum_d<kRedThreads>(ks, sh);
        if (threadIdx.x == 0) kpart[blockIdx.x] = ks;
    }
    if (THERMO == 2) {
        ss = block_sum_d<kRedThreads>(ss, sh);
        if (threadIdx.x == 0) spart[blockIdx.x] = ss;
    }
}

NlState* nl_of(gx_handle* h) {
    if (!h->nl) h->nl = new NlState();
    return static_cast<NlState*>(h->nl);
}

double skin_of(const gx_handle* h, const NlState* s) { return s->skin >= 0.0 ? s->skin : 0.1 * h->fs.rc; }

}  // namespace

void nl_free(gx_handle* h) {
    if (!h || !h->nl) return;
    NlState* s = static_cast<NlState*>(h->nl);
    cudaFree(s->list);
    cudaFree(s->cnt);
    cudaFree(s->ref);
    cudaFree(s->flag);
    cells_free(s->cl);
    if (s->side) cudaStreamDestroy(s->side);
    delete s;
    h->nl = nullptr;
}

// The list path applies to both precisions (mixed: variants 5-7; FP64: the
// full-list pass k_nl_force64) with at least 3 list-grid cells per axis (so
// the force grid has at least 3 too, and every pair within the cutoff occurs
// once in the reference's pair list) and atom indices below 2^27.
bool nl_eligible(gx_handle* h) {
    if (h->n == 0 || h->n >= (1u << 27)) return false;
    NlState* s = nl_of(h);
    double rl = h->fs.rc + skin_of(h, s);
    int ok = 0;
    GridGeom g = make_grid(h->p.box, rl, &ok);
    return ok && g.n[0] >= 3 && g.n[1] >= 3 && g.n[2] >= 3;
}

// Allocates the list state (outside any capture) and requests a rebuild
// when the handle's order no longer matches the list.
int nl_prepare(gx_handle* h, bool* stale) {
    NlState* s = nl_of(h);
    *stale = false;
    const double skin = skin_of(h, s);
    int ok = 0;
    GridGeom g = make_grid(h->p.box, h->fs.rc + skin, &ok);
    if (!ok) return set_err(h, GX_ERR_ARG, "neighbour-list grid is empty or too large");
    const double vol = h->p.box[0] * h->p.box[1] * h->p.box[2];
    const double rl = h->fs.rc + skin;
    const double expect = (double)h->n / vol * (4.0 / 3.0) * 3.14159265358979 * rl * rl * rl;
    int cap_nb = (int)std::ceil(2.0 * expect) + 32;
    cap_nb = (cap_nb + 7) & ~7;
    if (cap_nb > 1024) cap_nb = 1024;
    if (!s->flag) {
        GX_CUDA(h, cudaMalloc(&s->flag, 4 * sizeof(uint32_t)));
        GX_CUDA(h, cudaMemsetAsync(s->flag, 0, 4 * sizeof(uint32_t), h->stream));
        s->body_runs_seen = 0;
    }
    if (!s->side) GX_CUDA(h, cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    if (s->cap < h->cap || s->cap_nb < cap_nb) {
        cudaFree(s->list);
        cudaFree(s->cnt);
        cudaFree(s->ref);
        s->list = nullptr;
        s->cnt = nullptr;
        s->ref = nullptr;
        s->cap = 0;
        GX_CUDA(h, cudaMalloc(&s->list, (size_t)cap_nb * h->cap * sizeof(uint32_t)));
        GX_CUDA(h, cudaMalloc(&s->cnt, h->cap * sizeof(uint32_t)));
        GX_CUDA(h, cudaMalloc(&s->ref, h->cap * sizeof(float4)));
        GX_CUDA(h, cudaMemsetAsync(s->ref, 0, h->cap * sizeof(float4), h->stream));
        s->cap = h->cap;
        s->cap_nb = cap_nb;
        h->nl_valid = false;
        *stale = true;
    }
    // 6, 7 and automatic: half list; 5 and the FP64 pass: full list
    const int half = (h->kernel_variant == 5 || h->precision != GX_MIXED) ? 0 : 1;
    if (half != s->half) {
        s->half = half;
        h->nl_valid = false;
        *stale = true;
    }
    if (std::memcmp(&g, &s->lg, sizeof g) != 0 || s->skin_used != skin) {
        s->lg = g;
        s->skin_used = skin;
        h->nl_valid = false;
        *stale = true;
    }
    const size_t cl_cap = s->cl.cap_cells;
    int rc = ensure_cells(h, s->cl, g.ncell);
    if (rc) return rc;
    if ((rc = ensure_sort_tmp(h, s->cl, h->cap))) return rc;  // the captured rebuild must not allocate
    if (s->cl.cap_cells != cl_cap) *stale = true;
    if (!h->nl_valid) {
        const uint32_t one = 1u;
        GX_CUDA(h, cudaMemcpyAsync(s->flag, &one, sizeof one, cudaMemcpyHostToDevice, h->stream));
        h->nl_valid = true;
    }
    return GX_OK;
}

// One tick of the list path up to and including the second kick; with
// `kpart` also the kinetic-energy partials (nb blocks) of the kicked v, and
// with `spart` (which needs kpart) its speed partials.
int nl_tick(gx_handle* h, const double* lambda, double* kpart, double* spart, int* nb_out, bool energy) {
    NlState* s = nl_of(h);
    const uint32_t n = (uint32_t)h->n;
    const GridGeom& g = s->lg;
    StateBuf& b = h->buf[h->cur];
    StateBuf& o = h->buf[h->cur ^ 1];
    const double half_dt = 0.5 * h->p.dt;
    const float lim = (float)(0.5 * s->skin_used * (1.0 - 1e-4));
    prof_begin(h, "nl_advance");
    GX_LAUNCH(h, k_nl_advance, nblk(n, 256), 256, b, n, lambda, half_dt, h->p.dt, 0.5 * h->p.box[0],
              0.5 * h->p.box[1], 0.5 * h->p.box[2], h->p.enable_boundaries ? 1 : 0, g, h->key_sorted, h->pos4, s->ref,
              lim * lim, s->flag, h->derr, s->half == 1 ? h->F : nullptr, h->cap);
    prof_end(h, "nl_advance");
    // inside a capture: the rebuild goes into the body of an IF node
    cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
    GX_CUDA(h, cudaStreamIsCapturing(h->stream, &cst));
    const bool cond = cst == cudaStreamCaptureStatusActive;
    cudaStream_t main_stream = h->stream;
    uint64_t body_l0 = 0;
    if (cond) {
        cudaStreamCaptureStatus st;
        unsigned long long id = 0;
        cudaGraph_t gr = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        GX_CUDA(h, cudaStreamGetCaptureInfo(h->stream, &st, &id, &gr, &deps, &nd));
        cudaGraphConditionalHandle hc;
        GX_CUDA(h, cudaGraphConditionalHandleCreate(&hc, gr, 0, cudaGraphCondAssignDefault));
        GX_LAUNCH(h, k_nl_set_cond, 1, 1, hc, s->flag);
        GX_CUDA(h, cudaStreamGetCaptureInfo(h->stream, &st, &id, &gr, &deps, &nd));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = hc;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        GX_CUDA(h, cudaGraphAddNode(&node, gr, deps, nd, &cp));
        GX_CUDA(h, cudaStreamUpdateCaptureDependencies(h->stream, &node, 1, cudaStreamSetCaptureDependencies));
        GX_CUDA(h, cudaStreamBeginCaptureToGraph(s->side, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeRelaxed));
        h->stream = s->side;
        body_l0 = h->launches;
    }
    prof_begin(h, "nl_rebuild");
    auto rebuild = [&]() -> int {
        launch_cell_keys(h, g, b, n, h->key, s->flag);
        int r = counting_sort(h, s->cl, g.ncell, h->key, n, h->perm, s->flag);
        if (r) return r;
        launch_gather(h, b, o, h->perm, h->key, h->key_sorted, n, h->pos_of_slot, s->flag);
        prof_begin(h, "nl_copy");
        GX_LAUNCH(h, k_nl_copy, nblk(n, 256), 256, o, b, n, s->flag);
        prof_end(h, "nl_copy");
        prof_begin(h, "nl_stage");
        GX_LAUNCH(h, k_nl_stage, nblk(n, 256), 256, g, b, h->key_sorted, n, h->pos4, s->ref, s->flag);
        prof_end(h, "nl_stage");
        const float rl = (float)((h->fs.rc + s->skin_used) * (1.0 + 1e-6));
        prof_begin(h, "nl_build");
        if (h->kernel_variant == 8) {  // the brick build: candidates from the staged neighbourhood
            const uint32_t K = 8, nchunks = (g.n[0] + K - 1) / K;
            auto bb = s->half == 1 ? k_nl_build_brick<true, 2048> : k_nl_build_brick<false, 2048>;
            GX_LAUNCH(h, bb, nchunks * g.n[1] * g.n[2], kNlBuildThreads, g, h->pos4, h->key_sorted, s->cl.start,
                      rl * rl, s->list, s->cap, s->cap_nb, s->cnt, h->derr, K, nchunks, s->flag);
        } else {
            auto build = s->half == 1 ? k_nl_build<true> : k_nl_build<false>;
            GX_LAUNCH(h, build, nblk(n, kNlBuildThreads), kNlBuildThreads, g, h->pos4, h->key_sorted, s->cl.start,
                      n, rl * rl, s->list, s->cap, s->cap_nb, s->cnt, s->flag);
        }
        prof_end(h, "nl_build");
        return GX_OK;
    };
    int rc = rebuild();
    if (cond) {
        if (!rc) GX_LAUNCH(h, k_nl_body_done, 1, 1, s->flag);
        s->body_kernels = h->launches - body_l0;
        h->launches = body_l0;  // counted when the body runs (nl_rebuilds)
        cudaGraph_t body = nullptr;
        cudaError_t ce = cudaStreamEndCapture(s->side, &body);
        h->stream = main_stream;
        if (!rc && ce != cudaSuccess) rc = cuda_err(h, ce, "cudaStreamEndCapture (rebuild body)");
    }
    if (rc) return rc;
    GX_LAUNCH(h, k_nl_end, 1, 1, s->flag, h->p.enable_boundaries ? 1 : 0, h->dcount);
    prof_end(h, "nl_rebuild");
    // Positions and the slot map are final here (the pair pass, the spring,
    // the collision pass and the finish write only forces and velocities).
    if (h->io_events)
        GX_CUDA(h, cudaEventRecordWithFlags(h->io_ev[3], h->stream,
                                            cond ? cudaEventRecordExternal : cudaEventRecordDefault));
    const bool halfl = s->half == 1;
    const bool f64 = h->precision != GX_MIXED;
    LawF32 L = make_law32(h);
    prof_begin(h, "force_nl");
    if (f64) {
        double* vpart = h->red;  // row 0 of the block partials
        const double* psig = d_psig(h);
        const unsigned fb = nblk(n, kNlThreads);
        GX_LAUNCH(h, k_nl_force64, fb, kNlThreads, g, b, h->key_sorted, s->cl.start, n, make_law64(h), psig,
                  psig + kNElem * kNElem, s->list, s->cap, s->cap_nb, s->cnt, vpart, h->dcount + 0);
        launch_sum_rows(h, vpart, (int)fb, h->dscal + 2);
    } else if (halfl) {
        launch_nl_force<true>(h, s->tpp, g, s, n, L, energy);
    } else {
        launch_nl_force<false>(h, s->tpp, g, s, n, L, energy);
    }
    prof_end(h, "force_nl");
    const bool spring = bonds_on(h);
    if (spring && !f64) GX_LAUNCH(h, k_nl_fix_to_double, 1, 1, h->dcount + 1, h->dscal + 2, h->dscal + 3);
    if (spring && (rc = bond_spring(h, true))) return rc;  // into F before it becomes a
    if (h->p.enable_collisions && (rc = collide_pass(h))) return rc;  // CollisionSystem, before the second kick
    int nb = (int)nblk(n, kRedThreads);
    if (nb > 1184) nb = 1184;  // the block count of launch_kinetic
    if (nb < 1) nb = 1;
    prof_begin(h, "nl_finish");
    const unsigned long long* vsum = spring ? nullptr : h->dcount + 1;
    const int mode = kpart ? (spart ? 2 : 1) : 0;
    if (f64) {
        auto k = mode == 2 ? k_nl_finish64<2> : (mode == 1 ? k_nl_finish64<1> : k_nl_finish64<0>);
        GX_LAUNCH(h, k, nb, kRedThreads, b, n, half_dt, kpart, spart);
        if (!spring) GX_CUDA(h, cudaMemsetAsync(h->dscal + 3, 0, sizeof(double), h->stream));
    } else {
        auto k = mode == 2 ? k_nl_finish<2> : (mode == 1 ? k_nl_finish<1> : k_nl_finish<0>);
        GX_LAUNCH(h, k, nb, kRedThreads, b, h->F, h->cap, n, half_dt, kpart, spart, vsum, h->dscal + 2, h->dscal + 3);
    }
    prof_end(h, "nl_finish");
    if (nb_out) *nb_out = nb;
    return GX_OK;
}

// Rebuilds performed so far (reads the device counter; synchronises).
int nl_rebuilds(gx_handle* h, uint64_t* out) {
    *out = 0;
    if (!h->nl) return GX_OK;
    NlState* s = static_cast<NlState*>(h->nl);
    if (!s->flag) return GX_OK;
    uint32_t f[4] = {0, 0, 0, 0};
    GX_CUDA(h, cudaMemcpyAsync(f, s->flag, sizeof f, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    *out = f[1];
    // the kernels of the captured rebuild bodies that ran since the last read
    h->launches += (uint64_t)(f[3] - s->body_runs_seen) * s->body_kernels;
    s->body_runs_seen = f[3];
    return GX_OK;
}

// Times the list pass at 1, 2, 4 and 8 threads per atom on the current list
// (the best of three rounds of at least `reps` launches each) and keeps the
// fastest.  The state is not touched:
// the pass only writes the force scratch, which the next tick overwrites.
int nl_tune_tpp(gx_handle* h, int reps) {
    int rs = settle_step_errors(h);  // the error word is cleared after the timing below
    if (rs) return rs;
    NlState* s = nl_of(h);
    if (!s->list || !s->cap || h->n == 0) return GX_OK;
    const uint32_t n = (uint32_t)h->n;
    const LawF32 L = make_law32(h);
    // variant 7: the stash size (8 or 16 slots per thread); variant 8: the
    // brick length (4 or 8 cells); else threads per atom, and with one lane
    // per atom on the half list the block of the shared far-end sums (256,
    // 128 or none)
    const bool stash = h->kernel_variant == 7, brick = h->kernel_variant == 8;
    struct Cand {
        int tpp, block;
    };
    const Cand lanes[6] = {{1, 256}, {1, 128}, {1, 0}, {2, 0}, {4, 0}, {8, 0}};
    const int ncand = (stash || brick) ? 2 : (s->half == 1 ? 6 : 4);
    double best = 1e300;
    const int tpp0 = s->tpp, block0 = s->block;
    int pick = 0;
    int launches = reps;
    for (int k = 0; k < ncand; ++k) {
        int tpp = s->tpp;
        if (stash) s->slots = k == 0 ? 8 : 16;
        else if (brick) s->brick = k;
        else if (s->half == 1) {
            tpp = lanes[k].tpp;
            s->block = lanes[k].block;
        } else {
            tpp = lanes[k + 2].tpp;
        }
        // the best of three rounds of `launches` passes; a short pass (a
        // small system) gets enough launches for ~1 ms per round, so that
        // the event resolution and launch jitter do not decide the pick
        double t_min = 1e300;
        int rc = 0;
        for (int round = 0; round < 3 && !rc; ++round) {
            rc = gx_timer_mark(h, 14);
            for (int r = 0; r < launches && !rc; ++r) {
                if (s->half == 1) launch_nl_force<true>(h, tpp, s->lg, s, n, L, false);
                else launch_nl_force<false>(h, tpp, s->lg, s, n, L, false);
            }
            double t = 0.0;
            if (!rc) rc = gx_timer_mark(h, 15);
            if (!rc) rc = gx_timer_elapsed(h, 14, 15, &t);
            if (!rc && launches == reps && k == 0 && round == 0 && t < 1.0)
                launches = (int)std::min(200.0, std::ceil(reps * 1.0 / std::max(t, 1e-3)));
            else if (!rc)
                t_min = std::min(t_min, t / launches);
        }
        if (rc) {
            s->tpp = tpp0;
            s->block = block0;
            return rc;
        }
        if (t_min < best) {
            best = t_min;
            pick = k;
        }
    }
    if (stash) s->slots = pick == 0 ? 8 : 16;
    else if (brick) s->brick = pick;
    else if (s->half == 1) {
        s->tpp = lanes[pick].tpp;
        s->block = lanes[pick].block;
    } else {
        s->tpp = lanes[pick + 2].tpp;
        s->block = block0;
    }
    GX_CUDA(h, cudaMemsetAsync(h->derr, 0, sizeof(uint32_t), h->stream));
    return GX_OK;
}

__global__ void k_nl_stats(const uint32_t* __restrict__ cnt, uint32_t n, int cap_nb,
                           unsigned long long* __restrict__ out) {
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

// Entries held by the current list (an overflowed atom counts the entries it
// found) and atoms whose list overflowed; synchronises the stream.
int nl_stats(gx_handle* h, uint64_t* entries, uint64_t* overflowed) {
    *entries = 0;
    *overflowed = 0;
    NlState* s = h->nl ? static_cast<NlState*>(h->nl) : nullptr;
    if (!s || !s->cnt || !h->nl_valid || !h->n) return GX_OK;
    unsigned long long* d = h->dcount + 12;  // two scratch counters outside the tick's slots
    GX_CUDA(h, cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), h->stream));
    GX_LAUNCH(h, k_nl_stats, 256, 256, s->cnt, (uint32_t)h->n, s->cap_nb, d);
    unsigned long long v[2] = {0, 0};
    GX_CUDA(h, cudaMemcpyAsync(v, d, sizeof v, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    *entries = v[0];
    *overflowed = v[1];
    return GX_OK;
}

int nl_config(gx_handle* h, double* skin, int* tpp) {
    NlState* s = nl_of(h);
    if (skin) *skin = skin_of(h, s);
    if (tpp) *tpp = s->tpp;
    return GX_OK;
}

int nl_shape(gx_handle* h, int* tpp, int* block, int* stash, int* brick) {
    const NlState* s = nl_of(h);
    *tpp = s->tpp;
    *block = s->block;
    *stash = s->slots;
    *brick = s->brick == 0 ? 4 : 8;
    return GX_OK;
}

int nl_set_brick(gx_handle* h, int cells) {
    if (cells != 4 && cells != 8) return set_err(h, GX_ERR_ARG, "brick length must be 4 or 8 cells");
    nl_of(h)->brick = cells == 4 ? 0 : 1;
    return GX_OK;
}

int nl_set_block(gx_handle* h, int block) {
    if (block != 0 && block != 128 && block != 256)
        return set_err(h, GX_ERR_ARG, "list block must be 0 (far ends in global memory), 128 or 256");
    nl_of(h)->block = block;
    return GX_OK;
}

int nl_set_slots(gx_handle* h, int slots) {
    if (slots != 8 && slots != 16) return set_err(h, GX_ERR_ARG, "stash slots must be 8 or 16");
    nl_of(h)->slots = slots;
    return GX_OK;
}

int nl_set_tpp(gx_handle* h, int tpp) {
    if (tpp != 1 && tpp != 2 && tpp != 4 && tpp != 8) return set_err(h, GX_ERR_ARG, "threads per atom must be 1, 2, 4 or 8");
    nl_of(h)->tpp = tpp;
    return GX_OK;
}

int nl_set_skin(gx_handle* h, double skin) {
    NlState* s = nl_of(h);
    s->skin = skin;
    h->nl_valid = false;
    return GX_OK;
}

bool nl_view(const gx_handle* h, NlView* v) {
    const NlState* s = static_cast<const NlState*>(h->nl);
    if (!s || !h->nl_valid || !h->nl_fresh || !s->list || !s->cnt || s->cap < h->n) return false;
    v->list = s->list;
    v->stride = s->cap;
    v->cap_nb = s->cap_nb;
    v->cnt = s->cnt;
    v->lg = s->lg;
    v->start = s->cl.start;
    v->home = h->key_sorted;
    v->idx_mask = kIdxMask;
    return true;
}

}  // namespace gx
