// gx_batch_flat.cu -- a gx_batch advanced as one concatenated system (batch
// mode 2).
//
// The persistent mode (gx_batch.cu) gives every replica one CTA, so a sweep
// whose replicas differ 30-fold in size runs for as long as its largest
// replica takes on a single SM.  Here each phase of the tick is one kernel
// over the atoms of ALL replicas, spread over the whole GPU; a replica is
// only a range of atoms, a range of cells in one global cell index
// (cell_base[r] + local cell) and a row of the geometry table:
//
//   k_fb_advance  kick (pending Berendsen scale of the atom's replica),
//                 drift, wrap, global cell key
//   [sort]        counting sort of all atoms by global cell (the shared
//                 deterministic counting_sort)
//   k_fb_stage    FP32 cell-local positions in sorted order, zero forces
//   k_fb_force    one thread per atom over its replica's canonical half
//                 shell, pair_f32, int64 fixed-point sums (k_force_mixed's
//                 arithmetic), potential and pair count per replica on
//                 the tick that reports them
//   k_fb_finish   a = F 2^-32 / m, second kick
//   k_fb_thermo   one block per replica: kinetic energy in a fixed order,
//                 the replica's Berendsen lambda (thermostat.rs:52-71)
// One tick is captured once as a CUDA graph in two forms, with and without
// the potential and pair count; a step call replays the quiet form and ends
// with the reporting one (the forces are the same bits).  At the end of a
// step call the pending scales are applied (k_fb_commit), as the persistent
// mode does.  Every operation on a replica's atoms is the single-universe
// mixed path's, so an NVE replica reproduces gx_step (pair-pass variants
// 1-4) bit for bit.
#include <cmath>
#include <cstring>
#include <vector>

#include "gx_batch.cuh"

namespace gx {

struct RepGeo {
    double L[3], cell[3], half_box[3];
    float cellf[3], Lf[3], invLf[3];
    uint32_t n[3];
    uint32_t cell_base;
    int minimg_mask, nhalf;
    int8_t half[13][3];
};

struct BatchFlat {
    size_t cap = 0;
    int nrep = 0;
    uint32_t ncell = 0;
    RepGeo* geo = nullptr;
    RepThermo* th = nullptr;
    uint32_t* rep_of = nullptr;         // replica of each atom (concatenated order)
    uint32_t* srep = nullptr;           // replica of each sorted position
    double* lam = nullptr;              // pending Berendsen scale per replica
    unsigned long long* acc = nullptr;  // [2 nrep]: fixed-point V, pair count
    gx_handle* ctx = nullptr;           // launch context of the shared counting sort
    cudaGraphExec_t graph[2] = {};      // tick without / with the potential and pair count
    uint64_t graph_kernels = 0;
    unsigned* coop_bar = nullptr;       // mode 3: grid barrier (arrivals, generation), force chunk counters (2)
    uint32_t* coop_tile = nullptr;      // mode 3: scan tile totals
    int coop_grid = 0;
};

void batch_flat_free(BatchFlat* f) {
    if (!f) return;
    for (cudaGraphExec_t g : f->graph)
        if (g) cudaGraphExecDestroy(g);
    cudaFree(f->geo);
    cudaFree(f->th);
    cudaFree(f->rep_of);
    cudaFree(f->srep);
    cudaFree(f->lam);
    cudaFree(f->acc);
    cudaFree(f->coop_bar);
    cudaFree(f->coop_tile);
    if (f->ctx) {
        cells_free(f->ctx->cl);
        f->ctx->stream = nullptr;  // owned by the batch
        delete f->ctx;
    }
    delete f;
}

namespace {

constexpr int kFbThreads = 128;
constexpr int kFbRed = 256;

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ __forceinline__ uint32_t cell_of_rep(const RepGeo& G, double x, double y, double z) {
    uint32_t ix = axis_cell(x, G.L[0], G.cell[0], G.n[0]);
    uint32_t iy = axis_cell(y, G.L[1], G.cell[1], G.n[1]);
    uint32_t iz = axis_cell(z, G.L[2], G.cell[2], G.n[2]);
    return ix + G.n[0] * (iy + G.n[1] * iz);
}

// Kick (k_kick with the replica's scale), drift (k_drift), wrap (k_wrap),
// global cell key.
__device__ __forceinline__ void fb_advance_one(uint32_t i, const RepGeo* __restrict__ geo,
                                               const uint32_t* __restrict__ rep_of, const BatchArrays& A,
                                               const double* __restrict__ lam, double half_dt, double dt, int wrap,
                                               uint32_t* __restrict__ key, uint32_t* __restrict__ err) {
    const uint32_t r = rep_of[i];
    const RepGeo& G = geo[r];
    const double l = lam[r];
    double vx = xadd(xmul(A.vx[i], l), xmul(A.ax[i], half_dt));
    double vy = xadd(xmul(A.vy[i], l), xmul(A.ay[i], half_dt));
    double vz = xadd(xmul(A.vz[i], l), xmul(A.az[i], half_dt));
    double x = xadd(A.x[i], xmul(vx, dt)), y = xadd(A.y[i], xmul(vy, dt)), z = xadd(A.z[i], xmul(vz, dt));
    if (wrap) {
        x = xsub(rem_euclid(x, xmul(2.0, G.half_box[0])), G.half_box[0]);
        y = xsub(rem_euclid(y, xmul(2.0, G.half_box[1])), G.half_box[1]);
        z = xsub(rem_euclid(z, xmul(2.0, G.half_box[2])), G.half_box[2]);
    }
    A.vx[i] = vx;
    A.vy[i] = vy;
    A.vz[i] = vz;
    A.x[i] = x;
    A.y[i] = y;
    A.z[i] = z;
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) atomicOr(err, kErrNonFinite);
    key[i] = G.cell_base + cell_of_rep(G, x, y, z);
}

__global__ void k_fb_advance(const RepGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of, BatchArrays A,
                             const double* __restrict__ lam, double half_dt, double dt, int wrap, uint32_t total,
                             uint32_t* __restrict__ key, uint32_t* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < total) fb_advance_one(i, geo, rep_of, A, lam, half_dt, dt, wrap, key, err);
}

// Sorted staging: cell-local FP32 position + kind (as k_build_pos4), the
// local cell and replica of each sorted position, zeroed forces.
__device__ __forceinline__ void fb_stage_one(uint32_t s, const RepGeo* __restrict__ geo,
                                             const uint32_t* __restrict__ rep_of, const BatchArrays& A,
                                             const uint32_t* __restrict__ perm, const uint32_t* __restrict__ key,
                                             uint32_t* __restrict__ srep, size_t fstride) {
    const uint32_t i = perm[s], r = rep_of[i];
    const RepGeo& G = geo[r];
    const uint32_t c = key[i] - G.cell_base;
    const uint32_t nxny = G.n[0] * G.n[1];
    const uint32_t iz = c / nxny, rem = c - iz * nxny, iy = rem / G.n[0], ix = rem - iy * G.n[0];
    double ux = cell_local(A.x[i], G.L[0], G.cell[0], ix);
    double uy = cell_local(A.y[i], G.L[1], G.cell[1], iy);
    double uz = cell_local(A.z[i], G.L[2], G.cell[2], iz);
    A.pos4[s] = make_float4((float)ux, (float)uy, (float)uz, __int_as_float((int)A.kind[i]));
    A.skey[s] = c;
    srep[s] = r;
    A.F[s] = 0;
    A.F[fstride + s] = 0;
    A.F[2 * fstride + s] = 0;
}

__global__ void k_fb_stage(const RepGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of, BatchArrays A,
                           const uint32_t* __restrict__ perm, const uint32_t* __restrict__ key, uint32_t total,
                           uint32_t* __restrict__ srep, size_t fstride) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < total) fb_stage_one(s, geo, rep_of, A, perm, key, srep, fstride);
}

// k_force_mixed on the atom's own replica grid (canonical half shell, the
// same shifts, minimum image on axes with fewer than 3 cells).  Every lane of
// the warp calls it (s >= total: no atom), for the warp-level sums.
template <bool ENERGY>
__device__ __forceinline__ void fb_force_one(uint32_t s, const RepGeo* __restrict__ geo,
                                             const float4* __restrict__ pos4, const uint32_t* __restrict__ skey,
                                             const uint32_t* __restrict__ srep, const uint32_t* __restrict__ start,
                                             uint32_t total, const LawF32& L, const PairF* st,
                                             long long* __restrict__ F, size_t fstride,
                                             unsigned long long* __restrict__ racc, uint32_t* __restrict__ err) {
    long long vq = 0;
    unsigned long long np = 0;
    uint32_t r = 0xFFFFFFFFu;
    if (s < total) {
        r = srep[s];
        const RepGeo& G = geo[r];
        const uint32_t nx = G.n[0], ny = G.n[1], nz = G.n[2], cb = G.cell_base;
        const int mask = G.minimg_mask;
        float4 pi = pos4[s];
        int ki = __float_as_int(pi.w);
        const uint32_t c = skey[s];
        const uint32_t iz = c / (nx * ny), rem = c - iz * nx * ny, iy = rem / nx, ix = rem - iy * nx;
        long long fx = 0, fy = 0, fz = 0;
        for (int k = -1; k < G.nhalf; ++k) {
            uint32_t B, lo;
            float sx = 0.f, sy = 0.f, sz = 0.f;
            if (k < 0) {
                B = c;
                lo = s + 1;
            } else {
                int ox = G.half[k][0], oy = G.half[k][1], oz = G.half[k][2];
                B = wrap_add(ix, ox, nx) + nx * (wrap_add(iy, oy, ny) + ny * wrap_add(iz, oz, nz));
                lo = start[cb + B];
                sx = -(float)ox * G.cellf[0];
                sy = -(float)oy * G.cellf[1];
                sz = -(float)oz * G.cellf[2];
            }
            const uint32_t hi = start[cb + B + 1];
            for (uint32_t j = lo; j < hi; ++j) {
                float4 pj = pos4[j];
                float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
                if (mask) {
                    if (mask & 1) dx = fsub(dx, fmul(G.Lf[0], rintf(fmul(dx, G.invLf[0]))));
                    if (mask & 2) dy = fsub(dy, fmul(G.Lf[1], rintf(fmul(dy, G.invLf[1]))));
                    if (mask & 4) dz = fsub(dz, fmul(G.Lf[2], rintf(fmul(dz, G.invLf[2]))));
                }
                float d2 = dist2(dx, dy, dz);
                if (!(d2 < L.rc2) || d2 == 0.f) continue;
                float fs, v;
                pair_f32(L, st[ki * L.nkinds + __float_as_int(pj.w)], d2, fs, v);
                long long qx, qy, qz;
                quant3(fmul(dx, fs), fmul(dy, fs), fmul(dz, fs), qx, qy, qz, err);
                fx += qx;
                fy += qy;
                fz += qz;
                atomicAdd((unsigned long long*)&F[j], (unsigned long long)(-qx));
                atomicAdd((unsigned long long*)&F[fstride + j], (unsigned long long)(-qy));
                atomicAdd((unsigned long long*)&F[2 * fstride + j], (unsigned long long)(-qz));
                if (ENERGY) {
                    vq += quant(v, err);
                    ++np;
                }
            }
        }
        atomicAdd((unsigned long long*)&F[s], (unsigned long long)fx);
        atomicAdd((unsigned long long*)&F[fstride + s], (unsigned long long)fy);
        atomicAdd((unsigned long long*)&F[2 * fstride + s], (unsigned long long)fz);
    }
    if (!ENERGY) return;
    // per-replica potential and pair count: one atomic per warp when the
    // warp lies in one replica (the usual case), else one per lane
    const uint32_t r0 = __shfl_sync(0xffffffffu, r, 0);
    if (__all_sync(0xffffffffu, r == r0) && r0 != 0xFFFFFFFFu) {
        unsigned long long a = (unsigned long long)vq, b = np;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&racc[2 * r0], a);
            atomicAdd(&racc[2 * r0 + 1], b);
        }
    } else if (r != 0xFFFFFFFFu) {
        atomicAdd(&racc[2 * r], (unsigned long long)vq);
        atomicAdd(&racc[2 * r + 1], np);
    }
}

template <bool ENERGY>
__global__ void __launch_bounds__(kFbThreads) k_fb_force(const RepGeo* __restrict__ geo, const float4* __restrict__ pos4,
                                                          const uint32_t* __restrict__ skey,
                                                          const uint32_t* __restrict__ srep,
                                                          const uint32_t* __restrict__ start, uint32_t total, LawF32 L,
                                                          const PairF* __restrict__ tab, long long* __restrict__ F,
                                                          size_t fstride, unsigned long long* __restrict__ racc,
                                                          uint32_t* __restrict__ err) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    const int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kFbThreads) st[t] = tab[t];
    __syncthreads();
    fb_force_one<ENERGY>(blockIdx.x * kFbThreads + threadIdx.x, geo, pos4, skey, srep, start, total, L, st, F, fstride,
                         racc, err);
}

// a = F 2^-32 (1/m) (k_fix_to_acc), v += a dt/2 (k_kick).
__device__ __forceinline__ void fb_finish_one(uint32_t s, const BatchArrays& A, const uint32_t* __restrict__ perm,
                                              double half_dt, size_t fstride) {
    const uint32_t i = perm[s];
    const double im = A.inv_mass[i];
    double ax = xmul(xmul(__ll2double_rn(A.F[s]), kFixInv), im);
    double ay = xmul(xmul(__ll2double_rn(A.F[fstride + s]), kFixInv), im);
    double az = xmul(xmul(__ll2double_rn(A.F[2 * fstride + s]), kFixInv), im);
    A.ax[i] = ax;
    A.ay[i] = ay;
    A.az[i] = az;
    A.vx[i] = xadd(A.vx[i], xmul(ax, half_dt));
    A.vy[i] = xadd(A.vy[i], xmul(ay, half_dt));
    A.vz[i] = xadd(A.vz[i], xmul(az, half_dt));
}

__global__ void k_fb_finish(BatchArrays A, const uint32_t* __restrict__ perm, uint32_t total, double half_dt,
                            size_t fstride) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < total) fb_finish_one(s, A, perm, half_dt, fstride);
}

__device__ __forceinline__ double block_sum_fb(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kFbRed / 32; ++k) t = xadd(t, sh[k]);
    __syncthreads();
    return t;  // valid in thread 0
}

// One block per replica: kinetic energy of its atoms in a fixed order and
// the Berendsen scale of ThermostatSystem::run (thermostat.rs:52-71), kept
// pending for the next kick; the tick's V, lambda and pair count to out.
__device__ __forceinline__ void fb_thermo_one(int r, const RepThermo* __restrict__ th, const BatchArrays& A,
                                              double* __restrict__ lam, unsigned long long* __restrict__ racc,
                                              double k_thermal, double* __restrict__ out, double* sh) {
    const RepThermo T = th[r];
    double ks = 0.0;
    for (uint32_t i = T.base + threadIdx.x; i < T.base + T.n; i += kFbRed) {
        double vx = A.vx[i], vy = A.vy[i], vz = A.vz[i];
        double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
        ks = xadd(ks, xmul(xmul(0.5, A.mass[i]), l2));
    }
    ks = block_sum_fb(ks, sh);
    if (threadIdx.x == 0) {
        double l = 1.0;
        if (T.thermo && T.n > 0) {
            double t = xdiv(xmul(2.0 / 3.0, xdiv(ks, (double)T.n)), k_thermal);
            if (isfinite(t) && t > 0.0) {
                double l2 = xadd(1.0, xmul(xdiv(1.0, T.tau), xsub(xdiv(T.target, t), 1.0)));
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
}

__global__ void __launch_bounds__(kFbRed) k_fb_thermo(const RepThermo* __restrict__ th, BatchArrays A,
                                                      double* __restrict__ lam, unsigned long long* __restrict__ racc,
                                                      double k_thermal, double* __restrict__ out) {
    __shared__ double sh[kFbRed / 32];
    fb_thermo_one(blockIdx.x, th, A, lam, racc, k_thermal, out, sh);
}

// End of a step call: apply the pending scales, kinetic energy after them.
__device__ __forceinline__ void fb_commit_one(int r, const RepThermo* __restrict__ th, const BatchArrays& A,
                                              double* __restrict__ lam, double* __restrict__ out, double* sh) {
    const RepThermo T = th[r];
    const double l = lam[r];
    double ks = 0.0;
    for (uint32_t i = T.base + threadIdx.x; i < T.base + T.n; i += kFbRed) {
        double vx = xmul(A.vx[i], l), vy = xmul(A.vy[i], l), vz = xmul(A.vz[i], l);
        A.vx[i] = vx;
        A.vy[i] = vy;
        A.vz[i] = vz;
        double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
        ks = xadd(ks, xmul(xmul(0.5, A.mass[i]), l2));
    }
    ks = block_sum_fb(ks, sh);
    if (threadIdx.x == 0) {
        out[4 * r + 0] = ks;
        lam[r] = 1.0;
    }
}

__global__ void __launch_bounds__(kFbRed) k_fb_commit(const RepThermo* __restrict__ th, BatchArrays A,
                                                      double* __restrict__ lam, double* __restrict__ out) {
    __shared__ double sh[kFbRed / 32];
    fb_commit_one(blockIdx.x, th, A, lam, out, sh);
}

// ---------------------------------------------------------------------------
// Batch mode 3: the same phases inside ONE persistent cooperative launch for
// all the ticks of a step call.  Every block of the grid is resident (the
// grid is sized from the occupancy and launched cooperatively), and the
// phases are separated by a grid barrier with a bounded wait: a block that
// waits longer than about two seconds sets kErrTimeout and every block
// leaves at its next barrier.  The counting sort is done in place (cell
// counts fused into the advance phase, a tiled scan, the scatter and the
// per-cell ranking of the shared counting_sort), and the other phases
// call the functions of the kernels above, so a tick is the same bits as a
// mode-2 tick.  The block size is kFbRed, as the per-replica reductions of
// k_fb_thermo and k_fb_commit need the same thread mapping.
constexpr int kCoopThreads = kFbRed;
constexpr int kCoopItems = 16;
constexpr uint32_t kCoopTile = kCoopThreads * kCoopItems;  // counters per scan tile
constexpr unsigned long long kCoopSpins = 20000000ull;     // x ~100 ns sleeps: the barrier's wait limit

struct CoopArgs {
    const RepGeo* geo;
    const RepThermo* th;
    const uint32_t* rep_of;
    uint32_t* srep;
    double* lam;
    unsigned long long* racc;
    BatchArrays A;
    LawF32 L;
    const PairF* tab;
    double* out;
    uint32_t* err;
    uint32_t *count, *start, *fill, *tile, *tmp;
    unsigned* bar;  // [0] arrivals, [1] generation, [2 + tick parity] next force chunk
    uint32_t ncell, total;
    int nrep;
    BatchParams P;
};

// Grid barrier: arrive, then wait (bounded) for the last arrival to advance
// the generation.  Returns false on every block once any block timed out.
__device__ __forceinline__ bool coop_sync(const CoopArgs& a, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = a.bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(a.bar, 1u) == gridDim.x - 1) {
            atomicExch(a.bar, 0u);
            __threadfence();
            atomicAdd(a.bar + 1, 1u);
        } else {
            unsigned long long spins = 0;
            while (*gen == g) {
                if (++spins > kCoopSpins || (*(volatile uint32_t*)a.err & kErrTimeout)) {
                    atomicOr(a.err, kErrTimeout);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        *s_ok = (*(volatile uint32_t*)a.err & kErrTimeout) == 0u;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Exclusive scan of one tile of cell counts into start; the tile's total to tile[t].
__device__ __forceinline__ void coop_scan_tile(const CoopArgs& a, uint32_t t, uint32_t m, uint32_t* s_warp) {
    const uint32_t base = t * kCoopTile + threadIdx.x * kCoopItems;
    uint32_t v[kCoopItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kCoopItems; ++k) {
        v[k] = base + k < m ? a.count[base + k] : 0u;
        local += v[k];
    }
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += u;
    }
    if (lane == 31) s_warp[w] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int k = 0; k < kCoopThreads / 32; ++k) {
            const uint32_t x = s_warp[k];
            s_warp[k] = run;
            run += x;
        }
        a.tile[t] = run;
    }
    __syncthreads();
    uint32_t run = s_warp[w] + inc - local;
#pragma unroll
    for (int k = 0; k < kCoopItems; ++k) {
        if (base + k < m) a.start[base + k] = run;
        run += v[k];
    }
    __syncthreads();  // s_warp is reused by the next tile
}

// Exclusive scan of the tile totals in place (block 0), 256 at a time.
__device__ __forceinline__ void coop_scan_tiles(const CoopArgs& a, uint32_t ntiles, uint32_t* s_warp) {
    uint32_t carry = 0;
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t c0 = 0; c0 < ntiles; c0 += kCoopThreads) {
        const uint32_t t = c0 + threadIdx.x;
        const uint32_t x = t < ntiles ? a.tile[t] : 0u;
        uint32_t inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += u;
        }
        if (lane == 31) s_warp[w] = inc;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (int k = 0; k < kCoopThreads / 32; ++k) {
                const uint32_t y = s_warp[k];
                s_warp[k] = run;
                run += y;
            }
            s_warp[kCoopThreads / 32] = run;
        }
        __syncthreads();
        if (t < ntiles) a.tile[t] = carry + s_warp[w] + inc - x;
        carry += s_warp[kCoopThreads / 32];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kCoopThreads) k_fb_coop(CoopArgs a) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ double sh[kCoopThreads / 32];
    __shared__ uint32_t s_warp[kCoopThreads / 32 + 1];
    __shared__ int s_ok;
    const int nk2 = a.L.nkinds * a.L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kCoopThreads) st[t] = a.tab[t];
    const uint32_t gt = blockIdx.x * kCoopThreads + threadIdx.x, gs = gridDim.x * kCoopThreads;
    const uint32_t n = a.total, m = a.ncell + 1;
    const uint32_t ntiles = (m + kCoopTile - 1) / kCoopTile;
    const uint32_t npad = (n + 31u) & ~31u;
    const size_t fs = a.A.total;
    const BatchArrays& A = a.A;
    for (uint32_t c = gt; c < m; c += gs) {
        a.count[c] = 0u;
        a.fill[c] = 0u;
    }
    if (!coop_sync(a, &s_ok)) return;
    for (int step = 0; step < a.P.nsteps; ++step) {
        const bool energy = step == a.P.nsteps - 1;  // only the last tick reports V and the pair count
        for (uint32_t i = gt; i < n; i += gs) {      // k_fb_advance + k_count
            fb_advance_one(i, a.geo, a.rep_of, A, a.lam, a.P.half_dt, a.P.dt, a.P.boundaries, A.key, a.err);
            atomicAdd(&a.count[A.key[i]], 1u);
        }
        if (!coop_sync(a, &s_ok)) return;
        for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) coop_scan_tile(a, t, m, s_warp);
        if (!coop_sync(a, &s_ok)) return;
        if (blockIdx.x == 0) coop_scan_tiles(a, ntiles, s_warp);
        if (!coop_sync(a, &s_ok)) return;
        for (uint32_t c = gt; c < m; c += gs) a.start[c] += a.tile[c / kCoopTile];
        if (!coop_sync(a, &s_ok)) return;
        for (uint32_t i = gt; i < n; i += gs) {  // k_scatter
            const uint32_t c = A.key[i];
            a.tmp[a.start[c] + atomicAdd(&a.fill[c], 1u)] = i;
        }
        if (!coop_sync(a, &s_ok)) return;
        for (uint32_t i = gt; i < n; i += gs) {  // k_rank: ascending source order within each cell
            const uint32_t c = A.key[i];
            const uint32_t lo = a.start[c], hi = a.start[c + 1];
            uint32_t r = 0;
            for (uint32_t q = lo; q < hi; ++q) r += a.tmp[q] < i ? 1u : 0u;
            A.idx[lo + r] = i;
        }
        if (!coop_sync(a, &s_ok)) return;
        for (uint32_t s2 = gt; s2 < n; s2 += gs) fb_stage_one(s2, a.geo, a.rep_of, A, A.idx, A.key, a.srep, fs);
        if (!coop_sync(a, &s_ok)) return;
        {  // the pair pass: warps take 32-atom chunks from a counter, as a chunk's
           // cost follows the local density (a static split waits for the densest)
            unsigned* next = a.bar + 2 + (step & 1);
            for (;;) {
                uint32_t base = 0;
                if ((threadIdx.x & 31) == 0) base = atomicAdd(next, 32u);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= npad) break;
                const uint32_t s2 = base + (threadIdx.x & 31);
                if (energy)
                    fb_force_one<true>(s2, a.geo, A.pos4, A.skey, a.srep, a.start, n, a.L, st, A.F, fs, a.racc, a.err);
                else
                    fb_force_one<false>(s2, a.geo, A.pos4, A.skey, a.srep, a.start, n, a.L, st, A.F, fs, a.racc,
                                        a.err);
            }
        }
        if (!coop_sync(a, &s_ok)) return;
        for (uint32_t s2 = gt; s2 < n; s2 += gs) fb_finish_one(s2, A, A.idx, a.P.half_dt, fs);
        if (!coop_sync(a, &s_ok)) return;
        for (int r = blockIdx.x; r < a.nrep; r += gridDim.x) fb_thermo_one(r, a.th, A, a.lam, a.racc, a.P.k_thermal, a.out, sh);
        for (uint32_t c = gt; c < m; c += gs) {  // the next tick's counters
            a.count[c] = 0u;
            a.fill[c] = 0u;
        }
        if (gt == 0) a.bar[2 + ((step + 1) & 1)] = 0u;  // last taken two ticks back, before several barriers
        if (!coop_sync(a, &s_ok)) return;
    }
    for (int r = blockIdx.x; r < a.nrep; r += gridDim.x) fb_commit_one(r, a.th, A, a.lam, a.out, sh);
}

int ferr(gx_batch* b, int code, const std::string& m) {
    b->err = m;
    return code;
}
#define GXF_CUDA(b, call)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return ferr(b, GX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int flat_prepare(gx_batch* b) {
    if (b->flat && b->flat->cap == b->total && b->flat->nrep == b->nrep) return GX_OK;
    batch_flat_free(b->flat);
    b->flat = nullptr;
    BatchFlat* f = new BatchFlat();
    b->flat = f;
    f->cap = b->total;
    f->nrep = b->nrep;
    std::vector<RepGeo> geo(b->nrep);
    std::vector<RepThermo> th(b->nrep);
    std::vector<uint32_t> rep_of(b->total);
    uint32_t cells = 0;
    for (int r = 0; r < b->nrep; ++r) {
        const RepDesc& d = b->reps[r];
        RepGeo& G = geo[r];
        std::memset(&G, 0, sizeof G);
        for (int k = 0; k < 3; ++k) {
            G.L[k] = d.g.L[k];
            G.cell[k] = d.g.cell[k];
            G.half_box[k] = d.half_box[k];
            G.cellf[k] = d.g.cellf[k];
            G.Lf[k] = d.g.Lf[k];
            G.invLf[k] = d.g.invLf[k];
            G.n[k] = d.g.n[k];
        }
        G.cell_base = cells;
        G.minimg_mask = d.g.minimg_mask;
        G.nhalf = d.g.nhalf;
        std::memcpy(G.half, d.g.half, sizeof G.half);
        if ((uint64_t)cells + d.g.ncell > 0xFFFFFFF0ull) return ferr(b, GX_ERR_CAPACITY, "too many cells in the batch");
        cells += d.g.ncell;
        th[r] = RepThermo{d.base, d.n, d.target, d.tau, d.thermo};
        for (uint32_t i = 0; i < d.n; ++i) rep_of[d.base + i] = (uint32_t)r;
    }
    f->ncell = cells;
    const size_t cap = b->total < 1 ? 1 : b->total;
    GXF_CUDA(b, cudaMalloc(&f->geo, b->nrep * sizeof(RepGeo)));
    GXF_CUDA(b, cudaMalloc(&f->th, b->nrep * sizeof(RepThermo)));
    GXF_CUDA(b, cudaMalloc(&f->rep_of, cap * sizeof(uint32_t)));
    GXF_CUDA(b, cudaMalloc(&f->srep, cap * sizeof(uint32_t)));
    GXF_CUDA(b, cudaMalloc(&f->lam, b->nrep * sizeof(double)));
    GXF_CUDA(b, cudaMalloc(&f->acc, 2 * b->nrep * sizeof(unsigned long long)));
    GXF_CUDA(b, cudaMemcpy(f->geo, geo.data(), b->nrep * sizeof(RepGeo), cudaMemcpyHostToDevice));
    GXF_CUDA(b, cudaMemcpy(f->th, th.data(), b->nrep * sizeof(RepThermo), cudaMemcpyHostToDevice));
    if (b->total)
        GXF_CUDA(b, cudaMemcpy(f->rep_of, rep_of.data(), b->total * sizeof(uint32_t), cudaMemcpyHostToDevice));
    std::vector<double> ones(b->nrep, 1.0);
    GXF_CUDA(b, cudaMemcpy(f->lam, ones.data(), b->nrep * sizeof(double), cudaMemcpyHostToDevice));
    GXF_CUDA(b, cudaMemset(f->acc, 0, 2 * b->nrep * sizeof(unsigned long long)));
    f->ctx = new gx_handle();
    f->ctx->stream = b->stream;
    if (ensure_cells(f->ctx, f->ctx->cl, f->ncell)) return ferr(b, GX_ERR_OOM, f->ctx->err);
    if (ensure_sort_tmp(f->ctx, f->ctx->cl, b->total)) return ferr(b, GX_ERR_OOM, f->ctx->err);  // before capture
    return GX_OK;
}

// One tick, all replicas (launches only: capturable).  Without energy the
// force pass leaves the replicas' potential and pair count at zero: the
// forces are the same bits, and only the last tick of a step call reports.
int flat_tick(gx_batch* b, BatchParams P, bool energy) {
    BatchFlat* f = b->flat;
    gx_handle* h = f->ctx;
    const uint32_t n = (uint32_t)b->total;
    BatchArrays A = b->A;
    const size_t fs = A.total;
    GX_LAUNCH(h, k_fb_advance, nblk(n, 256), 256, f->geo, f->rep_of, A, f->lam, P.half_dt, P.dt, P.boundaries, n,
              A.key, b->d_err);
    int rc = counting_sort(h, h->cl, f->ncell, A.key, n, A.idx);
    if (rc) return ferr(b, rc, h->err);
    GX_LAUNCH(h, k_fb_stage, nblk(n, 256), 256, f->geo, f->rep_of, A, A.idx, A.key, n, f->srep, fs);
    if (energy)
        GX_LAUNCH(h, k_fb_force<true>, nblk(n, kFbThreads), kFbThreads, f->geo, A.pos4, A.skey, f->srep, h->cl.start,
                  n, b->L, b->d_tab, A.F, fs, f->acc, b->d_err);
    else
        GX_LAUNCH(h, k_fb_force<false>, nblk(n, kFbThreads), kFbThreads, f->geo, A.pos4, A.skey, f->srep,
                  h->cl.start, n, b->L, b->d_tab, A.F, fs, f->acc, b->d_err);
    GX_LAUNCH(h, k_fb_finish, nblk(n, 256), 256, A, A.idx, n, P.half_dt, fs);
    GX_LAUNCH(h, k_fb_thermo, b->nrep, kFbRed, f->th, A, f->lam, f->acc, P.k_thermal, b->d_out);
    return GX_OK;
}

}  // namespace

int flat_shared(gx_batch* b, FlatShared* out) {
    int rc = flat_prepare(b);
    if (rc) return rc;
    out->rep_of = b->flat->rep_of;
    out->th = b->flat->th;
    out->lam = b->flat->lam;
    out->acc = b->flat->acc;
    return GX_OK;
}

void flat_commit(gx_batch* b, gx_handle* h) {
    GX_LAUNCH(h, k_fb_commit, b->nrep, kFbRed, b->flat->th, b->A, b->flat->lam, b->d_out);
}

// Mode 3: nsteps ticks of every replica in one cooperative launch.
int batch_coop_step(gx_batch* b, int nsteps, uint64_t* launches) {
    int rc = flat_prepare(b);
    if (rc) return rc;
    if (launches) *launches = 0;
    if (!b->total || nsteps <= 0) return GX_OK;
    BatchFlat* f = b->flat;
    if (!f->coop_bar) {
        const uint32_t m = f->ncell + 1;
        const size_t ntiles = (m + kCoopTile - 1) / kCoopTile;
        GXF_CUDA(b, cudaMalloc(&f->coop_bar, 4 * sizeof(unsigned)));
        GXF_CUDA(b, cudaMalloc(&f->coop_tile, ntiles * sizeof(uint32_t)));
        int dev = 0, sms = 0, per_sm = 0, coop = 0;
        GXF_CUDA(b, cudaGetDevice(&dev));
        GXF_CUDA(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        GXF_CUDA(b, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        if (!coop) return ferr(b, GX_ERR_UNSUPPORTED, "the device does not support cooperative launches");
        GXF_CUDA(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fb_coop, kCoopThreads, 0));
        if (per_sm < 1) return ferr(b, GX_ERR_UNSUPPORTED, "the cooperative batch kernel does not fit on an SM");
        f->coop_grid = sms * per_sm;
    }
    GXF_CUDA(b, cudaMemsetAsync(f->coop_bar, 0, 4 * sizeof(unsigned), b->stream));
    CoopArgs a;
    a.geo = f->geo;
    a.th = f->th;
    a.rep_of = f->rep_of;
    a.srep = f->srep;
    a.lam = f->lam;
    a.racc = f->acc;
    a.A = b->A;
    a.L = b->L;
    a.tab = b->d_tab;
    a.out = b->d_out;
    a.err = b->d_err;
    a.count = f->ctx->cl.count;
    a.start = f->ctx->cl.start;
    a.fill = f->ctx->cl.fill;
    a.tmp = f->ctx->cl.tmp;
    a.tile = f->coop_tile;
    a.bar = f->coop_bar;
    a.ncell = f->ncell;
    a.total = (uint32_t)b->total;
    a.nrep = b->nrep;
    a.P.dt = b->p.dt;
    a.P.half_dt = 0.5 * b->p.dt;
    a.P.k_thermal = b->p.thermal_constant;
    a.P.boundaries = b->p.enable_boundaries ? 1 : 0;
    a.P.nsteps = nsteps;
    void* args[] = {&a};
    GXF_CUDA(b, cudaLaunchCooperativeKernel((const void*)k_fb_coop, dim3(f->coop_grid), dim3(kCoopThreads), args, 0,
                                            b->stream));
    if (launches) *launches = 1;
    return GX_OK;
}

// nsteps ticks of every replica as one system; device time between the
// events b->ev[0], b->ev[1] (recorded by the caller).
int batch_flat_step(gx_batch* b, int nsteps, uint64_t* launches) {
    int rc = flat_prepare(b);
    if (rc) return rc;
    BatchFlat* f = b->flat;
    BatchParams P;
    P.dt = b->p.dt;
    P.half_dt = 0.5 * b->p.dt;
    P.k_thermal = b->p.thermal_constant;
    P.boundaries = b->p.enable_boundaries ? 1 : 0;
    P.nsteps = nsteps;
    gx_handle* h = f->ctx;
    const uint64_t l0 = h->launches;
    if (!b->total) return GX_OK;
    for (int e = 0; e < 2; ++e) {
        if (f->graph[e]) continue;
        cudaGraph_t g = nullptr;
        GXF_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const uint64_t c0 = h->launches;
        int trc = flat_tick(b, P, e == 1);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (trc || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return trc ? trc : ferr(b, GX_ERR_CUDA, cudaGetErrorString(ce));
        }
        ce = cudaGraphInstantiate(&f->graph[e], g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return ferr(b, GX_ERR_CUDA, cudaGetErrorString(ce));
        f->graph_kernels = h->launches - c0;
        h->launches = c0;
    }
    for (int s = 0; s < nsteps; ++s) {
        GXF_CUDA(b, cudaGraphLaunch(f->graph[s == nsteps - 1], b->stream));
        h->launches += f->graph_kernels;
    }
    GX_LAUNCH(h, k_fb_commit, b->nrep, kFbRed, f->th, b->A, f->lam, b->d_out);
    GXF_CUDA(b, cudaGetLastError());
    if (launches) *launches = h->launches - l0;
    return GX_OK;
}

}  // namespace gx
