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

struct RepThermo {
    uint32_t base, n;
    double target, tau;
    int thermo;
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
    if (f->ctx) {
        cudaFree(f->ctx->cl.count);
        cudaFree(f->ctx->cl.start);
        cudaFree(f->ctx->cl.fill);
        for (auto q : f->ctx->cl.scan_levels) cudaFree(q);
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
__global__ void k_fb_advance(const RepGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of, BatchArrays A,
                             const double* __restrict__ lam, double half_dt, double dt, int wrap, uint32_t total,
                             uint32_t* __restrict__ key, uint32_t* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
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

// Sorted staging: cell-local FP32 position + kind (as k_build_pos4), the
// local cell and replica of each sorted position, zeroed forces.
__global__ void k_fb_stage(const RepGeo* __restrict__ geo, const uint32_t* __restrict__ rep_of, BatchArrays A,
                           const uint32_t* __restrict__ perm, const uint32_t* __restrict__ key, uint32_t total,
                           uint32_t* __restrict__ srep, size_t fstride) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
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

// k_force_mixed on the atom's own replica grid (canonical half shell, the
// same shifts, minimum image on axes with fewer than 3 cells).
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
    const uint32_t s = blockIdx.x * kFbThreads + threadIdx.x;
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
                long long qx = quant(fmul(dx, fs), err), qy = quant(fmul(dy, fs), err), qz = quant(fmul(dz, fs), err);
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

// a = F 2^-32 (1/m) (k_fix_to_acc), v += a dt/2 (k_kick).
__global__ void k_fb_finish(BatchArrays A, const uint32_t* __restrict__ perm, uint32_t total, double half_dt,
                            size_t fstride) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
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
__global__ void __launch_bounds__(kFbRed) k_fb_thermo(const RepThermo* __restrict__ th, BatchArrays A,
                                                      double* __restrict__ lam, unsigned long long* __restrict__ racc,
                                                      double k_thermal, double* __restrict__ out) {
    __shared__ double sh[kFbRed / 32];
    const int r = blockIdx.x;
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

// End of a step call: apply the pending scales, kinetic energy after them.
__global__ void __launch_bounds__(kFbRed) k_fb_commit(const RepThermo* __restrict__ th, BatchArrays A,
                                                      double* __restrict__ lam, double* __restrict__ out) {
    __shared__ double sh[kFbRed / 32];
    const int r = blockIdx.x;
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
