// gx_cells.cu -- cell assignment, counting sort by cell, SoA reorder, and the
// memory-bound integrator/thermostat kernels.
//
// Cell assignment follows SpatialGrid::cell_of (src/physics/grid.rs:228-246)
// bit for bit.  The reference keeps a per-cell linked list rebuilt every tick
// (grid.rs:99-113); here the same cell index drives a counting sort that
// reorders the SoA state so each cell's atoms are contiguous (cell_start[c],
// cell_start[c+1]) and a row of cells along x is one contiguous span.
#include "gx_internal.cuh"

namespace gx {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// `gate` (may be null): when it points at 0 the kernel does nothing, so a
// captured CUDA graph can carry a rebuild that runs only when requested.
__device__ __forceinline__ bool gated_off(const uint32_t* gate) { return gate && *gate == 0u; }

__global__ void k_count(const uint32_t* __restrict__ key, uint32_t n, uint32_t* __restrict__ count,
                        const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&count[key[i]], 1u);
}

// Exclusive scan of one tile of kScanTile elements; block total to sums.
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const uint32_t* in, uint32_t* out, uint32_t n,
                                                            uint32_t* sums, const uint32_t* __restrict__ gate) {
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    if (gated_off(gate)) return;
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        local += v[k];
    }
    // warp inclusive scan of thread totals
    uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += t;
    }
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
        uint32_t winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= (uint32_t)o) winc += t;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = winc - w;  // exclusive warp offsets
        if (lane == kScanThreads / 32 - 1 && sums) sums[blockIdx.x] = winc;
    }
    __syncthreads();
    uint32_t run = warp_tot[wid] + inc - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

__global__ void k_scan_add(uint32_t* out, uint32_t n, const uint32_t* offs, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / kScanTile];
}

__global__ void k_scatter(const uint32_t* __restrict__ key, uint32_t n, const uint32_t* __restrict__ start,
                          uint32_t* __restrict__ fill, uint32_t* __restrict__ perm,
                          const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c = key[i];
    perm[start[c] + atomicAdd(&fill[c], 1u)] = i;
}

// Makes the scatter deterministic: atom i goes to start[c] + (the number of
// atoms of its cell with a smaller index), so each cell lists its atoms in
// ascending source order.  One thread per atom reads its cell's segment of
// the scatter's order: a cell of k atoms costs k^2 reads spread over its k
// atoms, where a per-cell insertion sort ran them on one thread.
__global__ void k_rank(const uint32_t* __restrict__ key, uint32_t n, const uint32_t* __restrict__ start,
                       const uint32_t* __restrict__ scattered, uint32_t* __restrict__ perm,
                       const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = key[i];
    const uint32_t lo = start[c], hi = start[c + 1];
    uint32_t r = 0;
    for (uint32_t b = lo; b < hi; ++b) r += __ldg(scattered + b) < i ? 1u : 0u;
    perm[lo + r] = i;
}

__global__ void k_cell_keys(GridGeom g, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, uint32_t n, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ err, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double px = x[i], py = y[i], pz = z[i];
    if (!isfinite(px) || !isfinite(py) || !isfinite(pz)) atomicOr(err, kErrNonFinite);
    key[i] = cell_of(g, px, py, pz);
}

__global__ void k_gather(StateBuf s, StateBuf d, const uint32_t* __restrict__ perm,
                         const uint32_t* __restrict__ key_in, uint32_t* __restrict__ key_out, uint32_t n,
                         uint32_t* __restrict__ pos_of_slot, const uint32_t* __restrict__ gate) {
    if (gated_off(gate)) return;
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t q = perm[p];
    d.x[p] = s.x[q];
    d.y[p] = s.y[q];
    d.z[p] = s.z[q];
    d.vx[p] = s.vx[q];
    d.vy[p] = s.vy[q];
    d.vz[p] = s.vz[q];
    d.ax[p] = s.ax[q];
    d.ay[p] = s.ay[q];
    d.az[p] = s.az[q];
    d.charge[p] = s.charge[q];
    d.mass[p] = s.mass[q];
    d.inv_mass[p] = s.inv_mass[q];
    d.elem[p] = s.elem[q];
    d.kind[p] = s.kind[q];
    uint32_t sl = s.slot[q];
    d.slot[p] = sl;
    key_out[p] = key_in[q];
    pos_of_slot[sl] = p;
}

// Cell-local FP32 coordinates (u - i*cell, u as in cell_of) + kind in w.
__global__ void k_build_pos4(GridGeom g, StateBuf b, const uint32_t* __restrict__ key, uint32_t n,
                             float4* __restrict__ pos4) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t ix, iy, iz;
    decode(g, key[i], ix, iy, iz);
    double ux = cell_local(b.x[i], g.L[0], g.cell[0], ix);
    double uy = cell_local(b.y[i], g.L[1], g.cell[1], iy);
    double uz = cell_local(b.z[i], g.L[2], g.cell[2], iz);
    pos4[i] = make_float4((float)ux, (float)uy, (float)uz, __int_as_float((int)b.kind[i]));
}

// VelocityHalfKick (src/systems/integrate.rs:38-45), with the pending
// Berendsen scale of the previous tick applied first (thermostat.rs:68-70).
__global__ void k_kick(StateBuf b, uint32_t n, double half_dt, const double* __restrict__ lambda) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double vx = b.vx[i], vy = b.vy[i], vz = b.vz[i];
    if (lambda) {
        double l = *lambda;
        vx = xmul(vx, l);
        vy = xmul(vy, l);
        vz = xmul(vz, l);
    }
    b.vx[i] = xadd(vx, xmul(b.ax[i], half_dt));
    b.vy[i] = xadd(vy, xmul(b.ay[i], half_dt));
    b.vz[i] = xadd(vz, xmul(b.az[i], half_dt));
}

// PositionDrift (src/systems/integrate.rs:61-67).
__global__ void k_drift(StateBuf b, uint32_t n, double dt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    b.x[i] = xadd(b.x[i], xmul(b.vx[i], dt));
    b.y[i] = xadd(b.y[i], xmul(b.vy[i], dt));
    b.z[i] = xadd(b.z[i], xmul(b.vz[i], dt));
}

// BoundarySystem (src/systems/boundary.rs:22-35): x <- x.rem_euclid(2h) - h.
__global__ void k_wrap(StateBuf b, uint32_t n, double hx, double hy, double hz) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    b.x[i] = xsub(rem_euclid(b.x[i], xmul(2.0, hx)), hx);
    b.y[i] = xsub(rem_euclid(b.y[i], xmul(2.0, hy)), hy);
    b.z[i] = xsub(rem_euclid(b.z[i], xmul(2.0, hz)), hz);
}

__global__ void k_apply_lambda(StateBuf b, uint32_t n, const double* __restrict__ lambda) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double l = *lambda;
    b.vx[i] = xmul(b.vx[i], l);
    b.vy[i] = xmul(b.vy[i], l);
    b.vz[i] = xmul(b.vz[i], l);
}

__global__ void k_set_one(double* p) { *p = 1.0; }

template <int BS>
__device__ __forceinline__ double block_sum(double v, double* sh) {
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

constexpr int kRedThreads = 256;

// Kinetic energy 0.5*m*|v|^2 (thermostat.rs:52-57, aggregate.rs:86-93) and
// speed sums, optionally of lambda*v (the pending scale not yet stored).
// Grid-stride over a fixed number of blocks: deterministic for a given n.
__global__ void __launch_bounds__(kRedThreads) k_kinetic(StateBuf b, uint32_t n, const double* __restrict__ lambda,
                                                         double* __restrict__ kpart, double* __restrict__ spart) {
    __shared__ double sh[kRedThreads / 32];
    double l = lambda ? *lambda : 1.0;
    double ks = 0.0, ss = 0.0;
    for (uint32_t i = blockIdx.x * kRedThreads + threadIdx.x; i < n; i += gridDim.x * kRedThreads) {
        double vx = b.vx[i], vy = b.vy[i], vz = b.vz[i];
        if (lambda) {
            vx = xmul(vx, l);
            vy = xmul(vy, l);
            vz = xmul(vz, l);
        }
        double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
        ks = xadd(ks, xmul(xmul(0.5, b.mass[i]), l2));
        ss = xadd(ss, xsqrt(l2));
    }
    ks = block_sum<kRedThreads>(ks, sh);
    ss = block_sum<kRedThreads>(ss, sh);
    if (threadIdx.x == 0) {
        kpart[blockIdx.x] = ks;
        if (spart) spart[blockIdx.x] = ss;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_finalize_sum(const double* __restrict__ part, int nb, double* out) {
    __shared__ double sh[kRedThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += kRedThreads) s = xadd(s, part[i]);
    s = block_sum<kRedThreads>(s, sh);
    if (threadIdx.x == 0) *out = s;
}

// ThermostatSystem::run tail (src/systems/thermostat.rs:58-71): lambda from K.
__global__ void __launch_bounds__(kRedThreads) k_thermostat_lambda(const double* __restrict__ part, int nb, double k,
                                                                   double target, double tau, uint32_t n,
                                                                   double* lambda_out, double* K_out) {
    __shared__ double sh[kRedThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += kRedThreads) s = xadd(s, part[i]);
    s = block_sum<kRedThreads>(s, sh);
    if (threadIdx.x == 0) {
        double lam = 1.0;
        if (n > 0) {
            double t = xdiv(xmul(2.0 / 3.0, xdiv(s, (double)n)), k);
            if (isfinite(t) && t > 0.0) {
                double l2 = xadd(1.0, xmul(xdiv(1.0, tau), xsub(xdiv(target, t), 1.0)));
                lam = xsqrt(fmax(l2, 0.0));
            }
        }
        *lambda_out = lam;
        if (K_out) *K_out = s;
    }
}

inline unsigned nblk(uint32_t n, int bs) { return (n + bs - 1) / bs; }

}  // namespace

void cells_free(CellList& cl) {
    cudaFree(cl.count);
    cudaFree(cl.start);
    cudaFree(cl.fill);
    cudaFree(cl.tmp);
    for (auto p : cl.scan_levels) cudaFree(p);
    cl.count = cl.start = cl.fill = cl.tmp = nullptr;
    cl.scan_levels.clear();
    cl.scan_sizes.clear();
    cl.cap_cells = 0;
    cl.cap_tmp = 0;
}

int ensure_sort_tmp(gx_handle* h, CellList& cl, size_t n) {
    if (n <= cl.cap_tmp) return GX_OK;
    cudaFree(cl.tmp);
    cl.tmp = nullptr;
    cl.cap_tmp = 0;
    const size_t cap = n + n / 8 + 64;
    GX_CUDA(h, cudaMalloc(&cl.tmp, cap * sizeof(uint32_t)));
    cl.cap_tmp = cap;
    return GX_OK;
}

int ensure_cells(gx_handle* h, CellList& cl, uint32_t ncell) {
    if (ncell + 1 > cl.cap_cells) {
        cudaFree(cl.count);
        cudaFree(cl.start);
        cudaFree(cl.fill);
        for (auto p : cl.scan_levels) cudaFree(p);
        cl.scan_levels.clear();
        cl.scan_sizes.clear();
        size_t cap = (size_t)ncell + 1;
        cap += cap / 8 + 64;
        GX_CUDA(h, cudaMalloc(&cl.count, cap * sizeof(uint32_t)));
        GX_CUDA(h, cudaMalloc(&cl.start, cap * sizeof(uint32_t)));
        GX_CUDA(h, cudaMalloc(&cl.fill, cap * sizeof(uint32_t)));
        size_t m = cap;
        while (m > (size_t)kScanTile) {
            m = (m + kScanTile - 1) / kScanTile;
            uint32_t* p = nullptr;
            GX_CUDA(h, cudaMalloc(&p, (m + 1) * sizeof(uint32_t)));
            cl.scan_levels.push_back(p);
            cl.scan_sizes.push_back(m);
        }
        cl.cap_cells = cap;
    }
    return GX_OK;
}

static void scan_rec(gx_handle* h, CellList& cl, const uint32_t* in, uint32_t* out, uint32_t n, int level,
                     const uint32_t* gate) {
    unsigned nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1) {
        GX_LAUNCH(h, k_scan_tile, 1, kScanThreads, in, out, n, nullptr, gate);
        return;
    }
    uint32_t* sums = cl.scan_levels[level];
    GX_LAUNCH(h, k_scan_tile, nb, kScanThreads, in, out, n, sums, gate);
    scan_rec(h, cl, sums, sums, nb, level + 1, gate);
    GX_LAUNCH(h, k_scan_add, nblk(n, 256), 256, out, n, sums, gate);
}

// Exclusive scan of cl.count (ncell + 1 entries) into cl.start.
void cell_scan(gx_handle* h, CellList& cl, uint32_t ncell) {
    prof_begin(h, "cell_scan");
    scan_rec(h, cl, cl.count, cl.start, ncell + 1, 0, nullptr);
    prof_end(h, "cell_scan");
}

int counting_sort(gx_handle* h, CellList& cl, uint32_t ncell, const uint32_t* key, uint32_t n, uint32_t* perm,
                  const uint32_t* gate) {
    int rc = ensure_cells(h, cl, ncell);
    if (rc) return rc;
    prof_begin(h, "cell_count");
    GX_CUDA(h, cudaMemsetAsync(cl.count, 0, ((size_t)ncell + 1) * sizeof(uint32_t), h->stream));
    GX_CUDA(h, cudaMemsetAsync(cl.fill, 0, (size_t)ncell * sizeof(uint32_t), h->stream));
    if (n) GX_LAUNCH(h, k_count, nblk(n, 256), 256, key, n, cl.count, gate);
    prof_end(h, "cell_count");
    prof_begin(h, "cell_scan");
    scan_rec(h, cl, cl.count, cl.start, ncell + 1, 0, gate);
    prof_end(h, "cell_scan");
    if ((rc = ensure_sort_tmp(h, cl, n))) return rc;  // allocated before any capture by the callers that capture
    prof_begin(h, "cell_scatter");
    if (n) GX_LAUNCH(h, k_scatter, nblk(n, 256), 256, key, n, cl.start, cl.fill, cl.tmp, gate);
    prof_end(h, "cell_scatter");
    prof_begin(h, "cell_rank");
    if (n) GX_LAUNCH(h, k_rank, nblk(n, 256), 256, key, n, cl.start, cl.tmp, perm, gate);
    prof_end(h, "cell_rank");
    return GX_OK;
}

void launch_cell_keys(gx_handle* h, const GridGeom& g, const StateBuf& b, uint32_t n, uint32_t* key,
                      const uint32_t* gate) {
    if (!n) return;
    prof_begin(h, "cell_keys");
    GX_LAUNCH(h, k_cell_keys, nblk(n, 256), 256, g, b.x, b.y, b.z, n, key, h->derr, gate);
    prof_end(h, "cell_keys");
}

void launch_gather(gx_handle* h, const StateBuf& src, const StateBuf& dst, const uint32_t* perm,
                   const uint32_t* key_in, uint32_t* key_out, uint32_t n, uint32_t* pos_of_slot,
                   const uint32_t* gate) {
    if (!n) return;
    prof_begin(h, "reorder");
    GX_LAUNCH(h, k_gather, nblk(n, 256), 256, src, dst, perm, key_in, key_out, n, pos_of_slot, gate);
    prof_end(h, "reorder");
}

void launch_build_pos4(gx_handle* h, const GridGeom& g, const StateBuf& b, const uint32_t* key, uint32_t n,
                       float4* pos4) {
    if (!n) return;
    prof_begin(h, "stage_pos4");
    GX_LAUNCH(h, k_build_pos4, nblk(n, 256), 256, g, b, key, n, pos4);
    prof_end(h, "stage_pos4");
}

void launch_kick(gx_handle* h, const StateBuf& b, uint32_t n, double half_dt, const double* lambda) {
    if (!n) return;
    prof_begin(h, "kick");
    GX_LAUNCH(h, k_kick, nblk(n, 256), 256, b, n, half_dt, lambda);
    prof_end(h, "kick");
}
void launch_drift(gx_handle* h, const StateBuf& b, uint32_t n, double dt) {
    if (!n) return;
    prof_begin(h, "drift");
    GX_LAUNCH(h, k_drift, nblk(n, 256), 256, b, n, dt);
    prof_end(h, "drift");
}
void launch_wrap(gx_handle* h, const StateBuf& b, uint32_t n) {
    if (!n) return;
    prof_begin(h, "wrap");
    GX_LAUNCH(h, k_wrap, nblk(n, 256), 256, b, n, 0.5 * h->p.box[0], 0.5 * h->p.box[1], 0.5 * h->p.box[2]);
    prof_end(h, "wrap");
}
void launch_apply_lambda(gx_handle* h, const StateBuf& b, uint32_t n, double* lambda) {
    if (n) GX_LAUNCH(h, k_apply_lambda, nblk(n, 256), 256, b, n, lambda);
    GX_LAUNCH(h, k_set_one, 1, 1, lambda);
}
void launch_kinetic(gx_handle* h, const StateBuf& b, uint32_t n, const double* lambda, double* kpart,
                    double* spart, int* nblocks) {
    int nb = (int)nblk(n, kRedThreads);
    if (nb > 1184) nb = 1184;  // 8 x 148 SMs; fixed for a given n
    if (nb < 1) nb = 1;
    prof_begin(h, "kinetic");
    GX_LAUNCH(h, k_kinetic, nb, kRedThreads, b, n, lambda, kpart, spart);
    prof_end(h, "kinetic");
    *nblocks = nb;
}
void launch_finalize_sum(gx_handle* h, const double* partials, int nblocks, double* out) {
    GX_LAUNCH(h, k_finalize_sum, 1, kRedThreads, partials, nblocks, out);
}
void launch_thermostat_lambda(gx_handle* h, const double* partials, int nblocks, double k, double target,
                              double tau, uint32_t n, double* lambda_out, double* K_out) {
    GX_LAUNCH(h, k_thermostat_lambda, 1, kRedThreads, partials, nblocks, k, target, tau, n, lambda_out, K_out);
}

}  // namespace gx
