// gx_force.cu -- the pair-force pass (ForceSystem::run, src/systems/forces.rs:163-353).
//
// Two precisions share the cell list built by gx_cells.cu:
//
//  * GX_FP64 ("plain"): every pair is evaluated with the reference's FP64
//    operation order (exact intrinsics, no FMA), so each pair's force and
//    energy are bit-identical to the reference; only the order in which an
//    atom's contributions are summed differs.  Each thread gathers the full
//    neighbourhood of its atom (every pair visited from both ends), so the
//    accumulation needs no atomics and is deterministic.
//
//  * GX_MIXED: pair arithmetic in FP32 on cell-local coordinates; every pair
//    force is quantised to 64-bit fixed point (2^-32 units) before any sum,
//    and sums are integer atomics, so the result does not depend on launch
//    configuration or scheduling.  Each pair is evaluated once (canonical
//    half shell) and contributes +F / -F to its two ends.
#include "gx_law64.cuh"
#include "gx_pair_f32.cuh"

namespace gx {

namespace {

constexpr int kForceThreads = 128;

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

// FP64 gather pass.  Each thread owns one atom i and visits every j of its
// cell and of the cells at all offsets; V and the pair count are taken only
// on visits through the canonical half shell (or j > i in the same cell), so
// each reference pair-list entry is counted once.
__global__ void __launch_bounds__(kForceThreads) k_force_f64(GridGeom g, StateBuf b, const uint32_t* __restrict__ key,
                                                              const uint32_t* __restrict__ start, uint32_t n, LawF64 L,
                                                              const double* __restrict__ psig,
                                                              const double* __restrict__ peps, double* __restrict__ vpart,
                                                              unsigned long long* __restrict__ npairs) {
    __shared__ double shd[kForceThreads / 32];
    __shared__ unsigned long long shu[kForceThreads / 32];
    uint32_t i = blockIdx.x * kForceThreads + threadIdx.x;
    double V = 0.0;
    unsigned long long np = 0;
    if (i < n) {
        uint32_t c = key[i];
        uint32_t cx, cy, cz;
        decode(g, c, cx, cy, cz);
        double xi = b.x[i], yi = b.y[i], zi = b.z[i];
        int ti = b.elem[i];
        double qi = b.charge[i], mi = b.mass[i], inv_mi = b.inv_mass[i];
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int k = -1; k < g.nfull; ++k) {
            uint32_t B;
            bool half;
            if (k < 0) {
                B = c;
                half = true;
            } else {
                B = encode(g, wrap_add(cx, g.full[k][0], g.n[0]), wrap_add(cy, g.full[k][1], g.n[1]),
                           wrap_add(cz, g.full[k][2], g.n[2]));
                half = k < g.nhalf;
            }
            uint32_t lo = start[B], hi = start[B + 1];
            for (uint32_t j = lo; j < hi; ++j) {
                if (j == i) continue;
                double dx = min_image1(xsub(xi, b.x[j]), L.box[0]);
                double dy = min_image1(xsub(yi, b.y[j]), L.box[1]);
                double dz = min_image1(xsub(zi, b.z[j]), L.box[2]);
                double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                if (d2 >= L.rc2) continue;
                double d = xsqrt(d2);
                if (d <= kEpsF64) continue;
                bool count = (k < 0) ? (j > i) : half;
                int tj = b.elem[j];
                double fmag, Vij = 0.0;
                pair_f64(L, d, psig[ti * kNElem + tj], peps[ti * kNElem + tj], qi, b.charge[j], mi, b.mass[j], fmag,
                         Vij);
                if (count) {
                    V = xadd(V, Vij);
                    ++np;
                }
                if (fmag != 0.0) {
                    double inv = xdiv(1.0, d);
                    ax = xadd(ax, xmul(xmul(xmul(dx, inv), fmag), inv_mi));
                    ay = xadd(ay, xmul(xmul(xmul(dy, inv), fmag), inv_mi));
                    az = xadd(az, xmul(xmul(xmul(dz, inv), fmag), inv_mi));
                }
            }
        }
        b.ax[i] = ax;
        b.ay[i] = ay;
        b.az[i] = az;
    }
    V = block_sum_d<kForceThreads>(V, shd);
    np = block_sum_u<kForceThreads>(np, shu);
    if (threadIdx.x == 0) {
        vpart[blockIdx.x] = V;
        if (np) atomicAdd(npairs, np);
    }
}

// Mixed pass: one thread per atom, canonical half shell, FP32 pair math,
// fixed-point +F/-F via integer atomics.
__global__ void __launch_bounds__(kForceThreads) k_force_mixed(GridGeom g, const float4* __restrict__ pos4,
                                                                const uint32_t* __restrict__ key,
                                                                const uint32_t* __restrict__ start, uint32_t n,
                                                                LawF32 L, const PairF* __restrict__ tab,
                                                                long long* __restrict__ F, size_t fstride,
                                                                unsigned long long* __restrict__ vacc,
                                                                unsigned long long* __restrict__ npairs,
                                                                uint32_t* __restrict__ err) {
    __shared__ PairF st[kMaxKinds * kMaxKinds];
    __shared__ unsigned long long shu[kForceThreads / 32];
    int nk2 = L.nkinds * L.nkinds;
    for (int t = threadIdx.x; t < nk2; t += kForceThreads) st[t] = tab[t];
    __syncthreads();
    uint32_t i = blockIdx.x * kForceThreads + threadIdx.x;
    long long vq = 0;
    unsigned long long np = 0;
    if (i < n) {
        float4 pi = pos4[i];
        int ki = __float_as_int(pi.w);
        uint32_t c = key[i];
        uint32_t cx, cy, cz;
        decode(g, c, cx, cy, cz);
        long long fx = 0, fy = 0, fz = 0;
        for (int k = -1; k < g.nhalf; ++k) {
            uint32_t B, lo, hi;
            float sx = 0.f, sy = 0.f, sz = 0.f;
            if (k < 0) {
                B = c;
                lo = i + 1;
            } else {
                int ox = g.half[k][0], oy = g.half[k][1], oz = g.half[k][2];
                B = encode(g, wrap_add(cx, ox, g.n[0]), wrap_add(cy, oy, g.n[1]), wrap_add(cz, oz, g.n[2]));
                lo = start[B];
                sx = -(float)ox * g.cellf[0];
                sy = -(float)oy * g.cellf[1];
                sz = -(float)oz * g.cellf[2];
            }
            hi = start[B + 1];
            for (uint32_t j = lo; j < hi; ++j) {
                float4 pj = pos4[j];
                float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
                if (g.minimg_mask) {
                    if (g.minimg_mask & 1) dx = fsub(dx, fmul(g.Lf[0], rintf(fmul(dx, g.invLf[0]))));
                    if (g.minimg_mask & 2) dy = fsub(dy, fmul(g.Lf[1], rintf(fmul(dy, g.invLf[1]))));
                    if (g.minimg_mask & 4) dz = fsub(dz, fmul(g.Lf[2], rintf(fmul(dz, g.invLf[2]))));
                }
                float d2 = dist2(dx, dy, dz);
                if (!(d2 < L.rc2) || d2 == 0.f) continue;
                ++np;
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
                vq += quant(v, err);
            }
        }
        atomicAdd((unsigned long long*)&F[i], (unsigned long long)fx);
        atomicAdd((unsigned long long*)&F[fstride + i], (unsigned long long)fy);
        atomicAdd((unsigned long long*)&F[2 * fstride + i], (unsigned long long)fz);
    }
    unsigned long long s = block_sum_u<kForceThreads>((unsigned long long)vq, shu);
    np = block_sum_u<kForceThreads>(np, shu);
    if (threadIdx.x == 0) {
        if (s) atomicAdd(vacc, s);
        if (np) atomicAdd(npairs, np);
    }
}

// a = F * 2^-32 * (1/m) for the mixed path.
__global__ void k_fix_to_acc(StateBuf b, const long long* __restrict__ F, size_t fstride, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double im = b.inv_mass[i];
    b.ax[i] = xmul(xmul(__ll2double_rn(F[i]), kFixInv), im);
    b.ay[i] = xmul(xmul(__ll2double_rn(F[fstride + i]), kFixInv), im);
    b.az[i] = xmul(xmul(__ll2double_rn(F[2 * fstride + i]), kFixInv), im);
}

// Observed-bond spring (src/systems/forces.rs:305-317, bond_harmonic_raw
// forces.rs:290-293) for each bond in the list, applied as many times as the
// reference's pair list holds the pair (once when `key` is null).  FP64 in
// both precisions; the mixed path quantises the result into the fixed-point
// accumulators.  The bond count is read on the device (at most `cap`), and
// the fixed grid strides over it, so the launch does not change with it.
__global__ void k_bonds(GridGeom g, StateBuf b, const uint32_t* __restrict__ key,
                        const uint32_t* __restrict__ pos_of_slot, const uint32_t* __restrict__ bonds,
                        const unsigned long long* __restrict__ nbonds_dev, size_t cap, LawF64 L,
                        const double* __restrict__ psig, const double* __restrict__ peps, double k_bind,
                        double r_eq_factor, double curv_factor, int mixed, long long* __restrict__ F, size_t fstride,
                        double* __restrict__ vbpart, unsigned long long* __restrict__ vbfix, uint32_t* __restrict__ err) {
    __shared__ double shd[kForceThreads / 32];
    const size_t nbonds = min((size_t)*nbonds_dev, cap);
    double vb = 0.0;
    for (size_t t = (size_t)blockIdx.x * kForceThreads + threadIdx.x; t < nbonds;
         t += (size_t)gridDim.x * kForceThreads) {
        uint32_t ia = pos_of_slot[bonds[2 * t]], ib = pos_of_slot[bonds[2 * t + 1]];
        double dx = min_image1(xsub(b.x[ia], b.x[ib]), L.box[0]);
        double dy = min_image1(xsub(b.y[ia], b.y[ib]), L.box[1]);
        double dz = min_image1(xsub(b.z[ia], b.z[ib]), L.box[2]);
        double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
        double d = xsqrt(d2);
        if (d2 < L.rc2 && d > kEpsF64) {
            int ta = b.elem[ia], tb = b.elem[ib];
            double sg = psig[ta * kNElem + tb], ep = peps[ta * kNElem + tb];
            double r_eq = xmul(sg, r_eq_factor);
            double rc_bond = xmul(k_bind, sg);
            if (d < rc_bond) {
                double kk = xdiv(xmul(curv_factor, ep), xmul(sg, sg));
                double dr = xsub(d, r_eq);
                double m = xmul(-kk, dr);
                double v = xmul(xmul(xmul(0.5, kk), dr), dr);
                double sw, dsw;
                smooth_f64(d, r_eq, rc_bond, sw, dsw);
                double fm = xsub(xmul(m, sw), xmul(v, dsw));
                double vv = xmul(v, sw);
                int mult = key ? pair_multiplicity(g, key[ia], key[ib]) : 1;
                double inv = xdiv(1.0, d);
                double nx = xmul(dx, inv), ny = xmul(dy, inv), nz = xmul(dz, inv);
                for (int r = 0; r < mult; ++r) {
                    vb = xadd(vb, vv);
                    if (fm == 0.0) continue;
                    if (mixed) {
                        long long qx = __double2ll_rn(xmul(xmul(nx, fm), kFixScale));
                        long long qy = __double2ll_rn(xmul(xmul(ny, fm), kFixScale));
                        long long qz = __double2ll_rn(xmul(xmul(nz, fm), kFixScale));
                        atomicAdd((unsigned long long*)&F[ia], (unsigned long long)qx);
                        atomicAdd((unsigned long long*)&F[fstride + ia], (unsigned long long)qy);
                        atomicAdd((unsigned long long*)&F[2 * fstride + ia], (unsigned long long)qz);
                        atomicAdd((unsigned long long*)&F[ib], (unsigned long long)(-qx));
                        atomicAdd((unsigned long long*)&F[fstride + ib], (unsigned long long)(-qy));
                        atomicAdd((unsigned long long*)&F[2 * fstride + ib], (unsigned long long)(-qz));
                    } else {
                        atomicAdd(&b.ax[ia], xmul(xmul(nx, fm), b.inv_mass[ia]));
                        atomicAdd(&b.ay[ia], xmul(xmul(ny, fm), b.inv_mass[ia]));
                        atomicAdd(&b.az[ia], xmul(xmul(nz, fm), b.inv_mass[ia]));
                        atomicAdd(&b.ax[ib], xmul(xmul(nx, -fm), b.inv_mass[ib]));
                        atomicAdd(&b.ay[ib], xmul(xmul(ny, -fm), b.inv_mass[ib]));
                        atomicAdd(&b.az[ib], xmul(xmul(nz, -fm), b.inv_mass[ib]));
                    }
                }
            }
        }
    }
    if (mixed) {
        long long q = __double2ll_rn(xmul(vb, kFixScale));
        if (q) atomicAdd(vbfix, (unsigned long long)q);
        (void)err;
    } else {
        vb = block_sum_d<kForceThreads>(vb, shd);
        if (threadIdx.x == 0) vbpart[blockIdx.x] = vb;
    }
}

__global__ void k_fix_to_double(const unsigned long long* __restrict__ v, double* out) {
    *out = xmul(__ll2double_rn((long long)*v), kFixInv);
}

__global__ void __launch_bounds__(256) k_sum_rows(const double* __restrict__ part, int nb, double* out) {
    __shared__ double sh[8];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += 256) s = xadd(s, part[i]);
    s = block_sum_d<256>(s, sh);
    if (threadIdx.x == 0) *out = s;
}

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// Device copies of the FP64 pair table (the mixed table is built in gx_api.cu).
double* d_psig(gx_handle* h) { return h->red + 6 * (size_t)h->cap / 64 + 6 * kRedCap; }

void launch_sum_rows(gx_handle* h, const double* part, int nb, double* out) {
    GX_LAUNCH(h, k_sum_rows, 1, 256, part, nb, out);
}

int bond_spring(gx_handle* h, bool unit_mult) {
    if (!bonds_on(h)) {
        GX_CUDA(h, cudaMemsetAsync(h->dscal + 3, 0, sizeof(double), h->stream));
        return GX_OK;
    }
    const bool mixed = h->precision == GX_MIXED;
    const size_t rows = (size_t)h->cap / 64 + kRedCap;
    double* vbpart = h->red + 1 * rows;
    double* psig = d_psig(h);
    unsigned grid = nblk(h->bonds_cap, kForceThreads);
    if (grid > 4 * 148u) grid = 4 * 148u;  // four blocks per SM; the FP64 partials need grid <= rows
    prof_begin(h, "bonds");
    GX_LAUNCH(h, k_bonds, grid, kForceThreads, h->fgrid, h->buf[h->cur], unit_mult ? nullptr : h->key_sorted,
              h->pos_of_slot, h->bonds, dnbonds(h), h->bonds_cap, make_law64(h), psig, psig + kNElem * kNElem,
              h->fs.bond_k_bind, h->fs.r_eq_factor, h->fs.curv_factor, mixed ? 1 : 0, h->F, h->cap, vbpart,
              h->dcount + 2, h->derr);
    prof_end(h, "bonds");
    if (mixed)
        GX_LAUNCH(h, k_fix_to_double, 1, 1, h->dcount + 2, h->dscal + 3);
    else
        GX_LAUNCH(h, k_sum_rows, 1, 256, vbpart, (int)grid, h->dscal + 3);
    return GX_OK;
}

int force_pass(gx_handle* h, bool finalize_acc, double* V, double* Vb, uint64_t* npairs_out, bool sync_out) {
    uint32_t n = (uint32_t)h->n;
    const GridGeom& g = h->fgrid;
    StateBuf& b = h->buf[h->cur];
    size_t rows = (size_t)h->cap / 64 + kRedCap;
    double* vpart = h->red + 0 * rows;
    double* psig = d_psig(h);
    double* peps = psig + kNElem * kNElem;
    GX_CUDA(h, cudaMemsetAsync(h->dcount, 0, 4 * sizeof(unsigned long long), h->stream));
    bool mixed = h->precision == GX_MIXED;
    LawF64 L64 = make_law64(h);
    unsigned fb = nblk(n, kForceThreads);
    if (!mixed) {
        prof_begin(h, "force_f64");
        if (n) GX_LAUNCH(h, k_force_f64, fb, kForceThreads, g, b, h->key_sorted, h->cl.start, n, L64, psig, peps,
                                                                vpart, h->dcount + 0);
        prof_end(h, "force_f64");
    } else {
        LawF32 L = make_law32(h);
        GX_CUDA(h, cudaMemsetAsync(h->F, 0, 3 * h->cap * sizeof(long long), h->stream));
        // staged kernels pack atom indices in 27 bits and need >= 3 cells per axis
        const int var = h->kernel_variant;
        bool small_ids = n < (1u << 27);
        bool tiled = g.n[0] >= 3 && g.n[1] >= 3 && g.n[2] >= 3 && (var == 2 || var == 3) && small_ids;
        bool lists = (var == 0 || var == 4) && small_ids;
        prof_begin(h, "force_mixed");
        if (n && lists)
            launch_force_mixed_lists(h, g, h->pos4, h->key_sorted, h->cl.start, n, L, h->d_pairf, h->F, h->cap,
                                     h->dcount + 1, h->dcount + 0, h->derr);
        else if (n && tiled)
            launch_force_mixed_tiled(h, g, h->pos4, h->cl.start, L, h->d_pairf, h->F, h->cap, h->dcount + 1,
                                     h->dcount + 0, h->derr);
        else if (n)
            GX_LAUNCH(h, k_force_mixed, fb, kForceThreads, g, h->pos4, h->key_sorted, h->cl.start, n, L, h->d_pairf,
                      h->F, h->cap, h->dcount + 1, h->dcount + 0, h->derr);
        prof_end(h, "force_mixed");
    }
    int rc = bond_spring(h, false);
    if (rc) return rc;
    if (mixed) {
        if (finalize_acc && n) GX_LAUNCH(h, k_fix_to_acc, nblk(n, 256), 256, b, h->F, h->cap, n);
        GX_LAUNCH(h, k_fix_to_double, 1, 1, h->dcount + 1, h->dscal + 2);
    } else {
        GX_LAUNCH(h, k_sum_rows, 1, 256, vpart, (int)fb, h->dscal + 2);
    }
    if (sync_out) {
        double vv[2];
        unsigned long long cnt;
        GX_CUDA(h, cudaMemcpyAsync(vv, h->dscal + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(&cnt, h->dcount, sizeof(cnt), cudaMemcpyDeviceToHost, h->stream));
        uint32_t e = 0;
        GX_CUDA(h, cudaMemcpyAsync(&e, h->derr, sizeof(e), cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        if (V) *V = vv[0];
        if (Vb) *Vb = vv[1];
        if (npairs_out) *npairs_out = cnt;
        if (e) {
            GX_CUDA(h, cudaMemsetAsync(h->derr, 0, sizeof(uint32_t), h->stream));
            if (e & kErrNonFinite) return set_err(h, GX_ERR_NONFINITE, "non-finite force in the pair pass");
            if (e & kErrSaturation) return set_err(h, GX_ERR_SATURATION, "fixed-point force saturated");
            if (e & kErrTimeout) return set_err(h, GX_ERR_TIMEOUT, "shared-memory staging wait timed out");
        }
    }
    return GX_OK;
}

LawF32 make_law32(const gx_handle* h) {
    LawF32 L;
    L.rc2 = (float)(h->fs.rc * h->fs.rc);
    L.lj_rc = (float)h->fs.lj_rc;
    L.lj_ron = (float)h->fs.lj_ron;
    L.inv_lj_w = (float)(1.0 / (h->fs.lj_rc - h->fs.lj_ron));
    L.coul = h->p.enable_electrostatics ? 1 : 0;
    L.coul_rc = (float)h->fs.coul_rc;
    L.coul_ron = (float)h->fs.coul_ron;
    L.inv_coul_w = L.coul ? (float)(1.0 / (h->fs.coul_rc - h->fs.coul_ron)) : 0.f;
    L.grav = h->p.enable_gravity ? 1 : 0;
    L.grav_rc = (float)h->fs.grav_rc;
    L.grav_ron = (float)h->fs.grav_ron;
    L.inv_grav_w = L.grav ? (float)(1.0 / (h->fs.grav_rc - h->fs.grav_ron)) : 0.f;
    L.nkinds = h->nkinds;
    return L;
}

int upload_pair_table_f64(gx_handle* h) {
    double* psig = d_psig(h);
    GX_CUDA(h, cudaMemcpy(psig, h->fs.pair_sigma, sizeof(h->fs.pair_sigma), cudaMemcpyHostToDevice));
    GX_CUDA(h, cudaMemcpy(psig + kNElem * kNElem, h->fs.pair_eps, sizeof(h->fs.pair_eps), cudaMemcpyHostToDevice));
    // third table: (24 eps) / sigma per element pair, the two IEEE operations
    // of the law (lj_raw, src/physics/forces.rs:346-353) done once on the host
    double e24s[kNElem * kNElem];
    for (int k = 0; k < kNElem * kNElem; ++k) {
        volatile double t = 24.0 * h->fs.pair_eps[k];  // rounded before the division
        e24s[k] = t / h->fs.pair_sigma[k];
    }
    GX_CUDA(h, cudaMemcpy(psig + 2 * kNElem * kNElem, e24s, sizeof e24s, cudaMemcpyHostToDevice));
    return GX_OK;
}

size_t red_doubles(size_t cap) { return 6 * (cap / 64) + 6 * kRedCap + 3 * kNElem * kNElem + 64; }

}  // namespace gx
