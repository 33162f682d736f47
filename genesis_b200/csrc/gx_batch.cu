// gx_batch.cu -- many small universes (temperature-sweep replicas) in one
// persistent launch.
//
// The reference sweeps temperatures by building a fresh Universe per T and
// running it to completion, one after another
// (examples/temperature_sweep.rs:70-113).  Replicas never interact, so here
// each replica is owned by one CTA that runs the whole force schedule
// (src/universe/mod.rs:356-369) for all requested ticks inside a single
// kernel launch, synchronising only with __syncthreads:
//
//   A  kick (with the pending Berendsen scale), drift, wrap, cell key,
//      shared-memory cell histogram
//   B  block scan of the histogram -> cell starts
//   C  scatter into cell order: FP32 cell-local positions + kind (pos4) and
//      the sorted -> replica-local index map; zero the fixed-point forces
//   D  pair pass over the canonical half shell (pair_f32, int64 sums)
//   E  acceleration from the fixed-point force, second kick, kinetic energy
//      (fixed-order block reduction) and the replica's Berendsen lambda
//
// The arithmetic of every phase is the single-universe mixed path's
// (exact FP64 integration, the same cell-local staging, pair_f32 and
// quantisation), so an NVE replica reproduces gx_step bit for bit.  Replicas
// are processed largest first (block 0 gets the largest).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "gx_batch.cuh"

using namespace gx;

namespace {

__device__ __forceinline__ unsigned long long warp_sum_u(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kBThreads, 2)
    k_batch(const RepDesc* __restrict__ reps, const int* __restrict__ order, BatchArrays A, LawF32 L,
            const PairF* __restrict__ tab, BatchParams P, double* __restrict__ out, uint32_t* __restrict__ err) {
    __shared__ RepDesc R;
    __shared__ uint32_t s_cnt[kBMaxCells + 1];
    __shared__ uint32_t s_start[kBMaxCells + 1];
    __shared__ PairF s_tab[kMaxKinds * kMaxKinds];
    __shared__ double s_red[kBThreads / 32];
    __shared__ unsigned long long s_redu[kBThreads / 32][2];
    __shared__ uint32_t s_wsum[kBThreads / 32];
    __shared__ double s_lambda;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int r = order[blockIdx.x];
    if (tid == 0) R = reps[r];
    for (int t = tid; t < L.nkinds * L.nkinds; t += kBThreads) s_tab[t] = tab[t];
    if (tid == 0) s_lambda = 1.0;
    __syncthreads();
    const GridGeom& g = R.g;
    const uint32_t base = R.base, n = R.n, ncell = g.ncell;
    const int nk = L.nkinds;
    double Vlast = 0.0, lam_last = 1.0;
    unsigned long long np_last = 0;

    for (int step = 0; step < P.nsteps; ++step) {
        // ---- A: kick (pending lambda), drift, wrap, cell key, histogram
        for (uint32_t c = tid; c < ncell; c += kBThreads) s_cnt[c] = 0u;
        __syncthreads();
        const double lam = s_lambda;
        for (uint32_t i = tid; i < n; i += kBThreads) {
            const size_t gi = base + i;
            double vx = xadd(xmul(A.vx[gi], lam), xmul(A.ax[gi], P.half_dt));
            double vy = xadd(xmul(A.vy[gi], lam), xmul(A.ay[gi], P.half_dt));
            double vz = xadd(xmul(A.vz[gi], lam), xmul(A.az[gi], P.half_dt));
            double x = xadd(A.x[gi], xmul(vx, P.dt));
            double y = xadd(A.y[gi], xmul(vy, P.dt));
            double z = xadd(A.z[gi], xmul(vz, P.dt));
            if (P.boundaries) {
                x = xsub(rem_euclid(x, xmul(2.0, R.half_box[0])), R.half_box[0]);
                y = xsub(rem_euclid(y, xmul(2.0, R.half_box[1])), R.half_box[1]);
                z = xsub(rem_euclid(z, xmul(2.0, R.half_box[2])), R.half_box[2]);
            }
            if (!isfinite(x) || !isfinite(y) || !isfinite(z)) atomicOr(err, kErrNonFinite);
            A.vx[gi] = vx;
            A.vy[gi] = vy;
            A.vz[gi] = vz;
            A.x[gi] = x;
            A.y[gi] = y;
            A.z[gi] = z;
            uint32_t k = cell_of(g, x, y, z);
            A.key[gi] = k;
            atomicAdd(&s_cnt[k], 1u);
        }
        __syncthreads();
        // ---- B: exclusive scan of the histogram (ncell + 1 entries)
        {
            const uint32_t m = ncell + 1;
            const uint32_t per = (m + kBThreads - 1) / kBThreads;
            const uint32_t lo = tid * per, hi = lo + per < m ? lo + per : m;
            uint32_t local = 0;
            for (uint32_t c = lo; c < hi; ++c) local += c < ncell ? s_cnt[c] : 0u;
            uint32_t inc = local;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            if (lane == 31) s_wsum[w] = inc;
            __syncthreads();
            if (w == 0) {
                uint32_t x = lane < kBThreads / 32 ? s_wsum[lane] : 0u;
                uint32_t xi = x;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    uint32_t t = __shfl_up_sync(0xffffffffu, xi, o);
                    if (lane >= o) xi += t;
                }
                if (lane < kBThreads / 32) s_wsum[lane] = xi - x;
            }
            __syncthreads();
            uint32_t run = s_wsum[w] + inc - local;
            for (uint32_t c = lo; c < hi; ++c) {
                uint32_t cnt = c < ncell ? s_cnt[c] : 0u;
                s_start[c] = run;
                run += cnt;
            }
        }
        __syncthreads();
        for (uint32_t c = tid; c < ncell; c += kBThreads) s_cnt[c] = 0u;  // reused as fill counters
        __syncthreads();
        // ---- C: scatter into cell order, stage pos4, zero forces
        for (uint32_t i = tid; i < n; i += kBThreads) {
            const size_t gi = base + i;
            uint32_t k = A.key[gi];
            uint32_t p = s_start[k] + atomicAdd(&s_cnt[k], 1u);
            uint32_t ix, iy, iz;
            decode(g, k, ix, iy, iz);
            A.pos4[base + p] = make_float4((float)cell_local(A.x[gi], g.L[0], g.cell[0], ix),
                                           (float)cell_local(A.y[gi], g.L[1], g.cell[1], iy),
                                           (float)cell_local(A.z[gi], g.L[2], g.cell[2], iz),
                                           __int_as_float((int)A.kind[gi]));
            A.idx[base + p] = i;
            A.skey[base + p] = k;
            A.F[gi] = 0;
            A.F[A.total + gi] = 0;
            A.F[2 * A.total + gi] = 0;
        }
        __syncthreads();
        // ---- D: pair pass over the canonical half shell
        long long vq = 0;
        unsigned long long np = 0;
        for (uint32_t p = tid; p < n; p += kBThreads) {
            const float4 pi = A.pos4[base + p];
            const int ki = __float_as_int(pi.w);
            const uint32_t c = A.skey[base + p];
            uint32_t cx, cy, cz;
            decode(g, c, cx, cy, cz);
            long long fx = 0, fy = 0, fz = 0;
            for (int t = -1; t < g.nhalf; ++t) {
                uint32_t B, lo;
                float sx = 0.f, sy = 0.f, sz = 0.f;
                if (t < 0) {
                    B = c;
                    lo = p + 1;
                } else {
                    int ox = g.half[t][0], oy = g.half[t][1], oz = g.half[t][2];
                    B = encode(g, wrap_add(cx, ox, g.n[0]), wrap_add(cy, oy, g.n[1]), wrap_add(cz, oz, g.n[2]));
                    lo = s_start[B];
                    sx = -(float)ox * g.cellf[0];
                    sy = -(float)oy * g.cellf[1];
                    sz = -(float)oz * g.cellf[2];
                }
                const uint32_t hi = s_start[B + 1];
                for (uint32_t j = lo; j < hi; ++j) {
                    const float4 pj = A.pos4[base + j];
                    float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
                    if (g.minimg_mask) {
                        if (g.minimg_mask & 1) dx = fsub(dx, fmul(g.Lf[0], rintf(fmul(dx, g.invLf[0]))));
                        if (g.minimg_mask & 2) dy = fsub(dy, fmul(g.Lf[1], rintf(fmul(dy, g.invLf[1]))));
                        if (g.minimg_mask & 4) dz = fsub(dz, fmul(g.Lf[2], rintf(fmul(dz, g.invLf[2]))));
                    }
                    const float d2 = dist2(dx, dy, dz);
                    if (!(d2 < L.rc2) || d2 == 0.f) continue;
                    ++np;
                    float fs, v;
                    pair_f32(L, s_tab[ki * nk + __float_as_int(pj.w)], d2, fs, v);
                    long long qx, qy, qz;
                quant3(fmul(dx, fs), fmul(dy, fs), fmul(dz, fs), qx, qy, qz, err);
                    fx += qx;
                    fy += qy;
                    fz += qz;
                    const size_t gj = base + A.idx[base + j];
                    atomicAdd((unsigned long long*)&A.F[gj], (unsigned long long)(-qx));
                    atomicAdd((unsigned long long*)&A.F[A.total + gj], (unsigned long long)(-qy));
                    atomicAdd((unsigned long long*)&A.F[2 * A.total + gj], (unsigned long long)(-qz));
                    vq += quant(v, err);
                }
            }
            const size_t gp = base + A.idx[base + p];
            atomicAdd((unsigned long long*)&A.F[gp], (unsigned long long)fx);
            atomicAdd((unsigned long long*)&A.F[A.total + gp], (unsigned long long)fy);
            atomicAdd((unsigned long long*)&A.F[2 * A.total + gp], (unsigned long long)fz);
        }
        __syncthreads();
        // ---- E: a = F * 2^-32 / m, second kick, kinetic energy, lambda
        double kp = 0.0;
        for (uint32_t i = tid; i < n; i += kBThreads) {
            const size_t gi = base + i;
            const double im = A.inv_mass[gi];
            double ax = xmul(xmul(__ll2double_rn(A.F[gi]), kFixInv), im);
            double ay = xmul(xmul(__ll2double_rn(A.F[A.total + gi]), kFixInv), im);
            double az = xmul(xmul(__ll2double_rn(A.F[2 * A.total + gi]), kFixInv), im);
            A.ax[gi] = ax;
            A.ay[gi] = ay;
            A.az[gi] = az;
            double vx = xadd(A.vx[gi], xmul(ax, P.half_dt));
            double vy = xadd(A.vy[gi], xmul(ay, P.half_dt));
            double vz = xadd(A.vz[gi], xmul(az, P.half_dt));
            A.vx[gi] = vx;
            A.vy[gi] = vy;
            A.vz[gi] = vz;
            double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
            kp = xadd(kp, xmul(xmul(0.5, A.mass[gi]), l2));
        }
        kp = warp_sum_d(kp);
        unsigned long long uv = warp_sum_u((unsigned long long)vq), un = warp_sum_u(np);
        if (lane == 0) {
            s_red[w] = kp;
            s_redu[w][0] = uv;
            s_redu[w][1] = un;
        }
        __syncthreads();
        if (tid == 0) {
            double ks = 0.0;
            unsigned long long vs = 0, ns = 0;
            for (int k = 0; k < kBThreads / 32; ++k) {
                ks = xadd(ks, s_red[k]);
                vs += s_redu[k][0];
                ns += s_redu[k][1];
            }
            double l = 1.0;  // ThermostatSystem::run tail, src/systems/thermostat.rs:58-71
            if (R.thermo && n > 0) {
                double t = xdiv(xmul(2.0 / 3.0, xdiv(ks, (double)n)), P.k_thermal);
                if (isfinite(t) && t > 0.0) {
                    double l2 = xadd(1.0, xmul(xdiv(1.0, R.tau), xsub(xdiv(R.target, t), 1.0)));
                    l = xsqrt(fmax(l2, 0.0));
                }
            }
            s_lambda = l;
            Vlast = xmul(__ll2double_rn((long long)vs), kFixInv);
            lam_last = l;
            np_last = ns;
        }
        __syncthreads();
    }
    // Commit the last pending Berendsen scale and measure K after it, as
    // StatsSystem does after the thermostat (src/systems/aggregate.rs:86-93).
    const double lam = s_lambda;
    double kp = 0.0;
    for (uint32_t i = tid; i < n; i += kBThreads) {
        const size_t gi = base + i;
        double vx = xmul(A.vx[gi], lam), vy = xmul(A.vy[gi], lam), vz = xmul(A.vz[gi], lam);
        A.vx[gi] = vx;
        A.vy[gi] = vy;
        A.vz[gi] = vz;
        double l2 = xadd(xadd(xmul(vx, vx), xmul(vy, vy)), xmul(vz, vz));
        kp = xadd(kp, xmul(xmul(0.5, A.mass[gi]), l2));
    }
    kp = warp_sum_d(kp);
    if (lane == 0) s_red[w] = kp;
    __syncthreads();
    if (tid == 0) {
        double ks = 0.0;
        for (int k = 0; k < kBThreads / 32; ++k) ks = xadd(ks, s_red[k]);
        out[4 * r + 0] = ks;
        out[4 * r + 1] = Vlast;
        out[4 * r + 2] = lam_last;
        out[4 * r + 3] = (double)np_last;
    }
}

}  // namespace



namespace {

int berr(gx_batch* b, int code, const std::string& m) {
    if (b) b->err = m;
    return code;
}
#define GXB_CUDA(b, call)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return berr(b, GX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_arrays(gx_batch* b) {
    cudaFree(b->A.x);
    cudaFree(b->A.kind);
    cudaFree(b->A.key);
    cudaFree(b->A.pos4);
    cudaFree(b->A.F);
    b->A = BatchArrays{};
}

}  // namespace

extern "C" {

const char* gx_batch_last_error(const gx_batch* b) { return b ? b->err.c_str() : "null batch"; }

int gx_batch_create(const gx_params* p, int nrep, const double* box, const double* target_T, gx_batch** out) {
    if (!p || !out || nrep <= 0 || !box) return GX_ERR_ARG;
    *out = nullptr;
    gx_batch* b = new gx_batch();
    *out = b;
    b->p = *p;
    b->nrep = nrep;
    double max_pair = 0.0, max_sigma = 0.0;
    for (int i = 0; i < kNElem; ++i) {
        max_sigma = std::fmax(max_sigma, p->sigma[i]);
        for (int j = 0; j < kNElem; ++j) {
            double s = 0.5 * (p->sigma[i] + p->sigma[j]);
            b->pair_sigma[i * kNElem + j] = s;
            b->pair_eps[i * kNElem + j] = p->thermal_constant * std::sqrt(p->epsilon_k[i] * p->epsilon_k[j]);
            max_pair = std::fmax(max_pair, s);
        }
    }
    if (p->enable_gravity) return berr(b, GX_ERR_UNSUPPORTED, "batched replicas do not support gravity");
    double lj_rc = std::fmax(p->lj_cutoff_factor, 1.0) * max_pair;
    double coul_rc = p->enable_electrostatics ? std::fmax(p->coulomb_cutoff, 1.0) * max_sigma : 0.0;
    double rc = std::fmax(lj_rc, coul_rc);
    b->rc = rc;
    LawF32& L = b->L;
    L.rc2 = (float)(rc * rc);
    L.lj_rc = (float)lj_rc;
    L.lj_ron = (float)(0.9 * lj_rc);
    L.inv_lj_w = (float)(1.0 / (lj_rc - 0.9 * lj_rc));
    L.coul = p->enable_electrostatics ? 1 : 0;
    L.coul_rc = (float)coul_rc;
    L.coul_ron = (float)(0.9 * coul_rc);
    L.inv_coul_w = L.coul ? (float)(1.0 / (coul_rc - 0.9 * coul_rc)) : 0.f;
    L.nkinds = 0;
    b->reps.resize(nrep);
    for (int r = 0; r < nrep; ++r) {
        int ok = 0;
        RepDesc& d = b->reps[r];
        d.g = make_grid(box + 3 * r, rc, &ok);
        if (!ok) return berr(b, GX_ERR_ARG, "invalid replica box");
        for (int k = 0; k < 3; ++k) d.half_box[k] = 0.5 * box[3 * r + k];
        double T = target_T ? target_T[r] : p->thermostat_temperature;
        d.thermo = (p->enable_thermostat && T > 0.0) ? 1 : 0;
        d.target = T;
        d.tau = std::fmax(p->thermostat_tau, 1.0);
        d.base = 0;
        d.n = 0;
    }
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_reps, nrep * sizeof(RepDesc));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_order, nrep * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_out, 4 * nrep * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tab, kMaxKinds * kMaxKinds * sizeof(PairF));
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev[1]);
    if (e != cudaSuccess) return berr(b, GX_ERR_CUDA, cudaGetErrorString(e));
    cudaMemset(b->d_err, 0, sizeof(uint32_t));
    return GX_OK;
}

void gx_batch_destroy(gx_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_nl_free(b->nl);
    b->nl = nullptr;
    batch_flat_free(b->flat);
    b->flat = nullptr;
    free_arrays(b);
    cudaFree(b->d_reps);
    cudaFree(b->d_order);
    cudaFree(b->d_out);
    cudaFree(b->d_err);
    cudaFree(b->d_tab);
    if (b->ev[0]) cudaEventDestroy(b->ev[0]);
    if (b->ev[1]) cudaEventDestroy(b->ev[1]);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int gx_batch_set_state(gx_batch* b, const uint32_t* natoms, const double* pos, const double* vel, const double* acc,
                       const uint8_t* elem, const double* charge, const double* mass) {
    if (!b || !natoms) return GX_ERR_ARG;
    size_t total = 0;
    for (int r = 0; r < b->nrep; ++r) {
        b->reps[r].base = (uint32_t)total;
        b->reps[r].n = natoms[r];
        total += natoms[r];
    }
    if (total > 0x7FFFFFFFu) return berr(b, GX_ERR_ARG, "too many atoms");
    if (total && (!pos || !vel || !elem)) return GX_ERR_ARG;
    static const double kMass[kNElem] = {1.008, 4.0026, 12.011, 14.007, 15.999, 22.99, 28.085, 30.974, 32.06, 55.845};
    // kinds: distinct (element, charge), as gx_set_state builds them
    int nk = 0;
    uint8_t kel[kMaxKinds];
    double kq[kMaxKinds];
    std::vector<uint8_t> kind(total);
    for (size_t i = 0; i < total; ++i) {
        if (elem[i] >= kNElem) return berr(b, GX_ERR_ARG, "element index out of range (0..9)");
        double q = charge ? charge[i] : b->p.charge[elem[i]];
        int f = -1;
        for (int k = 0; k < nk; ++k)
            if (kel[k] == elem[i] && kq[k] == q) f = k;
        if (f < 0) {
            if (nk == kMaxKinds) return berr(b, GX_ERR_UNSUPPORTED, "at most 16 distinct (element, charge) kinds");
            kel[nk] = elem[i];
            kq[nk] = q;
            f = nk++;
        }
        kind[i] = (uint8_t)f;
    }
    PairF tab[kMaxKinds * kMaxKinds];
    std::memset(tab, 0, sizeof tab);
    for (int a = 0; a < nk; ++a)
        for (int c = 0; c < nk; ++c) {
            double sg = b->pair_sigma[kel[a] * kNElem + kel[c]], ep = b->pair_eps[kel[a] * kNElem + kel[c]];
            PairF& t = tab[a * nk + c];
            t.sigma = (float)sg;
            t.half_sigma = (float)(0.5 * sg);
            t.inv_half_sigma = (float)(2.0 / sg);
            t.eps4 = (float)(4.0 * ep);
            t.eps24 = (float)(24.0 * ep);
            int lo = a < c ? a : c, hi = a < c ? c : a;
            t.qq = (float)(b->p.coulomb_constant * kq[lo] * kq[hi]);
        }
    b->L.nkinds = nk;
    GXB_CUDA(b, cudaSetDevice(b->p.device));
    GXB_CUDA(b, cudaStreamSynchronize(b->stream));
    batch_flat_free(b->flat);  // replica ranges, kinds and sizes change
    b->flat = nullptr;
    GXB_CUDA(b, cudaMemcpy(b->d_tab, tab, sizeof tab, cudaMemcpyHostToDevice));
    free_arrays(b);
    size_t cap = total < 1 ? 1 : total;
    BatchArrays& A = b->A;
    GXB_CUDA(b, cudaMalloc(&A.x, 11 * cap * sizeof(double)));
    A.y = A.x + cap;
    A.z = A.x + 2 * cap;
    A.vx = A.x + 3 * cap;
    A.vy = A.x + 4 * cap;
    A.vz = A.x + 5 * cap;
    A.ax = A.x + 6 * cap;
    A.ay = A.x + 7 * cap;
    A.az = A.x + 8 * cap;
    A.mass = A.x + 9 * cap;
    A.inv_mass = A.x + 10 * cap;
    GXB_CUDA(b, cudaMalloc(&A.kind, cap));
    GXB_CUDA(b, cudaMalloc(&A.key, 3 * cap * sizeof(uint32_t)));
    A.idx = A.key + cap;
    A.skey = A.key + 2 * cap;
    GXB_CUDA(b, cudaMalloc(&A.pos4, cap * sizeof(float4)));
    GXB_CUDA(b, cudaMalloc(&A.F, 3 * cap * sizeof(long long)));
    A.total = cap;
    b->total = total;
    std::vector<double> col(cap);
    auto up_aos = [&](const double* src, double* dx, double* dy, double* dz) -> int {
        double* dst[3] = {dx, dy, dz};
        for (int k = 0; k < 3; ++k) {
            for (size_t i = 0; i < total; ++i) col[i] = src ? src[3 * i + k] : 0.0;
            GXB_CUDA(b, cudaMemcpy(dst[k], col.data(), total * sizeof(double), cudaMemcpyHostToDevice));
        }
        return GX_OK;
    };
    int rc;
    if ((rc = up_aos(pos, A.x, A.y, A.z))) return rc;
    if ((rc = up_aos(vel, A.vx, A.vy, A.vz))) return rc;
    if ((rc = up_aos(acc, A.ax, A.ay, A.az))) return rc;
    for (size_t i = 0; i < total; ++i) col[i] = mass ? mass[i] : kMass[elem[i]];
    GXB_CUDA(b, cudaMemcpy(A.mass, col.data(), total * sizeof(double), cudaMemcpyHostToDevice));
    for (size_t i = 0; i < total; ++i) col[i] = 1.0 / (mass ? mass[i] : kMass[elem[i]]);  // 1.0 / mass
    GXB_CUDA(b, cudaMemcpy(A.inv_mass, col.data(), total * sizeof(double), cudaMemcpyHostToDevice));
    GXB_CUDA(b, cudaMemcpy(A.kind, kind.data(), total, cudaMemcpyHostToDevice));
    GXB_CUDA(b, cudaMemcpy(b->d_reps, b->reps.data(), b->nrep * sizeof(RepDesc), cudaMemcpyHostToDevice));
    std::vector<int> order(b->nrep);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->reps[a].n > b->reps[c].n; });
    GXB_CUDA(b, cudaMemcpy(b->d_order, order.data(), b->nrep * sizeof(int), cudaMemcpyHostToDevice));
    b->has_state = true;
    ++b->version;
    batch_nl_free(b->nl);  // sized for the old atom counts
    b->nl = nullptr;
    return GX_OK;
}

int gx_batch_step(gx_batch* b, int nsteps, double* stats, double* device_ms) {
    if (!b || nsteps < 0) return GX_ERR_ARG;
    if (!b->has_state) return berr(b, GX_ERR_STATE, "no state uploaded (call gx_batch_set_state first)");
    BatchParams P;
    P.dt = b->p.dt;
    P.half_dt = 0.5 * b->p.dt;
    P.k_thermal = b->p.thermal_constant;
    P.boundaries = b->p.enable_boundaries ? 1 : 0;
    P.nsteps = nsteps;
    if (b->mode == 1)
        for (const RepDesc& d : b->reps)
            if (d.g.ncell > kBMaxCells)
                return berr(b, GX_ERR_CAPACITY,
                            "a replica grid exceeds 4096 force cells (the persistent mode keeps them in shared memory)");
    GXB_CUDA(b, cudaEventRecord(b->ev[0], b->stream));
    if (b->mode == 1) {
        if (nsteps > 0)
            k_batch<<<b->nrep, kBThreads, 0, b->stream>>>(b->d_reps, b->d_order, b->A, b->L, b->d_tab, P, b->d_out,
                                                          b->d_err);
        GXB_CUDA(b, cudaGetLastError());
    } else if (b->mode == 3) {
        int rc = batch_coop_step(b, nsteps, nullptr);
        if (rc) return rc;
    } else if (b->mode == 4) {
        int rc = batch_nl_step(b, nsteps, nullptr);
        if (rc) return rc;
    } else {
        int rc = batch_flat_step(b, nsteps, nullptr);
        if (rc) return rc;
    }
    if (b->mode != 4) ++b->version;  // a mode-4 list no longer matches the state
    GXB_CUDA(b, cudaEventRecord(b->ev[1], b->stream));
    uint32_t e = 0;
    GXB_CUDA(b, cudaMemcpyAsync(&e, b->d_err, sizeof e, cudaMemcpyDeviceToHost, b->stream));
    if (stats)
        GXB_CUDA(b, cudaMemcpyAsync(stats, b->d_out, 4 * b->nrep * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    GXB_CUDA(b, cudaStreamSynchronize(b->stream));
    if (device_ms) {
        float t = 0.f;
        cudaEventElapsedTime(&t, b->ev[0], b->ev[1]);
        *device_ms = t;
    }
    if (e) {
        cudaMemset(b->d_err, 0, sizeof(uint32_t));
        if (e & kErrNonFinite) return berr(b, GX_ERR_NONFINITE, "non-finite position or force in a replica");
        if (e & kErrSaturation) return berr(b, GX_ERR_SATURATION, "fixed-point force saturated");
        if (e & kErrTimeout) return berr(b, GX_ERR_TIMEOUT, "a grid barrier of the cooperative launch timed out");
    }
    return GX_OK;
}

int gx_batch_set_mode(gx_batch* b, int mode) {
    if (!b || mode < 0 || mode > 4) return GX_ERR_ARG;
    b->mode = mode == 0 ? 2 : mode;
    return GX_OK;
}

int gx_batch_set_list_skin(gx_batch* b, double skin) {
    if (!b || !(skin >= 0.0) || !std::isfinite(skin)) return GX_ERR_ARG;
    b->nl_skin = skin;  // the next mode-4 step rebuilds its lists on the new grid
    return GX_OK;
}

int gx_batch_list_rebuilds(gx_batch* b, uint64_t* rebuilds) {
    if (!b || !rebuilds) return GX_ERR_ARG;
    return batch_nl_rebuilds(b, rebuilds);
}

int gx_batch_list_stats(gx_batch* b, uint64_t* entries, uint64_t* overflowed_slots) {
    if (!b || !entries || !overflowed_slots) return GX_ERR_ARG;
    return batch_nl_stats(b, entries, overflowed_slots);
}

int gx_batch_get_mode(gx_batch* b, int* mode) {
    if (!b || !mode) return GX_ERR_ARG;
    *mode = b->mode;
    return GX_OK;
}

int gx_batch_autotune(gx_batch* b, int ticks, int* mode, double* ms) {
    if (!b || ticks < 1) return GX_ERR_ARG;
    if (!b->has_state) return berr(b, GX_ERR_STATE, "no state uploaded (call gx_batch_set_state first)");
    const size_t n9 = 9 * b->A.total;
    double* snap = nullptr;
    GXB_CUDA(b, cudaMalloc(&snap, n9 * sizeof(double)));
    // x y z vx vy vz ax ay az are the first nine columns of one allocation
    GXB_CUDA(b, cudaMemcpyAsync(snap, b->A.x, n9 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    const int saved = b->mode;
    double t[4] = {-1.0, -1.0, -1.0, -1.0};
    int rc = GX_OK;
    bool fits1 = true;  // mode 1 keeps each replica's cells in shared memory
    for (const RepDesc& d : b->reps) fits1 = fits1 && d.g.ncell <= kBMaxCells;
    const double skin0 = b->nl_skin;
    double best_skin = skin0;
    for (int m = 1; m <= 4 && !rc; ++m) {
        if (m == 1 && !fits1) continue;
        if (m == 4 && !batch_nl_eligible(b)) continue;
        b->mode = m;
        // mode 4 also over its list skin: 0.1, 0.15 and 0.2 r_c
        const double fr[3] = {0.1, 0.15, 0.2};
        for (int k = 0; k < (m == 4 ? 3 : 1) && !rc; ++k) {
            if (m == 4) b->nl_skin = fr[k] * b->rc;
            double w = 0.0;
            if (!(rc = gx_batch_step(b, 1, nullptr, &w)) && !(rc = gx_batch_step(b, ticks, nullptr, &w)) &&
                (t[m - 1] < 0.0 || w < t[m - 1])) {
                t[m - 1] = w;
                if (m == 4) best_skin = b->nl_skin;
            }
            cudaMemcpyAsync(b->A.x, snap, n9 * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
            ++b->version;
        }
    }
    cudaStreamSynchronize(b->stream);
    cudaFree(snap);
    int pick = 2;
    for (int m = 1; m <= 4; ++m)
        if (t[m - 1] >= 0.0 && t[m - 1] < t[pick - 1]) pick = m;
    b->mode = rc ? saved : pick;
    b->nl_skin = (!rc && pick == 4) ? best_skin : skin0;
    if (mode) *mode = b->mode;
    if (ms)
        for (int m = 0; m < 4; ++m) ms[m] = t[m] >= 0.0 ? t[m] / ticks : -1.0;
    return rc;
}

int gx_batch_get_state(gx_batch* b, double* pos, double* vel, double* acc) {
    if (!b) return GX_ERR_ARG;
    if (!b->has_state) return berr(b, GX_ERR_STATE, "no state uploaded");
    const size_t total = b->total;
    std::vector<double> col(total);
    double* outs[3] = {pos, vel, acc};
    double* srcs[3][3] = {{b->A.x, b->A.y, b->A.z}, {b->A.vx, b->A.vy, b->A.vz}, {b->A.ax, b->A.ay, b->A.az}};
    GXB_CUDA(b, cudaStreamSynchronize(b->stream));
    for (int q = 0; q < 3; ++q) {
        if (!outs[q]) continue;
        for (int k = 0; k < 3; ++k) {
            GXB_CUDA(b, cudaMemcpy(col.data(), srcs[q][k], total * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < total; ++i) outs[q][3 * i + k] = col[i];
        }
    }
    return GX_OK;
}

}  // extern "C"
