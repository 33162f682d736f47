// gx_adjoint.cu -- reverse-mode derivatives of short NVE horizons.
//
// The reference has no derivatives.  This file differentiates its tick
// (src/universe/mod.rs:356-369: kick, drift, wrap, forces, kick) with respect
// to the per-element LJ parameters sigma[10] and epsilon_k[10], for two
// smoothed observables: the potential energy after each tick and a
// Gaussian-kernel pair distribution averaged over sampled ticks.
//
// Forward.  The trajectory is recomputed in slot order (atoms never move
// between arrays; a per-tick counting sort gives the cell list as an index),
// in FP64 with the reference's per-pair arithmetic (pair_f64).  On a handle
// of mixed precision the forward is the mixed method instead: the FP32 pair
// law of the list passes (pair_f32) on the FP64 minimum-image displacement
// rounded to FP32, the per-atom force summed in 2^-32 fixed point, and FP64
// positions, velocities and observables; the backward below stays FP64,
// linearised on that trajectory.  A checkpoint of (x, v, a) is kept every K
// ticks.
//
// Backward.  Per segment: restore the checkpoint, recompute the segment's
// positions, then walk the ticks backwards.  With adjoints (Lx, Lv, La) of
// the state after tick t, tick t's adjoint is
//     Lx += dO_t/dx                           (observables at tick t)
//     W   = La + (dt/2) Lv                    (cotangent of a_t)
//     Lx += (da/dx)^T W,  Ltheta += (da/dtheta)^T W
//     Lv += dt Lx,  La = (dt/2) Lv            (drift and first kick)
// and (da/dx)^T W is the pairwise Hessian-vector product: with
// a_i = sum_j f(d_ij) n_ij / m_i, u = W_i/m_i - W_j/m_j and rho = n.u, the
// pair adds  f'(d) rho n + (f/d) (u - rho n)  to Lx_i (and the opposite to
// Lx_j).  One thread owns one atom and gathers its full neighbourhood, so
// every sum is over a fixed order: the result is deterministic and needs no
// atomics.  Parameter partials are accumulated per atom (the own end of each
// visit takes half of the pair's derivative) and reduced per element once at
// the end.
//
// The cutoffs are multiples of max sigma; their derivative goes to the
// lowest-index element attaining the max.  The hard-core clamp
// r = max(d, sigma/2) and the Coulomb/gravity clamp r = max(d, 0.5) are
// differentiated on the side the value takes; the periodic wrap and the
// minimum image have derivative one.
#include <cmath>
#include <cstring>
#include <vector>

#include "gx_law64.cuh"
#include "gx_pair_f32.cuh"

namespace gx {
namespace {

constexpr int kAdjThreads = 128;
constexpr int kAdjLanes = 8;  // lanes per atom in the pair kernels: each takes every 8th neighbour cell
constexpr int kAdjMaxBins = 512;
constexpr double kRonFrac = 0.9;  // r_on = 0.9 rc for every switched term (forces.rs:237, systems/forces.rs:118-124)
constexpr double kHistScale = 4294967296.0;
constexpr double kHistInv = 1.0 / 4294967296.0;
constexpr int kNOut = 2 * kNElem + 3;  // per-element sigma, epsilon sums + three cutoff sums

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Component k of a 3-vector field stored as three rows of `cap` doubles.
struct Vec3Field {
    double* p;
    size_t cap;
    __device__ __forceinline__ double& c(int k, uint32_t i) const { return p[(size_t)k * cap + i]; }
};

struct GrSpec {
    int bins;
    double dr, width, reach, c2;  // bin width, kernel width, truncation radius, -1/(2 w^2)
};

// Switch S(r) of smooth_cutoff (forces.rs:302-318) with its first two
// r-derivatives and the derivatives of S and dS/dr with respect to rc
// (r_on = 0.9 rc moves with it).
struct SwD {
    double S, S1, S2, Src, S1rc;
};
__device__ __forceinline__ SwD switch_d(double r, double ron, double rc) {
    SwD o{0.0, 0.0, 0.0, 0.0, 0.0};
    if (r <= ron) {
        o.S = 1.0;
        return o;
    }
    if (r >= rc) return o;
    double iw = 1.0 / (rc - ron);
    double u = (r - ron) * iw, omu = 1.0 - u;
    double Su = -30.0 * u * u * omu * omu;
    double Suu = -60.0 * u * omu * (1.0 - 2.0 * u);
    o.S = 1.0 + u * u * u * (-10.0 + u * (15.0 - 6.0 * u));
    o.S1 = Su * iw;
    o.S2 = Suu * iw * iw;
    double urc = -(kRonFrac + (1.0 - kRonFrac) * u) * iw;
    o.Src = Su * urc;
    o.S1rc = Suu * urc * iw - Su * (1.0 - kRonFrac) * iw * iw;
    return o;
}

// One pair's force magnitude f (repulsive > 0) and energy U with the
// derivatives the adjoint needs.
struct PairG {
    double f, fd, Ud;         // f, df/dd, dU/dd
    double fs, Us, fe, Ue;    // d/dsigma_ab, d/deps_ab of the LJ term
    double frc[3], Urc[3];    // d/drc of the LJ, Coulomb and gravity terms
};

__device__ __forceinline__ void central_term(double q, double d, double ron, double rc, PairG& o, int slot) {
    bool clamped = d < 0.5;  // r = max(d, 0.5), systems/forces.rs:283,293
    double r = clamped ? 0.5 : d, rd = clamped ? 0.0 : 1.0;
    double ir = 1.0 / r;
    double v = q * ir, m = v * ir;
    double mr = -2.0 * m * ir, vr = -m;
    SwD w = switch_d(d, ron, rc);  // the switch is evaluated at d, not r
    o.f += m * w.S - v * w.S1;
    o.fd += mr * rd * w.S + m * w.S1 - vr * rd * w.S1 - v * w.S2;
    o.Ud += vr * rd * w.S + v * w.S1;
    o.frc[slot] = m * w.Src - v * w.S1rc;
    o.Urc[slot] = v * w.Src;
}

__device__ __forceinline__ PairG pair_grad(const LawF64& L, double d, double sg, double ep, double qa, double qb,
                                           double ma, double mb) {
    PairG o;
    o.f = o.fd = o.Ud = o.fs = o.Us = o.fe = o.Ue = 0.0;
    for (int k = 0; k < 3; ++k) o.frc[k] = o.Urc[k] = 0.0;
    if (d < L.lj_rc) {
        // force_switched_scalar (forces.rs:270-275): r = max(d, sigma/2)
        double half = 0.5 * sg;
        bool clamped = d < half;
        double r = clamped ? half : d, rd = clamped ? 0.0 : 1.0, rs = clamped ? 0.5 : 0.0;
        double is = 1.0 / sg;
        double s = sg / r, s2 = s * s, s6 = s2 * s2 * s2, s12 = s6 * s6;
        double v1 = 4.0 * (s12 - s6);                            // V / eps
        double m1 = 24.0 * is * s * (2.0 * s12 - s6);            // -dV/dr / eps
        double m1r = 24.0 * is * is * (7.0 * s6 * s2 - 26.0 * s12 * s2);
        double m1s = 144.0 * is * is * (4.0 * s12 * s - s6 * s);
        double v1s = 24.0 * is * (2.0 * s12 - s6);
        SwD w = switch_d(r, L.lj_ron, L.lj_rc);
        double F1 = m1 * w.S - v1 * w.S1;
        double fr = ep * (m1r * w.S + 2.0 * m1 * w.S1 - v1 * w.S2);
        double Ur = ep * (-m1 * w.S + v1 * w.S1);
        o.f = ep * F1;
        o.fd = fr * rd;
        o.Ud = Ur * rd;
        o.fs = ep * (m1s * w.S - v1s * w.S1) + fr * rs;
        o.Us = ep * v1s * w.S + Ur * rs;
        o.fe = F1;
        o.Ue = v1 * w.S;
        o.frc[0] = ep * (m1 * w.Src - v1 * w.S1rc);
        o.Urc[0] = ep * v1 * w.Src;
    }
    if (L.coul && d < L.coul_rc) central_term(L.k_e * qa * qb, d, L.coul_ron, L.coul_rc, o, 1);
    if (L.grav && d < L.grav_rc) central_term(-L.G * ma * mb, d, L.grav_ron, L.grav_rc, o, 2);
    return o;
}

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

// Neighbour cell `k` of cell (cx, cy, cz); k = -1 is the cell itself.
__device__ __forceinline__ uint32_t visit_cell(const GridGeom& g, uint32_t c, uint32_t cx, uint32_t cy, uint32_t cz,
                                               int k) {
    if (k < 0) return c;
    return encode(g, wrap_add(cx, g.full[k][0], g.n[0]), wrap_add(cy, g.full[k][1], g.n[1]),
                  wrap_add(cz, g.full[k][2], g.n[2]));
}

// min_image1 for |d| <= 0.49 L without the division: the rounded quotient
// is zero there and d - L * 0 is d itself, sign of a zero included.
__device__ __forceinline__ double near_image(double d, double L) {
    return fabs(d) <= xmul(0.49, L) ? d : min_image1(d, L);
}

// Sum over the kAdjLanes lanes of one atom (a butterfly: every lane ends
// with the same bits, and the association is fixed, so recomputed ticks
// reproduce the forward pass exactly).
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
    for (int o = kAdjLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, kAdjLanes);
    return v;
}
// Integer partials: any order gives the same sum.
__device__ __forceinline__ long long lane_sum_ll(long long v) {
#pragma unroll
    for (int o = kAdjLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, kAdjLanes);
    return v;
}

// ---------------------------------------------------------------------------
// Kernels (slot order unless noted).

// Handle state (cell-sorted) -> slot order.
__global__ void k_adj_import(StateBuf b, uint32_t n, Vec3Field x, Vec3Field v, Vec3Field a, uint8_t* elem,
                             double* charge, double* mass, double* inv_mass, uint8_t* kind) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t s = b.slot[p];
    x.c(0, s) = b.x[p];
    x.c(1, s) = b.y[p];
    x.c(2, s) = b.z[p];
    v.c(0, s) = b.vx[p];
    v.c(1, s) = b.vy[p];
    v.c(2, s) = b.vz[p];
    a.c(0, s) = b.ax[p];
    a.c(1, s) = b.ay[p];
    a.c(2, s) = b.az[p];
    elem[s] = b.elem[p];
    charge[s] = b.charge[p];
    mass[s] = b.mass[p];
    inv_mass[s] = b.inv_mass[p];
    kind[s] = b.kind[p];
}

// First kick, drift, wrap (integrate.rs:39-43, 62-66; boundary.rs:28-34) and
// the cell key of the new position; optionally saves the position.
__global__ void k_adj_kick_drift(GridGeom g, uint32_t n, Vec3Field x, Vec3Field v, Vec3Field a, double half_dt,
                                 double dt, double hx, double hy, double hz, int wrap, uint32_t* key, Vec3Field xsave,
                                 uint32_t* err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double hb[3] = {hx, hy, hz};
    double p[3];
    for (int k = 0; k < 3; ++k) {
        double vk = xadd(v.c(k, i), xmul(a.c(k, i), half_dt));
        double xk = xadd(x.c(k, i), xmul(vk, dt));
        if (wrap) xk = xsub(rem_euclid(xk, xmul(2.0, hb[k])), hb[k]);
        v.c(k, i) = vk;
        x.c(k, i) = xk;
        p[k] = xk;
        if (xsave.p) xsave.c(k, i) = xk;
    }
    if (!(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]))) atomicOr(err, kErrNonFinite);
    key[i] = cell_of(g, p[0], p[1], p[2]);
}

__global__ void k_adj_keys(GridGeom g, uint32_t n, Vec3Field x, uint32_t* key) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = cell_of(g, x.c(0, i), x.c(1, i), x.c(2, i));
}

// Cell-sorted copies of what the pair loops read (p = sorted position).
// With an adjoint, also W/m = (La + half_dt Lv) / m per atom.
__global__ void k_adj_stage(uint32_t n, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ key,
                            Vec3Field x, const uint8_t* __restrict__ elem, const double* __restrict__ charge,
                            const double* __restrict__ mass, const double* __restrict__ inv_mass, Vec3Field xs,
                            uint8_t* es, double* qs, double* ms, uint32_t* ks, Vec3Field Lv, Vec3Field La,
                            double half_dt, Vec3Field ws, const uint8_t* __restrict__ kind, uint8_t* kinds) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t i = perm[p];
    for (int k = 0; k < 3; ++k) xs.c(k, p) = x.c(k, i);
    es[p] = elem[i];
    if (kinds) kinds[p] = kind[i];
    qs[p] = charge[i];
    ms[p] = mass[i];
    ks[p] = key[i];
    if (ws.p) {
        double im = inv_mass[i];
        for (int k = 0; k < 3; ++k) ws.c(k, p) = (La.c(k, i) + half_dt * Lv.c(k, i)) * im;
    }
}

// Forward force pass + second kick.  kAdjLanes lanes own atom perm[p]: lane
// l visits the neighbour cells l - 1, l - 1 + kAdjLanes, ... (the atom's own
// cell first) in the reference's per-pair FP64 arithmetic, and lane_sum
// combines their accelerations; the potential and the smoothed histogram
// take each pair-list entry once (canonical half-shell visits, or j > p
// within a cell).  One histogram per warp in shared memory, integer counts.
// F32: the mixed method's pair law (pair_f32 on the FP64 displacement
// rounded to FP32, the kinds' FP32 pair table) with the force summed in
// 2^-32 fixed point and a = F 2^-32 / m as the list path's finish takes it;
// the potential sums the FP32 pair energies in FP64.
template <bool OBS, bool GR, bool F32>
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_force(GridGeom g, uint32_t n, LawF64 L, const double* __restrict__ psig, const double* __restrict__ peps,
                const uint32_t* __restrict__ start, const uint32_t* __restrict__ ks, Vec3Field xs,
                const uint8_t* __restrict__ es, const double* __restrict__ qs, const double* __restrict__ ms,
                const uint32_t* __restrict__ perm, const double* __restrict__ inv_mass, Vec3Field v, Vec3Field a,
                double half_dt, double* __restrict__ vpart, GrSpec gs, double* __restrict__ hpart, LawF32 L32,
                const PairF* __restrict__ tabf, const uint8_t* __restrict__ kinds, uint32_t* __restrict__ err) {
    constexpr int kWarps = kAdjThreads / 32;
    __shared__ double shd[kWarps];
    __shared__ unsigned long long hist[GR ? kWarps : 1][GR ? kAdjMaxBins : 1];
    if (GR)
        for (int k = threadIdx.x; k < kWarps * gs.bins; k += kAdjThreads) hist[k / gs.bins][k % gs.bins] = 0ull;
    if (GR) __syncthreads();
    unsigned long long* wh = hist[GR ? threadIdx.x / 32 : 0];
    const uint32_t t = blockIdx.x * kAdjThreads + threadIdx.x;
    const uint32_t p = t / kAdjLanes;
    const int lane = (int)(t % kAdjLanes);
    double V = 0.0;
    double ax = 0.0, ay = 0.0, az = 0.0;
    long long fx = 0, fy = 0, fz = 0;
    if (p < n) {
        uint32_t c = ks[p], cx, cy, cz;
        decode(g, c, cx, cy, cz);
        double xi = xs.c(0, p), yi = xs.c(1, p), zi = xs.c(2, p);
        int ti = es[p];
        const int kti = F32 ? (int)kinds[p] * L32.nkinds : 0;
        double qi = qs[p], mi = ms[p];
        double inv_mi = inv_mass[perm[p]];
        for (int k = lane - 1; k < g.nfull; k += kAdjLanes) {
            uint32_t B = visit_cell(g, c, cx, cy, cz, k);
            bool half = k < g.nhalf;
            uint32_t lo = start[B], hi = start[B + 1];
            for (uint32_t q = lo; q < hi; ++q) {
                if (q == p) continue;
                double dx = near_image(xsub(xi, xs.c(0, q)), L.box[0]);
                double dy = near_image(xsub(yi, xs.c(1, q)), L.box[1]);
                double dz = near_image(xsub(zi, xs.c(2, q)), L.box[2]);
                double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                if (d2 >= L.rc2) continue;
                double d = xsqrt(d2);
                if (d <= kEpsF64) continue;
                bool count = (k < 0) ? (q > p) : half;
                double fmag = 0.0, Vij = 0.0;
                if (F32) {
                    const float fdx = (float)dx, fdy = (float)dy, fdz = (float)dz;
                    float fs, vf;
                    pair_f32(L32, tabf[kti + kinds[q]], dist2(fdx, fdy, fdz), fs, vf);
                    long long qx, qy, qz;
                    quant3(fmul(fdx, fs), fmul(fdy, fs), fmul(fdz, fs), qx, qy, qz, err);
                    fx += qx;
                    fy += qy;
                    fz += qz;
                    Vij = (double)vf;
                } else {
                    int tj = es[q];
                    pair_f64(L, d, psig[ti * kNElem + tj], peps[ti * kNElem + tj], qi, qs[q], mi, ms[q], fmag, Vij);
                }
                if (OBS && count) V = xadd(V, Vij);
                if (GR && count) {
                    int k0 = (int)ceil((d - gs.reach) / gs.dr - 0.5), k1 = (int)floor((d + gs.reach) / gs.dr - 0.5);
                    k0 = k0 < 0 ? 0 : k0;
                    k1 = k1 > gs.bins - 1 ? gs.bins - 1 : k1;
                    for (int bb = k0; bb <= k1; ++bb) {
                        double z = d - (bb + 0.5) * gs.dr;
                        if (fabs(z) >= gs.reach) continue;
                        double G = exp(z * z * gs.c2);
                        atomicAdd(&wh[bb], (unsigned long long)llrint(G * kHistScale));
                    }
                }
                if (!F32 && fmag != 0.0) {
                    double inv = xdiv(1.0, d);
                    ax = xadd(ax, xmul(xmul(xmul(dx, inv), fmag), inv_mi));
                    ay = xadd(ay, xmul(xmul(xmul(dy, inv), fmag), inv_mi));
                    az = xadd(az, xmul(xmul(xmul(dz, inv), fmag), inv_mi));
                }
            }
        }
    }
    // every lane of an atom is in the same warp and takes part
    if (F32) {
        fx = lane_sum_ll(fx);
        fy = lane_sum_ll(fy);
        fz = lane_sum_ll(fz);
        if (p < n) {
            const double im = inv_mass[perm[p]];
            ax = xmul(xmul(__ll2double_rn(fx), kFixInv), im);
            ay = xmul(xmul(__ll2double_rn(fy), kFixInv), im);
            az = xmul(xmul(__ll2double_rn(fz), kFixInv), im);
        }
    } else {
        ax = lane_sum(ax);
        ay = lane_sum(ay);
        az = lane_sum(az);
    }
    if (p < n && lane == 0) {
        uint32_t i = perm[p];
        a.c(0, i) = ax;
        a.c(1, i) = ay;
        a.c(2, i) = az;
        v.c(0, i) = xadd(v.c(0, i), xmul(ax, half_dt));
        v.c(1, i) = xadd(v.c(1, i), xmul(ay, half_dt));
        v.c(2, i) = xadd(v.c(2, i), xmul(az, half_dt));
    }
    if (OBS) {
        V = block_sum<kAdjThreads>(V, shd);
        if (threadIdx.x == 0) vpart[blockIdx.x] = V;
    }
    if (GR) {
        __syncthreads();
        for (int k = threadIdx.x; k < gs.bins; k += kAdjThreads) {
            unsigned long long s = 0ull;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) s += hist[w][k];
            hpart[(size_t)blockIdx.x * gs.bins + k] = (double)s * kHistInv;
        }
    }
}

// hacc[k] += sum over blocks of hpart[b][k], blocks in order.
__global__ void k_adj_gr_finalize(int bins, int nblocks, const double* __restrict__ hpart, double* hacc) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= bins) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += hpart[(size_t)b * bins + k];
    hacc[k] += s;
}

// Backward pass of one tick (see the file comment).  P rows: sigma, epsilon,
// rc_lj, rc_coulomb, rc_gravity partials per atom.
template <bool GR>
__global__ void __launch_bounds__(kAdjThreads)
    k_adj_back(GridGeom g, uint32_t n, LawF64 L, const double* __restrict__ psig, const double* __restrict__ peps,
               const double* __restrict__ epsk, const uint32_t* __restrict__ start, const uint32_t* __restrict__ ks,
               Vec3Field xs, Vec3Field ws, const uint8_t* __restrict__ es, const double* __restrict__ qs,
               const double* __restrict__ ms, const uint32_t* __restrict__ perm, Vec3Field Lx, Vec3Field Lv,
               Vec3Field La, double* __restrict__ P, size_t cap, const double* __restrict__ alpha_t, double dt,
               double half_dt, GrSpec gs, const double* __restrict__ bw) {
    const uint32_t t = blockIdx.x * kAdjThreads + threadIdx.x;
    const uint32_t p = t / kAdjLanes;
    const int lane = (int)(t % kAdjLanes);
    double gx = 0.0, gy = 0.0, gz = 0.0;
    double Ps = 0.0, Pe = 0.0, Pr0 = 0.0, Pr1 = 0.0, Pr2 = 0.0;
    if (p < n) {
    const double alpha = *alpha_t;
    uint32_t c = ks[p], cx, cy, cz;
    decode(g, c, cx, cy, cz);
    double xi = xs.c(0, p), yi = xs.c(1, p), zi = xs.c(2, p);
    double wxi = ws.c(0, p), wyi = ws.c(1, p), wzi = ws.c(2, p);
    int ti = es[p];
    double qi = qs[p], mi = ms[p];
    double ehalf_base = 0.5 / epsk[ti];
    for (int k = lane - 1; k < g.nfull; k += kAdjLanes) {
        uint32_t B = visit_cell(g, c, cx, cy, cz, k);
        uint32_t lo = start[B], hi = start[B + 1];
        for (uint32_t q = lo; q < hi; ++q) {
            if (q == p) continue;
            double dx = near_image(xi - xs.c(0, q), L.box[0]);
            double dy = near_image(yi - xs.c(1, q), L.box[1]);
            double dz = near_image(zi - xs.c(2, q), L.box[2]);
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 >= L.rc2) continue;
            double d = sqrt(d2);
            if (d <= kEpsF64) continue;
            double inv = 1.0 / d;
            double nx = dx * inv, ny = dy * inv, nz = dz * inv;
            double ux = wxi - ws.c(0, q), uy = wyi - ws.c(1, q), uz = wzi - ws.c(2, q);
            double rho = nx * ux + ny * uy + nz * uz;
            int tj = es[q];
            double sg = psig[ti * kNElem + tj], ep = peps[ti * kNElem + tj];
            PairG G = pair_grad(L, d, sg, ep, qi, qs[q], mi, ms[q]);
            double psi = 0.0;
            if (GR) {
                int k0 = (int)ceil((d - gs.reach) / gs.dr - 0.5), k1 = (int)floor((d + gs.reach) / gs.dr - 0.5);
                k0 = k0 < 0 ? 0 : k0;
                k1 = k1 > gs.bins - 1 ? gs.bins - 1 : k1;
                for (int b = k0; b <= k1; ++b) {
                    double z = d - (b + 0.5) * gs.dr;
                    if (fabs(z) >= gs.reach) continue;
                    psi += bw[b] * (2.0 * gs.c2 * z) * exp(z * z * gs.c2);
                }
            }
            double c1 = rho * G.fd + alpha * G.Ud + psi;
            double c2 = G.f * inv;
            gx += c1 * nx + c2 * (ux - rho * nx);
            gy += c1 * ny + c2 * (uy - rho * ny);
            gz += c1 * nz + c2 * (uz - rho * nz);
            Ps += 0.5 * (rho * G.fs + alpha * G.Us);
            Pe += ep * ehalf_base * (rho * G.fe + alpha * G.Ue);
            Pr0 += 0.5 * (rho * G.frc[0] + alpha * G.Urc[0]);
            Pr1 += 0.5 * (rho * G.frc[1] + alpha * G.Urc[1]);
            Pr2 += 0.5 * (rho * G.frc[2] + alpha * G.Urc[2]);
        }
    }
    }
    // every lane of an atom is in the same warp and takes part
    gx = lane_sum(gx);
    gy = lane_sum(gy);
    gz = lane_sum(gz);
    Ps = lane_sum(Ps);
    Pe = lane_sum(Pe);
    Pr0 = lane_sum(Pr0);
    Pr1 = lane_sum(Pr1);
    Pr2 = lane_sum(Pr2);
    if (p >= n || lane != 0) return;
    uint32_t i = perm[p];
    double g3[3] = {gx, gy, gz};
    for (int k = 0; k < 3; ++k) {
        double lx = Lx.c(k, i) + g3[k];
        double lvh = Lv.c(k, i) + dt * lx;
        Lx.c(k, i) = lx;
        Lv.c(k, i) = lvh;
        La.c(k, i) = half_dt * lvh;
    }
    P[0 * cap + i] += Ps;
    P[1 * cap + i] += Pe;
    P[2 * cap + i] += Pr0;
    P[3 * cap + i] += Pr1;
    P[4 * cap + i] += Pr2;
}

// out[e] = sum of sigma partials of element e, out[10 + e] epsilon partials,
// out[20..22] the cutoff partials; one block per output, fixed order.
__global__ void __launch_bounds__(256) k_adj_reduce(uint32_t n, const uint8_t* __restrict__ elem,
                                                    const double* __restrict__ P, size_t cap, double* out) {
    __shared__ double sh[256 / 32];
    int o = blockIdx.x;
    int row = o < kNElem ? 0 : (o < 2 * kNElem ? 1 : 2 + (o - 2 * kNElem));
    int e = o < 2 * kNElem ? o % kNElem : -1;
    double s = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += 256)
        if (e < 0 || elem[i] == e) s += P[(size_t)row * cap + i];
    s = block_sum<256>(s, sh);
    if (threadIdx.x == 0) out[o] = s;
}

__global__ void k_adj_export(uint32_t n, Vec3Field f, double* aos) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 3; ++k) aos[3 * (size_t)i + k] = f.c(k, i);
}

}  // namespace

// Buffers of the adjoint, owned by one handle.
struct AdjBuffers {
    size_t cap = 0, n = 0;
    int T = 0, K = 0, nck = 0, bins = 0, every = 1, samples = 0;
    int cap_T = 0, cap_ck = 0, cap_K = 0, cap_bins = 0;
    double gr_rmax = 0, gr_width = 0, gr_support = 0;
    bool ready = false;
    bool f32 = false;  // the forward in the mixed method (a handle of mixed precision)
    uint8_t *kind = nullptr, *kinds = nullptr;  // kind per slot, per sorted position (F32 forward)
    double *S = nullptr, *Ladj = nullptr, *P = nullptr, *ck = nullptr, *seg = nullptr;
    double *xs = nullptr, *ws = nullptr, *qs = nullptr, *ms = nullptr;
    double *charge = nullptr, *mass = nullptr, *inv_mass = nullptr;
    uint8_t *elem = nullptr, *es = nullptr;
    uint32_t *key = nullptr, *perm = nullptr, *ks = nullptr;
    double *vpart = nullptr, *dV = nullptr, *alpha = nullptr, *bw = nullptr, *hpart = nullptr, *hacc = nullptr;
    double *tab = nullptr;  // psig[100], peps[100], epsk[10], out[kNOut]
    CellList cl;
    std::vector<void*> owned;
};

static void adj_release(AdjBuffers* A) {
    for (void* p : A->owned) cudaFree(p);
    A->owned.clear();
    cells_free(A->cl);
    A->cl = CellList();
}

void adjoint_free(gx_handle* h) {
    if (!h || !h->adj) return;
    AdjBuffers* A = static_cast<AdjBuffers*>(h->adj);
    adj_release(A);
    delete A;
    h->adj = nullptr;
}

namespace {

int adj_alloc(gx_handle* h, AdjBuffers* A, size_t n, int T, int K, int bins) {
    int nck = (T + K - 1) / K;
    if (n <= A->cap && T <= A->cap_T && nck <= A->cap_ck && K <= A->cap_K && bins <= A->cap_bins && A->tab) return GX_OK;
    for (void* p : A->owned) cudaFree(p);
    A->owned.clear();
    size_t cap = n < 1 ? 1 : n;
    cap = (cap + 31) & ~(size_t)31;
    size_t nb = nblk(cap * kAdjLanes, kAdjThreads);
    int binc = bins < 1 ? 1 : bins;
    auto get = [&](void** p, size_t bytes) -> int {
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
        if (e != cudaSuccess) return cuda_err(h, e, "adjoint buffers");
        A->owned.push_back(*p);
        return GX_OK;
    };
    int rc = 0;
    rc |= get((void**)&A->S, 9 * cap * sizeof(double));
    rc |= get((void**)&A->Ladj, 9 * cap * sizeof(double));
    rc |= get((void**)&A->P, 5 * cap * sizeof(double));
    rc |= get((void**)&A->ck, (size_t)nck * 9 * cap * sizeof(double));
    rc |= get((void**)&A->seg, (size_t)K * 3 * cap * sizeof(double));
    rc |= get((void**)&A->xs, 3 * cap * sizeof(double));
    rc |= get((void**)&A->ws, 3 * cap * sizeof(double));
    rc |= get((void**)&A->qs, cap * sizeof(double));
    rc |= get((void**)&A->ms, cap * sizeof(double));
    rc |= get((void**)&A->charge, cap * sizeof(double));
    rc |= get((void**)&A->mass, cap * sizeof(double));
    rc |= get((void**)&A->inv_mass, cap * sizeof(double));
    rc |= get((void**)&A->elem, cap);
    rc |= get((void**)&A->es, cap);
    rc |= get((void**)&A->kind, cap);
    rc |= get((void**)&A->kinds, cap);
    rc |= get((void**)&A->key, cap * sizeof(uint32_t));
    rc |= get((void**)&A->perm, cap * sizeof(uint32_t));
    rc |= get((void**)&A->ks, cap * sizeof(uint32_t));
    rc |= get((void**)&A->vpart, nb * sizeof(double));
    rc |= get((void**)&A->dV, (size_t)T * sizeof(double));
    rc |= get((void**)&A->alpha, (size_t)T * sizeof(double));
    rc |= get((void**)&A->bw, (size_t)binc * sizeof(double));
    rc |= get((void**)&A->hpart, nb * (size_t)binc * sizeof(double));
    rc |= get((void**)&A->hacc, (size_t)binc * sizeof(double));
    rc |= get((void**)&A->tab, (2 * kNElem * kNElem + kNElem + kNOut) * sizeof(double));
    if (rc) {
        for (void* p : A->owned) cudaFree(p);
        A->owned.clear();
        A->cap = 0;
        A->tab = nullptr;
        return rc;
    }
    A->cap = cap;
    A->cap_T = T;
    A->cap_ck = nck;
    A->cap_K = K;
    A->cap_bins = binc;
    return GX_OK;
}

Vec3Field field(double* base, size_t cap) { return Vec3Field{base, cap}; }

GrSpec gr_spec(const AdjBuffers* A) {
    GrSpec g;
    g.bins = A->bins;
    g.dr = A->bins > 0 ? A->gr_rmax / A->bins : 1.0;
    g.width = A->gr_width;
    g.reach = A->gr_support * A->gr_width;
    g.c2 = A->gr_width > 0 ? -0.5 / (A->gr_width * A->gr_width) : 0.0;
    return g;
}

// One forward tick in slot order.  obs: record V_t (and the histogram on
// sampled ticks); xsave: keep x_t; with_force false stops after the drift.
int adj_tick(gx_handle* h, AdjBuffers* A, int t, bool obs, double* xsave, bool with_force) {
    const uint32_t n = (uint32_t)A->n;
    const size_t cap = A->cap;
    const GridGeom& g = h->fgrid;
    Vec3Field x = field(A->S, cap), v = field(A->S + 3 * cap, cap), a = field(A->S + 6 * cap, cap);
    double half_dt = 0.5 * h->p.dt;
    GX_LAUNCH(h, k_adj_kick_drift, nblk(n, 256), 256, g, n, x, v, a, half_dt, h->p.dt, h->p.box[0] * 0.5,
              h->p.box[1] * 0.5, h->p.box[2] * 0.5, h->p.enable_boundaries ? 1 : 0, A->key,
              field(xsave, cap), h->derr);
    if (!with_force) return GX_OK;
    int rc = counting_sort(h, A->cl, g.ncell, A->key, n, A->perm);
    if (rc) return rc;
    Vec3Field xs = field(A->xs, cap), none = field(nullptr, cap);
    GX_LAUNCH(h, k_adj_stage, nblk(n, 256), 256, n, A->perm, A->key, x, A->elem, A->charge, A->mass, A->inv_mass,
              xs, A->es, A->qs, A->ms, A->ks, none, none, half_dt, none, A->kind, A->f32 ? A->kinds : nullptr);
    LawF64 L = make_law64(h);
    const double* psig = A->tab;
    const double* peps = A->tab + kNElem * kNElem;
    GrSpec gs = gr_spec(A);
    unsigned nb = nblk((size_t)n * kAdjLanes, kAdjThreads);
    bool gr = obs && A->bins > 0 && (t % A->every) == 0;
    auto kern = A->f32 ? (!obs ? k_adj_force<false, false, true>
                               : (gr ? k_adj_force<true, true, true> : k_adj_force<true, false, true>))
                       : (!obs ? k_adj_force<false, false, false>
                               : (gr ? k_adj_force<true, true, false> : k_adj_force<true, false, false>));
    GX_LAUNCH(h, kern, nb, kAdjThreads, g, n, L, psig, peps, A->cl.start, A->ks, xs, A->es, A->qs, A->ms, A->perm,
              A->inv_mass, v, a, half_dt, A->vpart, gs, A->hpart, make_law32(h), h->d_pairf, A->kinds, h->derr);
    if (obs) {
        launch_finalize_sum(h, A->vpart, (int)nb, A->dV + (t - 1));
        if (gr) {
            GX_LAUNCH(h, k_adj_gr_finalize, nblk(A->bins, 256), 256, A->bins, (int)nb, A->hpart, A->hacc);
            A->samples++;
        }
    }
    return GX_OK;
}

double gr_norm(const gx_handle* h, const AdjBuffers* A, int k) {
    const double pi = 3.14159265358979323846;
    double vol = h->p.box[0] * h->p.box[1] * h->p.box[2];
    double npair = 0.5 * (double)A->n * ((double)A->n - 1.0);
    double dr = A->gr_rmax / A->bins, r = (k + 0.5) * dr;
    return vol / (npair * 4.0 * pi * r * r * std::sqrt(2.0 * pi) * A->gr_width);
}

int check_err(gx_handle* h) {
    uint32_t e = 0;
    GX_CUDA(h, cudaMemcpyAsync(&e, h->derr, sizeof e, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    if (e & kErrNonFinite) {
        cudaMemsetAsync(h->derr, 0, sizeof(uint32_t), h->stream);
        return set_err(h, GX_ERR_NONFINITE, "non-finite position in the adjoint trajectory");
    }
    if (e & kErrSaturation) {  // the fixed-point force of the mixed forward
        cudaMemsetAsync(h->derr, 0, sizeof(uint32_t), h->stream);
        return set_err(h, GX_ERR_SATURATION, "fixed-point force saturated in the adjoint trajectory");
    }
    return GX_OK;
}

}  // namespace
}  // namespace gx

using namespace gx;

int gx_adjoint_forward(gx_handle* h, const gx_adjoint_spec* spec, double* potential, double* gr) {
    if (!h || !spec || !potential) return GX_ERR_ARG;
    int rc = GX_OK;
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    if (h->n == 0) return set_err(h, GX_ERR_ARG, "the adjoint needs at least one atom");
    if ((rc = settle_step_errors(h))) return rc;  // a queued step's error first: the word is cleared below
    h->nl_fresh = false;  // conservative: the passes below may reorder or move the resident state
    if (spec->nsteps < 1 || spec->checkpoint_every < 1) return set_err(h, GX_ERR_ARG, "nsteps and checkpoint_every must be >= 1");
    if (spec->gr_bins < 0 || spec->gr_bins > kAdjMaxBins) return set_err(h, GX_ERR_ARG, "gr_bins must be in [0, 512]");
    if (spec->gr_bins > 0) {
        if (spec->gr_every < 1 || !(spec->gr_rmax > 0.0) || !(spec->gr_width > 0.0) || !(spec->gr_support > 0.0))
            return set_err(h, GX_ERR_ARG, "g(r) spec needs gr_every >= 1 and positive rmax, width, support");
        if (spec->gr_rmax + spec->gr_support * spec->gr_width > h->fs.rc)
            return set_err(h, GX_ERR_ARG, "gr_rmax + gr_support * gr_width exceeds the force cutoff");
    }
    if (h->p.enable_thermostat || h->p.enable_bond_interaction)
        return set_err(h, GX_ERR_UNSUPPORTED, "the adjoint covers NVE ticks without the bond spring");
    for (int e = 0; e < kNElem; ++e)
        if (!(h->p.epsilon_k[e] > 0.0)) return set_err(h, GX_ERR_UNSUPPORTED, "the adjoint needs every epsilon_k > 0");
    if (h->n >= (1u << 31)) return set_err(h, GX_ERR_CAPACITY, "too many atoms");
    if (h->precision == GX_MIXED && h->nkinds > kMaxKinds)
        return set_err(h, GX_ERR_UNSUPPORTED, "the mixed forward supports at most 16 distinct (element, charge) kinds");
    // NVE only, so no Berendsen scale can be pending on the handle's velocities.
    if (!h->adj) h->adj = new AdjBuffers();
    AdjBuffers* A = static_cast<AdjBuffers*>(h->adj);
    A->ready = false;
    const int T = spec->nsteps, K = spec->checkpoint_every;
    if ((rc = adj_alloc(h, A, h->n, T, K, spec->gr_bins))) return rc;
    A->T = T;
    A->K = K;
    A->nck = (T + K - 1) / K;
    A->bins = spec->gr_bins;
    A->every = spec->gr_bins > 0 ? spec->gr_every : 1;
    A->gr_rmax = spec->gr_rmax;
    A->gr_width = spec->gr_width;
    A->gr_support = spec->gr_support;
    A->samples = 0;
    A->n = h->n;
    A->f32 = h->precision == GX_MIXED;
    const uint32_t n = (uint32_t)h->n;
    const size_t cap = A->cap;
    // pair table, epsilon_k
    std::vector<double> tab(2 * kNElem * kNElem + kNElem, 0.0);
    std::memcpy(tab.data(), h->fs.pair_sigma, sizeof h->fs.pair_sigma);
    std::memcpy(tab.data() + kNElem * kNElem, h->fs.pair_eps, sizeof h->fs.pair_eps);
    for (int e = 0; e < kNElem; ++e) tab[2 * kNElem * kNElem + e] = h->p.epsilon_k[e];
    GX_CUDA(h, cudaMemcpyAsync(A->tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    StateBuf& b = h->buf[h->cur];
    GX_LAUNCH(h, k_adj_import, nblk(n, 256), 256, b, n, field(A->S, cap), field(A->S + 3 * cap, cap),
              field(A->S + 6 * cap, cap), A->elem, A->charge, A->mass, A->inv_mass, A->kind);
    GX_CUDA(h, cudaMemcpyAsync(A->ck, A->S, 9 * cap * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (A->bins > 0) GX_CUDA(h, cudaMemsetAsync(A->hacc, 0, A->bins * sizeof(double), h->stream));
    for (int t = 1; t <= T; ++t) {
        if ((rc = adj_tick(h, A, t, true, nullptr, true))) return rc;
        if (t % K == 0 && t / K < A->nck)
            GX_CUDA(h, cudaMemcpyAsync(A->ck + (size_t)(t / K) * 9 * cap, A->S, 9 * cap * sizeof(double),
                                       cudaMemcpyDeviceToDevice, h->stream));
    }
    GX_CUDA(h, cudaMemcpyAsync(potential, A->dV, T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    std::vector<double> hacc(A->bins > 0 ? A->bins : 0);
    if (A->bins > 0)
        GX_CUDA(h, cudaMemcpyAsync(hacc.data(), A->hacc, A->bins * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    if ((rc = check_err(h))) return rc;
    if (gr)
        for (int k = 0; k < A->bins; ++k) gr[k] = A->samples ? hacc[k] * gr_norm(h, A, k) / A->samples : 0.0;
    A->ready = true;
    return GX_OK;
}

int gx_adjoint_backward(gx_handle* h, const double* dl_dpotential, const double* dl_dgr, double* grad_sigma,
                        double* grad_epsilon_k, double* grad_pos0, double* grad_vel0, double* grad_acc0) {
    if (!h || !grad_sigma || !grad_epsilon_k) return GX_ERR_ARG;
    AdjBuffers* A = static_cast<AdjBuffers*>(h->adj);
    if (!A || !A->ready) return set_err(h, GX_ERR_STATE, "call gx_adjoint_forward first");
    if (h->n != A->n) return set_err(h, GX_ERR_STATE, "atom count changed since gx_adjoint_forward");
    int rc = settle_step_errors(h);
    if (rc) return rc;
    const uint32_t n = (uint32_t)A->n;
    const size_t cap = A->cap;
    const int T = A->T, K = A->K;
    const GridGeom& g = h->fgrid;
    double half_dt = 0.5 * h->p.dt;
    // cotangents
    std::vector<double> alpha(T, 0.0), bw(A->bins > 0 ? A->bins : 1, 0.0);
    if (dl_dpotential)
        for (int t = 0; t < T; ++t) alpha[t] = dl_dpotential[t];
    if (dl_dgr && A->bins > 0 && A->samples > 0)
        for (int k = 0; k < A->bins; ++k) bw[k] = dl_dgr[k] * gr_norm(h, A, k) / A->samples;
    GX_CUDA(h, cudaMemcpyAsync(A->alpha, alpha.data(), T * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    GX_CUDA(h, cudaMemcpyAsync(A->bw, bw.data(), bw.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    GX_CUDA(h, cudaMemsetAsync(A->Ladj, 0, 9 * cap * sizeof(double), h->stream));
    GX_CUDA(h, cudaMemsetAsync(A->P, 0, 5 * cap * sizeof(double), h->stream));
    Vec3Field Lx = field(A->Ladj, cap), Lv = field(A->Ladj + 3 * cap, cap), La = field(A->Ladj + 6 * cap, cap);
    Vec3Field xs = field(A->xs, cap), ws = field(A->ws, cap);
    LawF64 L = make_law64(h);
    const double* psig = A->tab;
    const double* peps = A->tab + kNElem * kNElem;
    const double* epsk = A->tab + 2 * kNElem * kNElem;
    double* out = A->tab + 2 * kNElem * kNElem + kNElem;
    GrSpec gs = gr_spec(A);
    unsigned nb = nblk((size_t)n * kAdjLanes, kAdjThreads);
    bool has_gr = dl_dgr && A->bins > 0;
    for (int s = A->nck - 1; s >= 0; --s) {
        int t0 = s * K, t1 = t0 + K < T ? t0 + K : T;
        GX_CUDA(h, cudaMemcpyAsync(A->S, A->ck + (size_t)s * 9 * cap, 9 * cap * sizeof(double),
                                   cudaMemcpyDeviceToDevice, h->stream));
        for (int t = t0 + 1; t <= t1; ++t)
            if ((rc = adj_tick(h, A, t, false, A->seg + (size_t)(t - t0 - 1) * 3 * cap, t < t1))) return rc;
        for (int t = t1; t > t0; --t) {
            Vec3Field xt = field(A->seg + (size_t)(t - t0 - 1) * 3 * cap, cap);
            GX_LAUNCH(h, k_adj_keys, nblk(n, 256), 256, g, n, xt, A->key);
            if ((rc = counting_sort(h, A->cl, g.ncell, A->key, n, A->perm))) return rc;
            GX_LAUNCH(h, k_adj_stage, nblk(n, 256), 256, n, A->perm, A->key, xt, A->elem, A->charge, A->mass,
                      A->inv_mass, xs, A->es, A->qs, A->ms, A->ks, Lv, La, half_dt, ws, A->kind, nullptr);
            bool gr = has_gr && (t % A->every) == 0;
            auto kern = gr ? k_adj_back<true> : k_adj_back<false>;
            GX_LAUNCH(h, kern, nb, kAdjThreads, g, n, L, psig, peps, epsk, A->cl.start, A->ks, xs, ws, A->es, A->qs,
                      A->ms, A->perm, Lx, Lv, La, A->P, cap, A->alpha + (t - 1), h->p.dt, half_dt, gs, A->bw);
        }
    }
    GX_LAUNCH(h, k_adj_reduce, kNOut, 256, n, A->elem, A->P, cap, out);
    double sums[kNOut];
    GX_CUDA(h, cudaMemcpyAsync(sums, out, sizeof sums, cudaMemcpyDeviceToHost, h->stream));
    double* dsts[3] = {grad_pos0, grad_vel0, grad_acc0};
    double* stage = A->xs;  // 3 * cap, free once the sweep is done
    for (int q = 0; q < 3; ++q) {
        if (!dsts[q] || !n) continue;
        GX_LAUNCH(h, k_adj_export, nblk(n, 256), 256, n, field(A->Ladj + (size_t)q * 3 * cap, cap), stage);
        GX_CUDA(h, cudaMemcpyAsync(dsts[q], stage, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    if ((rc = check_err(h))) return rc;
    // The cutoffs: lj_rc = max(lj_cutoff_factor, 1) * max pair sigma (LjTable::new,
    // forces.rs:223-237), coulomb/gravity rc = max(factor, 1) * max sigma
    // (systems/forces.rs:108-116); the derivative goes to the first element
    // attaining the largest sigma.
    int mstar = 0;
    for (int e = 1; e < kNElem; ++e)
        if (h->p.sigma[e] > h->p.sigma[mstar]) mstar = e;
    double drc = std::fmax(h->p.lj_cutoff_factor, 1.0) * sums[2 * kNElem + 0];
    if (h->p.enable_electrostatics) drc += std::fmax(h->p.coulomb_cutoff, 1.0) * sums[2 * kNElem + 1];
    if (h->p.enable_gravity) drc += std::fmax(h->p.gravity_cutoff, 1.0) * sums[2 * kNElem + 2];
    for (int e = 0; e < kNElem; ++e) {
        grad_sigma[e] = sums[e] + (e == mstar ? drc : 0.0);
        grad_epsilon_k[e] = sums[kNElem + e];
    }
    return GX_OK;
}
