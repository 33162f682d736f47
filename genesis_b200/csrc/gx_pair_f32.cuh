// gx_pair_f32.cuh -- the mixed path's FP32 pair law, shared by its kernels.
//
// One in-cutoff pair: Lennard-Jones with the hardened core r = max(d, σ/2)
// and the quintic switch on [r_on, r_c] (force_switched_scalar, lj_raw,
// smooth_cutoff, switched: src/physics/forces.rs:270-353), plus Coulomb with
// the absolute core max(d, 0.5) and its own switch on d
// (src/systems/forces.rs:282-289), plus gravity -G m_i m_j / r^2 with the
// same core and its own switch (forces.rs:291-299, gravity_raw
// src/physics/forces.rs:338-341).  Returns the force magnitude divided by d
// (so F_vec = delta * fs) and the switched potential.
//
// Every operation is an explicit round-to-nearest intrinsic or fmaf, so the
// compiler has no contraction choices left: all pair kernels produce the same
// bits for the same pair, which keeps the fixed-point sums identical across
// kernel variants and launch shapes.
#pragma once

#include "gx_internal.cuh"

namespace gx {

struct LawF32 {
    float rc2, lj_rc, lj_ron, inv_lj_w, coul_rc, coul_ron, inv_coul_w;
    int coul, nkinds;
    int grav = 0;
    float grav_rc = 0.f, grav_ron = 0.f, inv_grav_w = 0.f;
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// (pi - pj) + shift: exactly antisymmetric under swapping the pair's ends.
__device__ __forceinline__ float delta1(float a, float b, float s) { return fadd(fsub(a, b), s); }
__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
    return fmaf(dz, dz, fmaf(dy, dy, fmul(dx, dx)));
}

// quintic switch 1 - 10u^3 + 15u^4 - 6u^5 and its derivative (per unit u)
__device__ __forceinline__ void switch5(float u, float& sw, float& dsw_du) {
    float u2 = fmul(u, u);
    float p = fmaf(-6.f, u, 15.f);       // 15 - 6u
    p = fmaf(p, u, -10.f);               // -10 + u(15 - 6u)
    sw = fmaf(fmul(u2, u), p, 1.f);
    float omu = fsub(1.f, u);
    dsw_du = fmul(fmul(fmul(-30.f, u2), omu), omu);
}

__device__ __forceinline__ void pair_f32(const LawF32& L, const PairF& t, float d2, float& fs, float& v) {
    float inv_d = rsqrtf(d2);
    float d = fmul(d2, inv_d);
    float f = 0.f;
    v = 0.f;
    if (d < L.lj_rc) {
        bool core = d < t.half_sigma;
        float r = core ? t.half_sigma : d;
        float inv_r = core ? t.inv_half_sigma : inv_d;
        float s = fmul(t.sigma, inv_r);
        float s2 = fmul(s, s);
        float s6 = fmul(fmul(s2, s2), s2);
        float s12 = fmul(s6, s6);
        float vl = fmul(t.eps4, fsub(s12, s6));
        float ml = fmul(fmul(t.eps24, inv_r), fmaf(2.f, s12, -s6));
        // u clamped to [0, 1] instead of branching: S(0) = 1 and S'(0) = -0
        // give f = fmaf(ml, 1, +-0) = ml and v = vl exactly, S(1) = 0 gives
        // zeros, so the result is bit-identical to skipping the switch
        // outside (r_on, r_c) -- and no lane of a warp diverges on it.
        float u = fminf(fmaxf(fmul(fsub(r, L.lj_ron), L.inv_lj_w), 0.f), 1.f);
        float sw, dsdu;
        switch5(u, sw, dsdu);
        float dsw = fmul(dsdu, L.inv_lj_w);
        f = fmaf(ml, sw, -fmul(vl, dsw));
        v = fmul(vl, sw);
    }
    if (L.coul && d < L.coul_rc) {
        float inv_r = d < 0.5f ? 2.f : inv_d;
        float vc = fmul(t.qq, inv_r);
        float mc = fmul(vc, inv_r);
        float u = fminf(fmaxf(fmul(fsub(d, L.coul_ron), L.inv_coul_w), 0.f), 1.f);  // as above
        float sw, dsdu;
        switch5(u, sw, dsdu);
        float dsw = fmul(dsdu, L.inv_coul_w);
        f = fadd(f, fmaf(mc, sw, -fmul(vc, dsw)));
        v = fadd(v, fmul(vc, sw));
    }
    if (L.grav && d < L.grav_rc) {
        float inv_r = d < 0.5f ? 2.f : inv_d;
        float vg = -fmul(t.gm, inv_r);  // attractive
        float mg = fmul(vg, inv_r);
        float u = fminf(fmaxf(fmul(fsub(d, L.grav_ron), L.inv_grav_w), 0.f), 1.f);  // as above
        float sw, dsdu;
        switch5(u, sw, dsdu);
        float dsw = fmul(dsdu, L.inv_grav_w);
        f = fadd(f, fmaf(mg, sw, -fmul(vg, dsw)));
        v = fadd(v, fmul(vg, sw));
    }
    fs = fmul(f, inv_d);
}

// One FP32 value to 2^-32 fixed point; flags saturation / non-finite.
__device__ __forceinline__ long long quant(float v, uint32_t* err) {
    float s = fmul(v, kFixScaleF);
    if (!(fabsf(s) < 9.0e18f)) {
        atomicOr(err, isfinite(v) ? kErrSaturation : kErrNonFinite);
        return 0;
    }
    return __float2ll_rn(s);
}

// The three components of one pair force: quant of each, with one range
// check on the fast path (the same integers and flags as three quant calls;
// a NaN fails the check and takes the per-component path, which flags it).
__device__ __forceinline__ void quant3(float fx, float fy, float fz, long long& qx, long long& qy, long long& qz,
                                       uint32_t* err) {
    const float ux = fmul(fx, kFixScaleF), uy = fmul(fy, kFixScaleF), uz = fmul(fz, kFixScaleF);
    if (fabsf(ux) < 9.0e18f && fabsf(uy) < 9.0e18f && fabsf(uz) < 9.0e18f) {
        qx = __float2ll_rn(ux);
        qy = __float2ll_rn(uy);
        qz = __float2ll_rn(uz);
    } else {
        qx = quant(fx, err);
        qy = quant(fy, err);
        qz = quant(fz, err);
    }
}

LawF32 make_law32(const gx_handle* h);

// Thread-per-atom pair pass with per-thread candidate lists (gx_force_tiled.cu);
// any grid, atom indices below 2^27.
void launch_force_mixed_lists(gx_handle* h, const GridGeom& g, const float4* pos4, const uint32_t* key,
                              const uint32_t* start, uint32_t n, const LawF32& L, const PairF* tab, long long* F,
                              size_t fstride, unsigned long long* vacc, unsigned long long* npairs, uint32_t* err);

// Tiled mixed pair pass (gx_force_tiled.cu); needs >= 3 cells on every axis.
void launch_force_mixed_tiled(gx_handle* h, const GridGeom& g, const float4* pos4, const uint32_t* start,
                              const LawF32& L, const PairF* tab, long long* F, size_t fstride,
                              unsigned long long* vacc, unsigned long long* npairs, uint32_t* err);

// One list entry's pair for the list passes: the law only inside r_c, the
// quantised force summed into `a`, with `far` also subtracted from the far
// end q (half lists), and with `once` the potential and pair count.
struct PairAcc {
    long long fx = 0, fy = 0, fz = 0, vq = 0;
    unsigned int np = 0;  // in-cutoff pairs of one thread (widened when summed)
};

// far != null: also subtract the pair force from the far end q (HALF lists).
__device__ __forceinline__ void nl_pair(const LawF32& L, const PairF* st, int ki, float4 pi, float4 pj, float sx,
                                        float sy, float sz, bool once, PairAcc& a, uint32_t* err,
                                        long long* far = nullptr, uint32_t q = 0, size_t fstride = 0) {
    float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
    float d2 = dist2(dx, dy, dz);
    if (!(d2 < L.rc2) || d2 == 0.f) return;
    float fs, v;
    pair_f32(L, st[ki * L.nkinds + __float_as_int(pj.w)], d2, fs, v);
    long long qx, qy, qz;
    if (far) {
        // The far end's share quantised directly: the conversion rounds to
        // nearest even, which is symmetric in sign, so these are exactly
        // -quant(f) (flags included), and this end subtracts them.
        quant3(-fmul(dx, fs), -fmul(dy, fs), -fmul(dz, fs), qx, qy, qz, err);
        a.fx -= qx;
        a.fy -= qy;
        a.fz -= qz;
        atomicAdd((unsigned long long*)&far[q], (unsigned long long)qx);
        atomicAdd((unsigned long long*)&far[fstride + q], (unsigned long long)qy);
        atomicAdd((unsigned long long*)&far[2 * fstride + q], (unsigned long long)qz);
    } else {
        quant3(fmul(dx, fs), fmul(dy, fs), fmul(dz, fs), qx, qy, qz, err);
        a.fx += qx;
        a.fy += qy;
        a.fz += qz;
    }
    if (once) {
        a.vq += quant(v, err);
        ++a.np;
    }
}

}  // namespace gx
