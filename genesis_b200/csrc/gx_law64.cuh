// gx_law64.cuh -- the FP64 pair law shared by the plain force pass and the
// adjoint's forward recomputation (src/physics/forces.rs:270-353,
// src/systems/forces.rs:270-299), evaluated with the reference's operation
// order so every pair's force and energy are bit-identical to it.
#pragma once

#include "gx_internal.cuh"

namespace gx {

struct LawF64 {
    double lj_rc, lj_ron, coul_rc, coul_ron, grav_rc, grav_ron;
    double rc2;
    double k_e, G;
    double box[3];
    int coul, grav;
};

// smooth_cutoff, src/physics/forces.rs:302-318 (exact FP64).
__device__ __forceinline__ void smooth_f64(double r, double ron, double rc, double& sw, double& dsw) {
    if (r <= ron) { sw = 1.0; dsw = 0.0; return; }
    if (r >= rc) { sw = 0.0; dsw = 0.0; return; }
    double w = xsub(rc, ron);
    double u = xdiv(xsub(r, ron), w);
    double u2 = xmul(u, u);
    double u3 = xmul(u2, u);
    double u4 = xmul(u3, u);
    double u5 = xmul(u4, u);
    sw = xsub(xadd(xsub(1.0, xmul(10.0, u3)), xmul(15.0, u4)), xmul(6.0, u5));
    double omu = xsub(1.0, u);
    dsw = xdiv(xmul(xmul(xmul(-30.0, u2), omu), omu), w);
}

// One pair's LJ + Coulomb + gravity scalar (systems/forces.rs:270-299), exact.
// e24s = (24 ep) / sg, which depends on the element pair only: a caller may
// pass it from a table computed with the same two IEEE operations (the same
// bits) instead of dividing per pair.
__device__ __forceinline__ void pair_f64_e24(const LawF64& L, double d, double sg, double ep, double e24s, double qa,
                                             double qb, double ma, double mb, double& fmag, double& V) {
    fmag = 0.0;
    double sw, dsw;
    if (d < L.lj_rc) {  // force_switched_scalar, forces.rs:270-275; lj_raw :346-353
        double r = fmax(d, xmul(0.5, sg));
        double s = xdiv(sg, r);
        double s6 = xmul(xmul(xmul(xmul(xmul(s, s), s), s), s), s);
        double s12 = xmul(s6, s6);
        double v = xmul(xmul(4.0, ep), xsub(s12, s6));
        double m = xmul(xmul(e24s, s), xsub(xmul(2.0, s12), s6));
        smooth_f64(r, L.lj_ron, L.lj_rc, sw, dsw);
        fmag = xadd(fmag, xsub(xmul(m, sw), xmul(v, dsw)));
        V = xadd(V, xmul(v, sw));
    }
    if (L.coul && d < L.coul_rc) {  // :282-289, coulomb_raw :330-333
        double r = fmax(d, 0.5);
        double q = xmul(xmul(L.k_e, qa), qb);
        double m = xdiv(q, xmul(r, r));
        double v = xdiv(q, r);
        smooth_f64(d, L.coul_ron, L.coul_rc, sw, dsw);
        fmag = xadd(fmag, xsub(xmul(m, sw), xmul(v, dsw)));
        V = xadd(V, xmul(v, sw));
    }
    if (L.grav && d < L.grav_rc) {  // :292-299, gravity_raw :338-341
        double r = fmax(d, 0.5);
        double mm = xmul(xmul(L.G, ma), mb);
        double m = xdiv(-mm, xmul(r, r));
        double v = xdiv(-mm, r);
        smooth_f64(d, L.grav_ron, L.grav_rc, sw, dsw);
        fmag = xadd(fmag, xsub(xmul(m, sw), xmul(v, dsw)));
        V = xadd(V, xmul(v, sw));
    }
}

__device__ __forceinline__ void pair_f64(const LawF64& L, double d, double sg, double ep, double qa, double qb,
                                         double ma, double mb, double& fmag, double& V) {
    pair_f64_e24(L, d, sg, ep, xdiv(xmul(24.0, ep), sg), qa, qb, ma, mb, fmag, V);
}

inline LawF64 make_law64(const gx_handle* h) {
    LawF64 L;
    L.lj_rc = h->fs.lj_rc;
    L.lj_ron = h->fs.lj_ron;
    L.coul_rc = h->fs.coul_rc;
    L.coul_ron = h->fs.coul_ron;
    L.grav_rc = h->fs.grav_rc;
    L.grav_ron = h->fs.grav_ron;
    L.rc2 = h->fs.rc * h->fs.rc;
    L.k_e = h->p.coulomb_constant;
    L.G = h->p.gravity_constant;
    for (int k = 0; k < 3; ++k) L.box[k] = h->p.box[k];
    L.coul = h->p.enable_electrostatics ? 1 : 0;
    L.grav = h->p.enable_gravity ? 1 : 0;
    return L;
}

}  // namespace gx
