// oracle_dual.cpp -- forward-mode dual-number reference for the adjoint.
//
// TEST INFRASTRUCTURE ONLY (the checker).  The reference has no derivatives;
// this file restates its NVE tick (src/universe/mod.rs:356-369: kick, drift,
// wrap, forces, kick) with the scalar type as a template parameter.  With
// T = double it performs the same operations in the same order as
// orc_ticks (oracle.cpp), which the tests check bit for bit; with T = Dual
// every quantity carries its 20 partial derivatives with respect to the
// per-element sigma[10] and epsilon_k[10], so the derivative of any output
// is exact up to rounding (no truncation error, unlike finite differences).
//
// The observables are the ones the adjoint differentiates:
//   V_t  the potential energy after tick t (LJ + Coulomb + gravity);
//   g_k  a Gaussian-kernel pair distribution averaged over sampled ticks,
//        g_k = c_k * sum_{pair list, |d - r_k| < R w} exp(-(d - r_k)^2 / (2 w^2)),
//        r_k = (k + 1/2) r_max / K, c_k = L^3 / (N(N-1)/2 * 4 pi r_k^2 * sqrt(2 pi) w).
//
// Non-smooth points take one side: max() passes the derivative of its first
// argument on ties (so the cutoff's derivative goes to the lowest-index
// element with the largest sigma), the hard-core clamp max(d, sigma/2)
// likewise, round()/floor() and rem_euclid's integer part have derivative 0.
#include <cmath>
#include <thread>
#include <vector>

#include "oracle.h"
#include "oracle_grid.h"

namespace {

using orcg::Grid;
using orcg::kEps;

constexpr int ND = 2 * ORC_NELEM;  // d/dsigma[0..9], d/depsilon_k[0..9]

struct Dual {
    double v;
    double d[ND];
    Dual() : v(0.0) {
        for (int k = 0; k < ND; ++k) d[k] = 0.0;
    }
    Dual(double x) : v(x) {  // implicit: constants promote to duals
        for (int k = 0; k < ND; ++k) d[k] = 0.0;
    }
};
inline Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
inline Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
    for (int k = 0; k < ND; ++k) r.d[k] = -a.d[k];
    return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    double inv = 1.0 / b.v;
    for (int k = 0; k < ND; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
inline Dual& operator+=(Dual& a, const Dual& b) {
    a.v = a.v + b.v;
    for (int k = 0; k < ND; ++k) a.d[k] += b.d[k];
    return a;
}

inline double val(double x) { return x; }
inline double val(const Dual& x) { return x.v; }
inline double tsqrt(double x) { return std::sqrt(x); }
inline Dual tsqrt(const Dual& a) {
    Dual r;
    r.v = std::sqrt(a.v);
    double h = 0.5 / r.v;
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * h;
    return r;
}
inline double texp(double x) { return std::exp(x); }
inline Dual texp(const Dual& a) {
    Dual r;
    r.v = std::exp(a.v);
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * r.v;
    return r;
}
// std::fmax's value; the first argument wins ties.
template <class T>
inline T tmax(const T& a, const T& b) {
    return val(b) > val(a) ? b : a;
}
// f64::rem_euclid against a constant period: the integer multiple removed is
// constant, so the derivative passes through unchanged.
inline double rem_euclid_t(double a, double b) { return orcg::rem_euclid(a, b); }
inline Dual rem_euclid_t(const Dual& a, double b) {
    Dual r = a;
    r.v = orcg::rem_euclid(a.v, b);
    return r;
}
template <class T>
inline T min_image_1(const T& d, double L) {  // grid.rs:300-306
    return d - L * std::round(val(d) / L);
}

template <class T>
struct V3T {
    T x, y, z;
};

// LjTable::new (forces.rs:223-237) and ForceSystem::new (systems/forces.rs:100-142)
// with sigma and epsilon_k as variables.
template <class T>
struct SetupT {
    T sig[100], eps[100];
    T lj_rc, lj_ron, coul_rc, coul_ron, grav_rc, grav_ron, rc;
    SetupT(const orc_params* p, const T* sigma, const T* epsk) {
        T max_pair = 0.0;
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) {
                T s = 0.5 * (sigma[i] + sigma[j]);
                T e = p->thermal_constant * tsqrt(epsk[i] * epsk[j]);
                max_pair = tmax(max_pair, s);
                sig[i * 10 + j] = s;
                eps[i * 10 + j] = e;
            }
        lj_rc = std::fmax(p->lj_cutoff_factor, 1.0) * max_pair;
        lj_ron = 0.9 * lj_rc;
        T max_sigma = 0.0;
        for (int i = 0; i < 10; ++i) max_sigma = tmax(max_sigma, sigma[i]);
        coul_rc = p->enable_electrostatics ? T(std::fmax(p->coulomb_cutoff, 1.0) * max_sigma) : T(0.0);
        grav_rc = p->enable_gravity ? T(std::fmax(p->gravity_cutoff, 1.0) * max_sigma) : T(0.0);
        rc = tmax(tmax(lj_rc, coul_rc), grav_rc);
        coul_ron = 0.9 * coul_rc;
        grav_ron = 0.9 * grav_rc;
    }
};

template <class T>
inline void smooth_t(const T& r, const T& r_on, const T& rc, T& sw, T& dsw) {  // forces.rs:302-318
    if (val(r) <= val(r_on)) { sw = 1.0; dsw = 0.0; return; }
    if (val(r) >= val(rc)) { sw = 0.0; dsw = 0.0; return; }
    T u = (r - r_on) / (rc - r_on);
    T u2 = u * u;
    T u3 = u2 * u;
    T u4 = u3 * u;
    T u5 = u4 * u;
    sw = 1.0 - 10.0 * u3 + 15.0 * u4 - 6.0 * u5;
    T dsdu = -30.0 * u2 * (1.0 - u) * (1.0 - u);
    dsw = dsdu / (rc - r_on);
}

template <class T>
struct PartT {
    std::vector<std::pair<uint32_t, V3T<T>>> forces;
    T v = 0.0;
};

template <class T>
inline V3T<T> delta_of(const orc_params* p, const std::vector<T>& pos, uint32_t a, uint32_t b) {
    return {min_image_1(pos[3 * a] - pos[3 * b], p->box[0]), min_image_1(pos[3 * a + 1] - pos[3 * b + 1], p->box[1]),
            min_image_1(pos[3 * a + 2] - pos[3 * b + 2], p->box[2])};
}

// Phase 3 body of systems/forces.rs:256-324 for one pair, the bond term
// excluded (the adjoint does not cover the bond spring).
template <class T>
void pair_fold_t(const orc_params* p, const SetupT<T>& fs, const std::vector<T>& pos, const uint8_t* elem,
                 const double* charge, const double* mass, uint32_t a, uint32_t b, PartT<T>& acc) {
    V3T<T> delta = delta_of(p, pos, a, b);
    T d2 = delta.x * delta.x + delta.y * delta.y + delta.z * delta.z;
    T rc2 = fs.rc * fs.rc;
    if (val(d2) >= val(rc2)) return;
    T d = tsqrt(d2);
    if (val(d) <= kEps) return;
    T inv = 1.0 / d;
    V3T<T> normal = {delta.x * inv, delta.y * inv, delta.z * inv};
    T fmag = 0.0;
    int ta = elem[a], tb = elem[b];
    if (val(d) < val(fs.lj_rc)) {  // :273-278, lj_raw forces.rs:346-353
        const T& sg = fs.sig[ta * 10 + tb];
        const T& ep = fs.eps[ta * 10 + tb];
        T r = tmax(d, T(0.5 * sg));
        T s = sg / r;
        T s6 = s * s * s * s * s * s;
        T s12 = s6 * s6;
        T v = 4.0 * ep * (s12 - s6);
        T m = 24.0 * ep / sg * s * (2.0 * s12 - s6);
        T sw, dsw;
        smooth_t(r, fs.lj_ron, fs.lj_rc, sw, dsw);
        fmag = fmag + (m * sw - v * dsw);
        acc.v = acc.v + v * sw;
    }
    if (p->enable_electrostatics && val(d) < val(fs.coul_rc)) {  // :282-289
        T r = tmax(d, T(0.5));
        double q = p->coulomb_constant * charge[a] * charge[b];
        T m = q / (r * r), v = q / r, sw, dsw;
        smooth_t(d, fs.coul_ron, fs.coul_rc, sw, dsw);
        fmag = fmag + (m * sw - v * dsw);
        acc.v = acc.v + v * sw;
    }
    if (p->enable_gravity && val(d) < val(fs.grav_rc)) {  // :292-299
        T r = tmax(d, T(0.5));
        double mm = p->gravity_constant * mass[a] * mass[b];
        T m = -mm / (r * r), v = -mm / r, sw, dsw;
        smooth_t(d, fs.grav_ron, fs.grav_rc, sw, dsw);
        fmag = fmag + (m * sw - v * dsw);
        acc.v = acc.v + v * sw;
    }
    if (val(fmag) != 0.0) {
        T nf = -fmag;
        acc.forces.push_back({a, {normal.x * fmag, normal.y * fmag, normal.z * fmag}});
        acc.forces.push_back({b, {normal.x * nf, normal.y * nf, normal.z * nf}});
    }
}

struct PairRec {
    uint32_t a, b;
};

template <class F>
void run_parts(int nt, F&& work) {
    if (nt == 1) {
        work(0);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
}

// One force pass (systems/forces.rs:163-353 without bonds): pair list from the
// grid of the positions' values, fold over contiguous splits, ordered merge.
template <class T>
T forces_t(const orc_params* p, const SetupT<T>& fs, size_t n, const std::vector<T>& pos, const uint8_t* elem,
           const double* charge, const double* mass, std::vector<T>& acc, int nthreads,
           std::vector<PairRec>& pairs) {
    for (size_t i = 0; i < 3 * n; ++i) acc[i] = 0.0;
    pairs.clear();
    if (n == 0) return T(0.0);
    std::vector<double> posv(3 * n);
    for (size_t i = 0; i < 3 * n; ++i) posv[i] = val(pos[i]);
    Grid grid(p->box, val(fs.rc));
    grid.build(posv.data(), n);
    grid.neighbors(posv.data(), val(fs.rc), [&](uint32_t a, uint32_t b, orcg::V3, double) { pairs.push_back({a, b}); });
    int nt = nthreads < 1 ? 1 : nthreads;
    if ((size_t)nt > pairs.size()) nt = pairs.empty() ? 1 : (int)pairs.size();
    std::vector<PartT<T>> parts(nt);
    run_parts(nt, [&](int t) {
        size_t lo = pairs.size() * (size_t)t / nt, hi = pairs.size() * (size_t)(t + 1) / nt;
        parts[t].forces.reserve(2 * (hi - lo));
        for (size_t q = lo; q < hi; ++q) pair_fold_t(p, fs, pos, elem, charge, mass, pairs[q].a, pairs[q].b, parts[t]);
    });
    T potential = 0.0;
    for (auto& part : parts) {
        potential = potential + part.v;
        for (auto& f : part.forces) {
            size_t i = f.first;
            double im = 1.0 / mass[i];
            acc[3 * i] = acc[3 * i] + f.second.x * im;
            acc[3 * i + 1] = acc[3 * i + 1] + f.second.y * im;
            acc[3 * i + 2] = acc[3 * i + 2] + f.second.z * im;
        }
    }
    return potential;
}

struct GrSpec {
    int bins, every;
    double rmax, width, support;
};

// Adds sum_{pair list} G(d - r_k) to h[k] (pairs in list order, splits merged in order).
template <class T>
void gr_accumulate(const orc_params* p, const GrSpec& g, const std::vector<T>& pos,
                   const std::vector<PairRec>& pairs, std::vector<T>& h, int nthreads) {
    double dr = g.rmax / g.bins, reach = g.support * g.width, c2 = -0.5 / (g.width * g.width);
    int nt = nthreads < 1 ? 1 : nthreads;
    if ((size_t)nt > pairs.size()) nt = pairs.empty() ? 1 : (int)pairs.size();
    std::vector<std::vector<T>> part(nt, std::vector<T>(g.bins, T(0.0)));
    run_parts(nt, [&](int t) {
        size_t lo = pairs.size() * (size_t)t / nt, hi = pairs.size() * (size_t)(t + 1) / nt;
        for (size_t q = lo; q < hi; ++q) {
            V3T<T> delta = delta_of(p, pos, pairs[q].a, pairs[q].b);
            T d = tsqrt(delta.x * delta.x + delta.y * delta.y + delta.z * delta.z);
            double dv = val(d);
            if (dv <= kEps) continue;
            int k0 = (int)std::ceil((dv - reach) / dr - 0.5), k1 = (int)std::floor((dv + reach) / dr - 0.5);
            if (k0 < 0) k0 = 0;
            if (k1 > g.bins - 1) k1 = g.bins - 1;
            for (int k = k0; k <= k1; ++k) {
                T z = d - (k + 0.5) * dr;
                if (std::fabs(val(z)) >= reach) continue;
                part[t][k] += texp(z * z * c2);
            }
        }
    });
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < g.bins; ++k) h[k] += part[t][k];
}

template <class T>
int run_adjoint_forward(const orc_params* p, size_t n, const double* pos0, const double* vel0, const double* acc0,
                        const uint8_t* elem, const double* charge, const double* mass, int nsteps, const GrSpec& gs,
                        int nthreads, const T* sigma, const T* epsk, std::vector<T>& Vt, std::vector<T>& gbar) {
    if (p->enable_bond_interaction || p->enable_thermostat) return -1;
    SetupT<T> fs(p, sigma, epsk);
    if (gs.bins > 0 && gs.rmax + gs.support * gs.width > val(fs.rc)) return -2;
    std::vector<T> pos(pos0, pos0 + 3 * n), vel(vel0, vel0 + 3 * n), acc(acc0, acc0 + 3 * n);
    std::vector<PairRec> pairs;
    std::vector<T> h(gs.bins > 0 ? gs.bins : 0, T(0.0));
    Vt.assign(nsteps, T(0.0));
    int samples = 0;
    double half_dt = 0.5 * p->dt;  // integrate.rs:39-43
    double hb[3] = {p->box[0] * 0.5, p->box[1] * 0.5, p->box[2] * 0.5};
    for (int t = 1; t <= nsteps; ++t) {  // universe/mod.rs:356-369
        for (size_t i = 0; i < 3 * n; ++i) vel[i] = vel[i] + acc[i] * half_dt;
        for (size_t i = 0; i < 3 * n; ++i) pos[i] = pos[i] + vel[i] * p->dt;  // integrate.rs:62-66
        if (p->enable_boundaries)  // boundary.rs:28-34
            for (size_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) pos[3 * i + k] = rem_euclid_t(pos[3 * i + k], 2.0 * hb[k]) - hb[k];
        Vt[t - 1] = forces_t(p, fs, n, pos, elem, charge, mass, acc, nthreads, pairs);
        for (size_t i = 0; i < 3 * n; ++i) vel[i] = vel[i] + acc[i] * half_dt;
        if (gs.bins > 0 && t % gs.every == 0) {
            gr_accumulate(p, gs, pos, pairs, h, nthreads);
            ++samples;
        }
    }
    gbar.assign(gs.bins > 0 ? gs.bins : 0, T(0.0));
    if (gs.bins > 0 && samples > 0) {
        const double pi = 3.14159265358979323846;
        double vol = p->box[0] * p->box[1] * p->box[2], dr = gs.rmax / gs.bins;
        double npair = 0.5 * (double)n * ((double)n - 1.0);
        for (int k = 0; k < gs.bins; ++k) {
            double r = (k + 0.5) * dr;
            double c = vol / (npair * 4.0 * pi * r * r * std::sqrt(2.0 * pi) * gs.width) / samples;
            gbar[k] = h[k] * c;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int orc_adjoint_forward(const orc_params* p, size_t n, const double* pos, const double* vel, const double* acc,
                        const uint8_t* elem, const double* charge, const double* mass, int nsteps, int gr_bins,
                        int gr_every, double gr_rmax, double gr_width, double gr_support, int nthreads,
                        double* potential, double* gr, double* dpotential, double* dgr) {
    if (!p || nsteps < 1 || (gr_bins > 0 && (gr_every < 1 || !(gr_width > 0.0) || !(gr_rmax > 0.0)))) return -3;
    GrSpec gs{gr_bins > 0 ? gr_bins : 0, gr_every, gr_rmax, gr_width, gr_support};
    if (!dpotential && !dgr) {
        std::vector<double> Vt, gbar;
        int rc = run_adjoint_forward<double>(p, n, pos, vel, acc, elem, charge, mass, nsteps, gs, nthreads, p->sigma,
                                             p->epsilon_k, Vt, gbar);
        if (rc) return rc;
        for (int t = 0; t < nsteps; ++t) potential[t] = Vt[t];
        if (gr)
            for (int k = 0; k < gs.bins; ++k) gr[k] = gbar[k];
        return 0;
    }
    Dual sig[ORC_NELEM], eps[ORC_NELEM];
    for (int e = 0; e < ORC_NELEM; ++e) {
        sig[e] = Dual(p->sigma[e]);
        sig[e].d[e] = 1.0;
        eps[e] = Dual(p->epsilon_k[e]);
        eps[e].d[ORC_NELEM + e] = 1.0;
    }
    std::vector<Dual> Vt, gbar;
    int rc = run_adjoint_forward<Dual>(p, n, pos, vel, acc, elem, charge, mass, nsteps, gs, nthreads, sig, eps, Vt,
                                       gbar);
    if (rc) return rc;
    for (int t = 0; t < nsteps; ++t) {
        potential[t] = Vt[t].v;
        if (dpotential)
            for (int j = 0; j < ND; ++j) dpotential[(size_t)t * ND + j] = Vt[t].d[j];
    }
    for (int k = 0; k < gs.bins; ++k) {
        if (gr) gr[k] = gbar[k].v;
        if (dgr)
            for (int j = 0; j < ND; ++j) dgr[(size_t)k * ND + j] = gbar[k].d[j];
    }
    return 0;
}

// The T = double trajectory only (positions, velocities, accelerations after
// nsteps), to check the template against orc_ticks bit for bit.
int orc_adjoint_trajectory(const orc_params* p, size_t n, double* pos, double* vel, double* acc, const uint8_t* elem,
                           const double* charge, const double* mass, int nsteps, int nthreads, double* potential) {
    if (!p || nsteps < 1 || p->enable_bond_interaction || p->enable_thermostat) return -1;
    SetupT<double> fs(p, p->sigma, p->epsilon_k);
    std::vector<double> P(pos, pos + 3 * n), Vv(vel, vel + 3 * n), A(acc, acc + 3 * n);
    std::vector<PairRec> pairs;
    double half_dt = 0.5 * p->dt;
    double hb[3] = {p->box[0] * 0.5, p->box[1] * 0.5, p->box[2] * 0.5};
    for (int t = 0; t < nsteps; ++t) {
        for (size_t i = 0; i < 3 * n; ++i) Vv[i] = Vv[i] + A[i] * half_dt;
        for (size_t i = 0; i < 3 * n; ++i) P[i] = P[i] + Vv[i] * p->dt;
        if (p->enable_boundaries)
            for (size_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) P[3 * i + k] = rem_euclid_t(P[3 * i + k], 2.0 * hb[k]) - hb[k];
        double V = forces_t(p, fs, n, P, elem, charge, mass, A, nthreads, pairs);
        for (size_t i = 0; i < 3 * n; ++i) Vv[i] = Vv[i] + A[i] * half_dt;
        if (potential) potential[t] = V;
    }
    for (size_t i = 0; i < 3 * n; ++i) {
        pos[i] = P[i];
        vel[i] = Vv[i];
        acc[i] = A[i];
    }
    return 0;
}

}  // extern "C"
