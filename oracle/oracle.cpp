// oracle.cpp -- CPU FP64 restatement of the GENESIS per-tick hot path.
//
// TEST INFRASTRUCTURE ONLY (the checker).  See oracle.h for the parity
// status.  Build with -O2 -ffp-contract=off (Makefile in this directory):
// the reference is Rust, which never fuses a*b+c, so every product and sum
// here must round separately to reproduce its FP64 results bit for bit.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_grid.h"

namespace {

using namespace orcg;

struct LjTable {  // forces.rs:212-276
    double sig[100], eps[100], rc, r_on;
    explicit LjTable(const orc_params* p) {  // forces.rs:223-237
        double max_sigma = 0.0;
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) {
                double s = 0.5 * (p->sigma[i] + p->sigma[j]);
                double e = p->thermal_constant * std::sqrt(p->epsilon_k[i] * p->epsilon_k[j]);
                max_sigma = std::fmax(max_sigma, s);
                sig[i * 10 + j] = s;
                eps[i * 10 + j] = e;
            }
        rc = std::fmax(p->lj_cutoff_factor, 1.0) * max_sigma;
        r_on = 0.9 * rc;
    }
};

inline void lj_raw(double sigma, double eps, double r, double* m, double* v) {  // forces.rs:346-353
    double s = sigma / r;
    double s6 = s * s * s * s * s * s;
    double s12 = s6 * s6;
    *v = 4.0 * eps * (s12 - s6);
    *m = (24.0 * eps / sigma) * s * (2.0 * s12 - s6);
}

inline void smooth_cutoff(double r, double r_on, double rc, double* sw, double* dsw) {  // forces.rs:302-318
    if (r <= r_on) { *sw = 1.0; *dsw = 0.0; return; }
    if (r >= rc) { *sw = 0.0; *dsw = 0.0; return; }
    double u = (r - r_on) / (rc - r_on);
    double u2 = u * u;
    double u3 = u2 * u;
    double u4 = u3 * u;
    double u5 = u4 * u;
    *sw = 1.0 - 10.0 * u3 + 15.0 * u4 - 6.0 * u5;
    double dsdu = -30.0 * u2 * (1.0 - u) * (1.0 - u);
    *dsw = dsdu / (rc - r_on);
}

inline void switched(double f, double v, double sw, double dsw, double* fo, double* vo) {  // forces.rs:322-324
    *fo = f * sw - v * dsw;
    *vo = v * sw;
}

inline double well_curvature(double eps, double sigma) {  // forces.rs:194-196
    return 72.0 * std::pow(2.0, -1.0 / 3.0) * eps / (sigma * sigma);
}
inline double equilibrium_distance(double sigma) {  // forces.rs:281-283
    return sigma * std::pow(2.0, 1.0 / 6.0);
}

// Everything ForceSystem::new derives from the config (systems/forces.rs:100-142).
struct ForceSetup {
    LjTable lj;
    double rc, coulomb_rc, coulomb_r_on, gravity_rc, gravity_r_on, bond_k_bind;
    explicit ForceSetup(const orc_params* p) : lj(p) {
        double max_sigma = 0.0;
        for (int i = 0; i < 10; ++i) max_sigma = std::fmax(max_sigma, p->sigma[i]);
        coulomb_rc = p->enable_electrostatics ? std::fmax(p->coulomb_cutoff, 1.0) * max_sigma : 0.0;
        gravity_rc = p->enable_gravity ? std::fmax(p->gravity_cutoff, 1.0) * max_sigma : 0.0;
        rc = std::fmax(std::fmax(lj.rc, coulomb_rc), gravity_rc);
        coulomb_r_on = 0.9 * coulomb_rc;
        gravity_r_on = 0.9 * gravity_rc;
        bond_k_bind = p->bond_k_bind;
    }
};

struct PairRec {
    uint32_t a, b;
};

struct Part {  // one rayon split: ForceParts = (Vec<(u32, Vec3)>, f64, f64), systems/forces.rs:66
    std::vector<std::pair<uint32_t, V3>> forces;
    double v = 0.0, vbond = 0.0;
};

// Phase 3 body of systems/forces.rs:256-324 for one pair.
inline void pair_fold(const orc_params* p, const ForceSetup& fs, const double* pos,
                      const uint8_t* elem, const double* charge, const double* mass,
                      const std::vector<std::vector<uint32_t>>& bond_of, PairRec pr, Part& acc) {
    (void)mass;
    const double rc2 = fs.rc * fs.rc;
    V3 delta = min_image(sub(at(pos, pr.a), at(pos, pr.b)), p->box);
    double d2 = len2(delta);
    if (d2 >= rc2) return;
    double d = std::sqrt(d2);
    if (d <= kEps) return;
    V3 normal = scale(delta, 1.0 / d);
    double fmag = 0.0;
    int ta = elem[pr.a], tb = elem[pr.b];
    if (d < fs.lj.rc) {  // :273-278
        double sg = fs.lj.sig[ta * 10 + tb], ep = fs.lj.eps[ta * 10 + tb];
        double r = std::fmax(d, 0.5 * sg);  // force_switched_scalar, forces.rs:270-275
        double m, v, sw, dsw, m2, v2;
        lj_raw(sg, ep, r, &m, &v);
        smooth_cutoff(r, fs.lj.r_on, fs.lj.rc, &sw, &dsw);
        switched(m, v, sw, dsw, &m2, &v2);
        fmag += m2;
        acc.v += v2;
    }
    if (p->enable_electrostatics && d < fs.coulomb_rc) {  // :282-289
        double r = std::fmax(d, 0.5);
        double q = p->coulomb_constant * charge[pr.a] * charge[pr.b];  // coulomb_raw, forces.rs:330-333
        double m = q / (r * r), v = q / r, sw, dsw, m2, v2;
        smooth_cutoff(d, fs.coulomb_r_on, fs.coulomb_rc, &sw, &dsw);
        switched(m, v, sw, dsw, &m2, &v2);
        fmag += m2;
        acc.v += v2;
    }
    if (p->enable_gravity && d < fs.gravity_rc) {  // :292-299
        double r = std::fmax(d, 0.5);
        double mm = p->gravity_constant * mass[pr.a] * mass[pr.b];  // gravity_raw, forces.rs:338-341
        double m = -mm / (r * r), v = -mm / r, sw, dsw, m2, v2;
        smooth_cutoff(d, fs.gravity_r_on, fs.gravity_rc, &sw, &dsw);
        switched(m, v, sw, dsw, &m2, &v2);
        fmag += m2;
        acc.v += v2;
    }
    if (p->enable_bond_interaction) {  // :305-317
        const auto& lst = bond_of[pr.a];
        if (std::find(lst.begin(), lst.end(), pr.b) != lst.end()) {
            double sg = fs.lj.sig[ta * 10 + tb], ep = fs.lj.eps[ta * 10 + tb];
            double r_eq = equilibrium_distance(sg);
            double rc_bond = fs.bond_k_bind * sg;
            if (d < rc_bond) {
                double k = well_curvature(ep, sg);
                double dr = d - r_eq;  // bond_harmonic_raw, forces.rs:290-293
                double m = -k * dr, v = 0.5 * k * dr * dr, sw, dsw, m2, v2;
                smooth_cutoff(d, r_eq, rc_bond, &sw, &dsw);
                switched(m, v, sw, dsw, &m2, &v2);
                fmag += m2;
                acc.vbond += v2;
            }
        }
    }
    if (fmag != 0.0) {
        acc.forces.push_back({pr.a, scale(normal, fmag)});
        acc.forces.push_back({pr.b, scale(normal, -fmag)});
    }
}

size_t forces_impl(const orc_params* p, size_t n, const double* pos, const uint8_t* elem,
                   const double* charge, const double* mass, size_t nbonds, const uint32_t* bonds,
                   double* acc_out, double* pot, double* bpot, int nthreads) {
    for (size_t i = 0; i < 3 * n; ++i) acc_out[i] = 0.0;
    *pot = 0.0;
    *bpot = 0.0;
    if (n == 0) return 0;  // systems/forces.rs:201-203
    ForceSetup fs(p);
    // Phase 1.5 (:208-226): bond adjacency in slot space.
    std::vector<std::vector<uint32_t>> bond_of;
    if (p->enable_bond_interaction) {
        bond_of.assign(n, {});
        for (size_t k = 0; k < nbonds; ++k) {
            uint32_t si = bonds[2 * k], sj = bonds[2 * k + 1];
            if (si >= n || sj >= n) continue;
            bond_of[si].push_back(sj);
            bond_of[sj].push_back(si);
        }
    }
    // Phase 2 (:230-232).
    Grid grid(p->box, fs.rc);
    grid.build(pos, n);
    std::vector<PairRec> pairs;
    grid.neighbors(pos, fs.rc, [&](uint32_t a, uint32_t b, V3, double) { pairs.push_back({a, b}); });
    // Phase 3 (:251-326): fold over contiguous splits.
    int nt = nthreads < 1 ? 1 : nthreads;
    if ((size_t)nt > pairs.size()) nt = pairs.empty() ? 1 : (int)pairs.size();
    std::vector<Part> parts(nt);
    auto work = [&](int t) {
        size_t lo = pairs.size() * (size_t)t / nt, hi = pairs.size() * (size_t)(t + 1) / nt;
        parts[t].forces.reserve(2 * (hi - lo));
        for (size_t q = lo; q < hi; ++q) pair_fold(p, fs, pos, elem, charge, mass, bond_of, pairs[q], parts[t]);
    };
    if (nt == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(work, t);
        for (auto& x : th) x.join();
    }
    // Phase 4 (:330-341): ordered merge, acc[index] += F * (1/m).
    double potential = 0.0, bond_potential = 0.0;
    for (auto& part : parts) {
        potential += part.v;
        bond_potential += part.vbond;
        for (auto& f : part.forces) {
            V3 a = at(acc_out, f.first);
            V3 c = add(a, scale(f.second, 1.0 / mass[f.first]));
            acc_out[3 * f.first] = c.x;
            acc_out[3 * f.first + 1] = c.y;
            acc_out[3 * f.first + 2] = c.z;
        }
    }
    *pot = potential;
    *bpot = bond_potential;
    return pairs.size();
}

// Chunked parallel-for mirroring World::par_for_each*_mut (ecs/world.rs:436-491).
template <class F>
void par_chunks(size_t n, int nthreads, F&& f) {
    if (nthreads <= 1 || n < 4096) {
        f((size_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t) {
        size_t lo = n * (size_t)t / nthreads, hi = n * (size_t)(t + 1) / nthreads;
        th.emplace_back(f, lo, hi);
    }
    for (auto& x : th) x.join();
}

void half_kick_range(double* vel, const double* acc, double dt, size_t lo, size_t hi) {
    double half_dt = 0.5 * dt;  // integrate.rs:39-43
    for (size_t i = lo; i < hi; ++i)
        for (int k = 0; k < 3; ++k) vel[3 * i + k] = vel[3 * i + k] + acc[3 * i + k] * half_dt;
}
void drift_range(double* pos, const double* vel, double dt, size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i)  // integrate.rs:62-66
        for (int k = 0; k < 3; ++k) pos[3 * i + k] = pos[3 * i + k] + vel[3 * i + k] * dt;
}
void wrap_range(double* pos, const double* box, size_t lo, size_t hi) {
    double h[3] = {box[0] * 0.5, box[1] * 0.5, box[2] * 0.5};  // boundary.rs:28-34
    for (size_t i = lo; i < hi; ++i)
        for (int k = 0; k < 3; ++k) pos[3 * i + k] = rem_euclid(pos[3 * i + k], 2.0 * h[k]) - h[k];
}

int thermostat_impl(size_t n, double* vel, const double* mass, double k, double target,
                    double tau_cfg, double* kin_out, double* lam_out, int nthreads) {
    double tau = std::fmax(tau_cfg, 1.0);  // thermostat.rs:26
    *kin_out = 0.0;
    *lam_out = 1.0;
    if (target <= 0.0) return 0;  // :48-50
    double kinetic = 0.0;
    for (size_t i = 0; i < n; ++i) {  // :52-57
        V3 v = at(vel, i);
        kinetic += 0.5 * mass[i] * len2(v);
    }
    *kin_out = kinetic;
    if (n == 0) return 0;
    double t = (2.0 / 3.0) * (kinetic / (double)n) / k;  // :62
    if (!std::isfinite(t) || t <= 0.0) return 0;
    double lambda2 = 1.0 + (1.0 / tau) * (target / t - 1.0);  // :66
    double lambda = std::sqrt(std::fmax(lambda2, 0.0));
    *lam_out = lambda;
    par_chunks(n, nthreads, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i)
            for (int c = 0; c < 3; ++c) vel[3 * i + c] = vel[3 * i + c] * lambda;  // v.0 *= lambda
    });
    return 1;
}

// Union-find of analysis/mod.rs:287-307.
size_t uf_find(std::vector<size_t>& parent, size_t x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}
void uf_union(std::vector<size_t>& parent, std::vector<uint32_t>& rank, size_t a, size_t b) {
    size_t ra = uf_find(parent, a), rb = uf_find(parent, b);
    if (ra == rb) return;
    size_t hi, lo;
    if (rank[ra] < rank[rb]) { hi = rb; lo = ra; } else { hi = ra; lo = rb; }
    parent[lo] = hi;
    if (rank[hi] == rank[lo]) rank[hi] += 1;
}

const size_t kGSampleCap = 8192;  // analysis/mod.rs:28

// analysis/mod.rs:32-46: returns the slot indices of the subsample.
std::vector<size_t> g_subsample(size_t n) {
    std::vector<size_t> idx;
    if (n <= kGSampleCap) {
        idx.resize(n);
        for (size_t i = 0; i < n; ++i) idx[i] = i;
        return idx;
    }
    size_t step = n / kGSampleCap + 1;
    size_t count = n / step;
    idx.resize(count);
    for (size_t i = 0; i < count; ++i) idx[i] = i * step;
    return idx;
}

int gr_impl(size_t n, const double* pos, const uint8_t* elem, int ta, int tb, const double* box,
            double r_max_in, size_t nbins_in, uint64_t* counts, double* bins, double* rmo, double* dro) {
    size_t nbins = std::min(std::max(nbins_in, (size_t)1), (size_t)1 << 16);
    double half_min = std::fmin(std::fmin(box[0], box[1]), box[2]) * 0.5;
    double r_max = std::fmin(std::fmax(r_max_in, 1e-9), half_min);
    double dr = r_max / (double)nbins;
    double vol = box[0] * box[1] * box[2];
    std::vector<size_t> sidx = g_subsample(n);
    size_t m = sidx.size();
    std::vector<double> sp(3 * m);
    std::vector<uint8_t> st(m);
    for (size_t i = 0; i < m; ++i) {
        for (int k = 0; k < 3; ++k) sp[3 * i + k] = pos[3 * sidx[i] + k];
        st[i] = elem ? elem[sidx[i]] : 0;
    }
    for (size_t b = 0; b < nbins; ++b) counts[b] = 0;
    Grid grid(box, r_max);
    grid.build(sp.data(), m);
    bool partial = ta >= 0;
    int bad = 0;
    grid.neighbors(sp.data(), r_max, [&](uint32_t a, uint32_t b, V3, double) {
        if (partial) {
            int x = st[a], y = st[b];
            if (!((x == ta && y == tb) || (x == tb && y == ta))) return;
        }
        V3 dl = min_image(sub(at(sp.data(), a), at(sp.data(), b)), box);
        double d = std::sqrt(len2(dl));  // Vec3::length
        if (d >= r_max) return;
        size_t bi = (size_t)(d / dr);
        if (bi >= nbins) { bad = 1; return; }  // the reference would panic on this index
        counts[bi] += 1;
    });
    *rmo = r_max;
    *dro = dr;
    for (size_t b = 0; b < nbins; ++b) bins[b] = 0.0;
    double pair_count;
    if (partial) {
        size_t na = 0, nb = 0;
        for (size_t i = 0; i < m; ++i) {
            na += st[i] == ta;
            nb += st[i] == tb;
        }
        pair_count = ta == tb ? (double)na * (double)(na == 0 ? 0 : na - 1) * 0.5 : (double)na * (double)nb;
        if (pair_count <= 0.0) return bad ? -1 : 0;
    } else {
        if (m < 2) return bad ? -1 : 0;
    }
    const double pi = 3.141592653589793;
    for (size_t i = 0; i < nbins; ++i) {
        double r_lo = (double)i * dr;
        double r_hi = r_lo + dr;
        double shell = 4.0 / 3.0 * pi * (r_hi * r_hi * r_hi - r_lo * r_lo * r_lo);
        double expected = partial ? pair_count * shell / vol
                                  : (double)(m * (m - 1)) * 0.5 * shell / vol;
        bins[i] = (double)counts[i] / std::fmax(expected, 2.2250738585072014e-308);
    }
    return bad ? -1 : 0;
}

}  // namespace

extern "C" {

void orc_lj_table(const orc_params* p, double* ps, double* pe, double* rc, double* r_on) {
    LjTable t(p);
    std::memcpy(ps, t.sig, sizeof t.sig);
    std::memcpy(pe, t.eps, sizeof t.eps);
    *rc = t.rc;
    *r_on = t.r_on;
}
void orc_lj_raw(double sigma, double eps, double r, double* m, double* v) { lj_raw(sigma, eps, r, m, v); }
void orc_smooth_cutoff(double r, double r_on, double rc, double* sw, double* dsw) {
    smooth_cutoff(r, r_on, rc, sw, dsw);
}
void orc_switched(double f, double v, double sw, double dsw, double* fo, double* vo) {
    switched(f, v, sw, dsw, fo, vo);
}
void orc_force_switched_scalar(double sigma, double eps, double r_in, double r_on, double rc,
                               double* m, double* v) {  // forces.rs:270-275
    double r = std::fmax(r_in, 0.5 * sigma);
    double mm, vv, sw, dsw;
    lj_raw(sigma, eps, r, &mm, &vv);
    smooth_cutoff(r, r_on, rc, &sw, &dsw);
    switched(mm, vv, sw, dsw, m, v);
}
void orc_coulomb_raw(double k_e, double qa, double qb, double r, double* f, double* v) {
    double q = k_e * qa * qb;  // forces.rs:330-333
    *f = q / (r * r);
    *v = q / r;
}
void orc_gravity_raw(double g, double ma, double mb, double r, double* f, double* v) {
    double m = g * ma * mb;  // forces.rs:338-341
    *f = -m / (r * r);
    *v = -m / r;
}
void orc_bond_harmonic_raw(double k, double r_eq, double r, double* f, double* v) {
    double dr = r - r_eq;  // forces.rs:290-293
    *f = -k * dr;
    *v = 0.5 * k * dr * dr;
}
double orc_well_curvature(double eps, double sigma) { return well_curvature(eps, sigma); }
double orc_vib_period(double eps, double sigma, double mu) {  // forces.rs:201-203
    return 2.0 * 3.141592653589793 * std::sqrt(mu / well_curvature(eps, sigma));
}
double orc_equilibrium_distance(double sigma) { return equilibrium_distance(sigma); }

void orc_grid_dims(const double box[3], double min_cell, uint32_t dims[3]) {
    Grid g(box, min_cell);
    for (int k = 0; k < 3; ++k) dims[k] = g.dims[k];
}
void orc_cell_of(size_t n, const double* pos, const double box[3], double min_cell, uint32_t* cell) {
    Grid g(box, min_cell);
    for (size_t i = 0; i < n; ++i) cell[i] = (uint32_t)g.cell_index(at(pos, i));
}
size_t orc_neighbors(size_t n, const double* pos, const double box[3], double min_cell, double cutoff,
                     uint32_t* pairs, double* normals, size_t cap) {
    Grid g(box, min_cell);
    g.build(pos, n);
    size_t cnt = 0;
    g.neighbors(pos, cutoff, [&](uint32_t a, uint32_t b, V3 delta, double d) {
        if (cnt < cap) {
            if (pairs) { pairs[2 * cnt] = a; pairs[2 * cnt + 1] = b; }
            if (normals) {
                V3 nrm = scale(delta, 1.0 / d);
                normals[3 * cnt] = nrm.x;
                normals[3 * cnt + 1] = nrm.y;
                normals[3 * cnt + 2] = nrm.z;
            }
        }
        ++cnt;
    });
    return cnt;
}
void orc_min_image(const double d[3], const double box[3], double out[3]) {
    V3 r = min_image({d[0], d[1], d[2]}, box);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
}

size_t orc_forces(const orc_params* p, size_t n, const double* pos, const uint8_t* elem,
                  const double* charge, const double* mass, size_t nbonds, const uint32_t* bonds,
                  double* acc, double* potential, double* bond_potential, int nthreads) {
    return forces_impl(p, n, pos, elem, charge, mass, nbonds, bonds, acc, potential, bond_potential,
                       nthreads);
}

void orc_half_kick(size_t n, double* vel, const double* acc, double dt) { half_kick_range(vel, acc, dt, 0, n); }
void orc_drift(size_t n, double* pos, const double* vel, double dt) { drift_range(pos, vel, dt, 0, n); }
void orc_wrap(size_t n, double* pos, const double box[3]) { wrap_range(pos, box, 0, n); }
int orc_thermostat(size_t n, double* vel, const double* mass, double k, double target, double tau,
                   double* kinetic, double* lambda) {
    return thermostat_impl(n, vel, mass, k, target, tau, kinetic, lambda, 1);
}
void orc_stats(size_t n, const double* vel, const double* mass, double* kinetic, double* speed_sum) {
    double kin = 0.0, sp = 0.0;  // systems/aggregate.rs:86-93
    for (size_t i = 0; i < n; ++i) {
        V3 v = at(vel, i);
        kin += 0.5 * mass[i] * len2(v);
        sp += std::sqrt(len2(v));
    }
    *kinetic = kin;
    *speed_sum = sp;
}

// elastic_pair, src/physics/collision.rs:16-32: the velocity changes of both
// particles (n points from 2 towards 1; Vec3 `/ x` scales by 1/x,
// src/math/mod.rs); false when they separate or a mass is not positive.
static bool elastic_pair(double m1, V3 v1, double m2, V3 v2, V3 n, V3* dv1, V3* dv2) {
    *dv1 = V3{0.0, 0.0, 0.0};
    *dv2 = V3{0.0, 0.0, 0.0};
    if (m1 <= 0.0 || m2 <= 0.0) return false;
    V3 vrel = sub(v1, v2);
    double vn = vrel.x * n.x + vrel.y * n.y + vrel.z * n.z;
    if (vn >= 0.0) return false;
    double j = -2.0 * vn / (1.0 / m1 + 1.0 / m2);
    V3 jv = scale(n, j);
    *dv1 = scale(jv, 1.0 / m1);
    *dv2 = scale(scale(jv, 1.0 / m2), -1.0);
    return true;
}

// CollisionSystem::run, src/systems/collisions.rs:40-88: the pairs within 2r
// on a grid of cell 2r, impulses from the velocities before the pass, summed
// per particle in pair order and applied when any pair collided.  Returns
// the collisions counted.
static size_t collisions_impl(const orc_params* p, size_t n, const double* pos, double* vel, const double* mass) {
    if (n == 0) return 0;
    const double contact = 2.0 * p->particle_radius;
    Grid g(p->box, contact);
    g.build(pos, n);
    std::vector<V3> dv(n, V3{0.0, 0.0, 0.0});
    size_t count = 0;
    g.neighbors(pos, contact, [&](uint32_t a, uint32_t b, V3 delta, double d) {
        V3 da, db;
        elastic_pair(mass[a], at(vel, a), mass[b], at(vel, b), scale(delta, 1.0 / d), &da, &db);
        if (da.x != 0.0 || da.y != 0.0 || da.z != 0.0) {
            dv[a] = add(dv[a], da);
            dv[b] = add(dv[b], db);
            ++count;
        }
    });
    if (count)
        for (size_t i = 0; i < n; ++i) {
            vel[3 * i] += dv[i].x;
            vel[3 * i + 1] += dv[i].y;
            vel[3 * i + 2] += dv[i].z;
        }
    return count;
}

size_t orc_collisions(const orc_params* p, size_t n, const double* pos, double* vel, const double* mass) {
    return collisions_impl(p, n, pos, vel, mass);
}

int orc_ticks(const orc_params* p, size_t n, double* pos, double* vel, double* acc, const uint8_t* elem,
              const double* charge, const double* mass, size_t nbonds, const uint32_t* bonds, int nticks,
              int nthreads, double* out_stats) {
    int nt = nthreads < 1 ? 1 : nthreads;
    for (int t = 0; t < nticks; ++t) {  // universe/mod.rs:356-369
        par_chunks(n, nt, [&](size_t lo, size_t hi) { half_kick_range(vel, acc, p->dt, lo, hi); });
        par_chunks(n, nt, [&](size_t lo, size_t hi) { drift_range(pos, vel, p->dt, lo, hi); });
        if (p->enable_boundaries)
            par_chunks(n, nt, [&](size_t lo, size_t hi) { wrap_range(pos, p->box, lo, hi); });
        double V = 0.0, Vb = 0.0;
        size_t np = forces_impl(p, n, pos, elem, charge, mass, nbonds, bonds, acc, &V, &Vb, nt);
        if (p->enable_collisions) collisions_impl(p, n, pos, vel, mass);  // universe/mod.rs:363-365
        par_chunks(n, nt, [&](size_t lo, size_t hi) { half_kick_range(vel, acc, p->dt, lo, hi); });
        double K = 0.0, lam = 1.0;
        if (p->enable_thermostat)
            thermostat_impl(n, vel, mass, p->thermal_constant, p->thermostat_temperature,
                            p->thermostat_tau, &K, &lam, nt);
        if (out_stats) {
            double kin, sp;
            orc_stats(n, vel, mass, &kin, &sp);
            double* o = out_stats + 5 * t;
            o[0] = kin;
            o[1] = V;
            o[2] = Vb;
            o[3] = lam;
            o[4] = (double)np;
        }
    }
    return 0;
}

int orc_radial_distribution(size_t n, const double* pos, const double box[3], double r_max, size_t nbins,
                            uint64_t* counts, double* bins, double* rmo, double* dro) {
    return gr_impl(n, pos, nullptr, -1, -1, box, r_max, nbins, counts, bins, rmo, dro);
}
int orc_radial_distribution_between(size_t n, const double* pos, const uint8_t* elem, uint8_t ta, uint8_t tb,
                                    const double box[3], double r_max, size_t nbins, uint64_t* counts,
                                    double* bins, double* rmo, double* dro) {
    return gr_impl(n, pos, elem, ta, tb, box, r_max, nbins, counts, bins, rmo, dro);
}

int orc_clusters(size_t n, const double* pos, const uint8_t* elem, const double box[3], double bond_factor,
                 const double sigma[10], uint32_t* labels, uint64_t stats[4], double* mean_size) {
    stats[0] = stats[1] = stats[2] = stats[3] = 0;
    *mean_size = 0.0;
    if (n == 0) return 0;  // analysis/mod.rs:228-232
    std::vector<double> sig(n);
    double max_sigma = 0.0;
    for (size_t i = 0; i < n; ++i) {
        sig[i] = sigma[elem[i]];
        max_sigma = std::fmax(max_sigma, sig[i]);
    }
    double cutoff = std::fmax(std::fmax(bond_factor, 0.1) * max_sigma, 1e-9);  // :238
    Grid grid(box, cutoff);
    grid.build(pos, n);
    std::vector<size_t> parent(n);
    std::vector<uint32_t> rank(n, 0);
    for (size_t i = 0; i < n; ++i) parent[i] = i;
    uint64_t bound_pairs = 0;
    grid.neighbors(pos, cutoff, [&](uint32_t a, uint32_t b, V3, double) {  // :248-255
        V3 dl = min_image(sub(at(pos, a), at(pos, b)), box);
        double d = std::sqrt(len2(dl));
        double bond = bond_factor * 0.5 * (sig[a] + sig[b]);
        if (d < bond) {
            uf_union(parent, rank, a, b);
            bound_pairs += 1;
        }
    });
    std::vector<size_t> sizes(n, 0);
    std::vector<uint32_t> minmember(n, 0xFFFFFFFFu);
    for (size_t i = 0; i < n; ++i) {
        size_t r = uf_find(parent, i);
        sizes[r] += 1;
        if (minmember[r] == 0xFFFFFFFFu) minmember[r] = (uint32_t)i;
    }
    uint64_t monomers = 0, aggregates = 0, largest = 0, total = 0;
    for (size_t s : sizes) {  // :257-276
        if (s == 0) continue;
        total += 1;
        if (s == 1) monomers += 1; else aggregates += 1;
        largest = std::max<uint64_t>(largest, s);
    }
    if (labels)
        for (size_t i = 0; i < n; ++i) labels[i] = minmember[uf_find(parent, i)];
    stats[0] = monomers;
    stats[1] = aggregates;
    stats[2] = largest;
    stats[3] = bound_pairs;
    *mean_size = (double)n / (double)std::max<uint64_t>(total, 1);
    return 0;
}

size_t orc_bound_pairs(size_t n, const double* pos, const uint8_t* elem, const uint32_t* entity,
                       const double box[3], double k_bind, const double sigma[10], uint32_t* out, size_t cap) {
    double ms = 0.0;  // bind_cutoff, analysis/pairs.rs:112-114
    for (int i = 0; i < 10; ++i) ms = std::fmax(ms, sigma[i]);
    double cutoff = k_bind * ms;
    Grid grid(box, cutoff);
    grid.build(pos, n);
    size_t cnt = 0;
    grid.neighbors(pos, cutoff, [&](uint32_t a, uint32_t b, V3, double) {  // analysis/pairs.rs:159-172
        V3 dl = min_image(sub(at(pos, a), at(pos, b)), box);
        double d = std::sqrt(len2(dl));
        double threshold = k_bind * (0.5 * (sigma[elem[a]] + sigma[elem[b]]));
        if (d < threshold) {
            uint32_t ea = entity ? entity[a] : a, eb = entity ? entity[b] : b;
            if (eb < ea) std::swap(ea, eb);
            if (cnt < cap) { out[2 * cnt] = ea; out[2 * cnt + 1] = eb; }
            ++cnt;
        }
    });
    return cnt;
}

}  // extern "C"
