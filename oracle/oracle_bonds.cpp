// oracle_bonds.cpp -- CPU restatement of the bond observation of one tick.
//
// TEST INFRASTRUCTURE ONLY (the checker).  Follows PairTracker::track_tick
// (src/analysis/pairs.rs:61-85, debounce :38-58) and
// BondObservationSystem::run (src/systems/bonds.rs:73-185): episodes of bound
// pairs with a debounce, persistence once an episode reaches the pair's
// threshold ceil(max(min_periods, 0.1) * vib_period(eps_ij, sigma_ij, mu) / dt)
// (bonds.rs:94-99, physics/forces.rs:194-203), the persistent pairs as the
// Bonds adjacency, and the BondObservation summary (pair and entity counts,
// species matrix, bonds formed and their lifetimes).  Pairs are keyed by
// slot (the slot-entity map is fixed for a universe), kept in ordered maps.
#include <cmath>
#include <map>
#include <set>
#include <vector>

#include "oracle.h"

namespace {

// AtomType::mass, src/components/atom_type.rs:80-93 (element order of forces.rs:176-189)
const double kMass[ORC_NELEM] = {1.008, 4.0026, 12.011, 14.007, 15.999, 22.99, 28.085, 30.974, 32.06, 55.845};

struct Open {
    uint64_t ticks = 0;
    uint64_t missing = 0;
};

}  // namespace

struct orc_tracker {
    uint64_t debounce = 1;
    std::map<uint64_t, Open> open;              // PairTracker::open + missing
    std::map<uint64_t, uint64_t> active_since;  // BondObservationSystem::active_since
    uint64_t completed = 0, completed_ticks = 0;
    uint64_t bonds_formed = 0;
    double lifetime_sum = 0.0;
};

extern "C" {

orc_tracker* orc_tracker_new(int debounce) {
    orc_tracker* t = new orc_tracker();
    t->debounce = debounce < 1 ? 1 : (uint64_t)debounce;  // debounce.max(1), pairs.rs:52
    return t;
}

void orc_tracker_free(orc_tracker* t) { delete t; }

uint64_t orc_bond_threshold(const orc_params* p, double min_periods, int ea, int eb) {
    double ma = kMass[ea], mb = kMass[eb];
    double mu = ma * mb / (ma + mb);
    double eps = p->thermal_constant * std::sqrt(p->epsilon_k[ea] * p->epsilon_k[eb]);  // mix_epsilon
    double sig = 0.5 * (p->sigma[ea] + p->sigma[eb]);                                   // mix_sigma
    double k = 72.0 * std::pow(2.0, -1.0 / 3.0) * eps / (sig * sig);                    // well_curvature
    double period = 2.0 * 3.14159265358979323846 * std::sqrt(mu / k);                   // vib_period
    double mp = std::fmax(min_periods, 0.1);                                            // bonds.rs:49
    return (uint64_t)std::ceil(mp * period / p->dt);
}

// stats: [0] bonded_pairs, [1] bonded_entities, [2] mean_coordination,
// [3] bonds_formed, [4] lifetime_sum_ticks, [5] open episodes,
// [6] completed episodes, [7] sum of completed episodes' ticks.
int orc_bond_observe(orc_tracker* t, const orc_params* p, double min_periods, size_t nbound, const uint32_t* bound,
                     const uint8_t* elem_of_slot, uint64_t tick, double* stats, uint64_t* matrix,
                     uint32_t* persistent, size_t cap, size_t* npersistent) {
    // 1. PairTracker::track_tick (pairs.rs:61-85)
    std::set<uint64_t> current;
    for (size_t k = 0; k < nbound; ++k) {
        uint32_t a = bound[2 * k], b = bound[2 * k + 1];
        if (a > b) std::swap(a, b);
        current.insert(((uint64_t)a << 32) | b);
    }
    for (uint64_t key : current) {
        Open& o = t->open[key];
        o.missing = 0;
        o.ticks += 1;
    }
    for (auto it = t->open.begin(); it != t->open.end();) {
        if (current.count(it->first)) {
            ++it;
            continue;
        }
        it->second.missing += 1;
        if (it->second.missing >= t->debounce) {
            t->completed += 1;
            t->completed_ticks += it->second.ticks;
            it = t->open.erase(it);
        } else {
            ++it;
        }
    }
    // 2. persistence per pair (bonds.rs:88-113)
    std::vector<uint64_t> pers;
    for (const auto& kv : t->open) {
        uint32_t a = (uint32_t)(kv.first >> 32), b = (uint32_t)kv.first;
        if (kv.second.ticks < orc_bond_threshold(p, min_periods, elem_of_slot[a], elem_of_slot[b])) continue;
        pers.push_back(kv.first);
    }
    // 4. summary (bonds.rs:124-182)
    std::set<uint64_t> cur(pers.begin(), pers.end());
    std::set<uint32_t> ents;
    for (int k = 0; k < ORC_NELEM * ORC_NELEM; ++k) matrix[k] = 0;
    for (uint64_t key : pers) {
        uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
        ents.insert(a);
        ents.insert(b);
        int ia = elem_of_slot[a], ib = elem_of_slot[b];
        matrix[ia * ORC_NELEM + ib] += 1;
        matrix[ib * ORC_NELEM + ia] += 1;
    }
    for (auto it = t->active_since.begin(); it != t->active_since.end();) {
        if (cur.count(it->first)) {
            ++it;
            continue;
        }
        t->bonds_formed += 1;
        t->lifetime_sum += (double)(tick - it->second);
        it = t->active_since.erase(it);
    }
    for (uint64_t key : pers) t->active_since.emplace(key, tick);
    stats[0] = (double)pers.size();
    stats[1] = (double)ents.size();
    stats[2] = ents.empty() ? 0.0 : 2.0 * (double)pers.size() / (double)ents.size();
    stats[3] = (double)t->bonds_formed;
    stats[4] = t->lifetime_sum;
    stats[5] = (double)t->open.size();
    stats[6] = (double)t->completed;
    stats[7] = (double)t->completed_ticks;
    size_t w = 0;
    for (uint64_t key : pers) {
        if (w < cap) {
            persistent[2 * w] = (uint32_t)(key >> 32);
            persistent[2 * w + 1] = (uint32_t)key;
        }
        ++w;
    }
    *npersistent = w;
    return w > cap ? -1 : 0;
}

// PairTracker::close_all (pairs.rs:88-94).
void orc_tracker_close_all(orc_tracker* t) {
    for (const auto& kv : t->open) {
        t->completed += 1;
        t->completed_ticks += kv.second.ticks;
    }
    t->open.clear();
}

}  // extern "C"
