// gx_bondtrack.cu -- bond observation on the device: BondObservationSystem::run
// (src/systems/bonds.rs:73-185) with its PairTracker (src/analysis/pairs.rs:38-94).
//
// The reference keeps the open episodes in hash maps on the host.  Here they
// live on the device as arrays sorted by pair key ((slot a << 32) | slot b,
// a < b; the slot-entity map is fixed for a handle).  One observation:
//
//   1. the tick's bound pairs (bound_pairs_with_grid, pairs.rs:132-174),
//      found on the device as slot pairs;
//   2. the open keys and the tick's keys sorted together (CUB radix sort;
//      the open entry of a key precedes its current entries);
//   3. one thread per key: the episode's new tick count, missing count and
//      persistence (track_tick, pairs.rs:61-85; threshold bonds.rs:94-99),
//      closing it after `debounce` absent ticks -- a closed persistent pair
//      is a formed bond with lifetime now - since (bonds.rs:155-167);
//   4. scans compact the open set and emit the persistent pairs, which
//      become the handle's bond list (the Bonds component the next force
//      pass reads, bonds.rs:116-121), with the species matrix and the number
//      of bonded atoms.
// Every count is an integer, so the result does not depend on scheduling.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstring>

#include "gx_internal.cuh"

namespace gx {

int bound_pairs_device(gx_handle* h, double k_bind, uint32_t* out, size_t cap, unsigned long long* dcount);
void bonds_changed(gx_handle* h, size_t nbonds, bool realloc);

namespace {

constexpr uint64_t kNever = ~0ull;
constexpr uint32_t kCurrent = 0x80000000u;
// device counters: [0] bound pairs this tick, [1] completed episodes,
// [2] their ticks, [3] bonds formed, [4] lifetime sum, [5] bonded atoms,
// [6..105] species matrix, [106] open episodes after, [107] persistent pairs
constexpr int kNCount = 108;
// AtomType::mass, src/components/atom_type.rs:80-93
const double kElemMass[kNElem] = {1.008, 4.0026, 12.011, 14.007, 15.999, 22.99, 28.085, 30.974, 32.06, 55.845};

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__global__ void k_bt_keys(const uint64_t* __restrict__ key, size_t M, const uint32_t* __restrict__ bound, size_t C,
                          uint64_t* __restrict__ ck, uint32_t* __restrict__ cv) {
    size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < M) {
        ck[s] = key[s];
        cv[s] = (uint32_t)s;
    } else if (s < M + C) {
        size_t j = s - M;
        uint32_t a = bound[2 * j], b = bound[2 * j + 1];
        if (b < a) {
            uint32_t t = a;
            a = b;
            b = t;
        }
        ck[s] = ((uint64_t)a << 32) | b;
        cv[s] = kCurrent | (uint32_t)j;
    }
}

__global__ void k_bt_merge(const uint64_t* __restrict__ ck, const uint32_t* __restrict__ cv, size_t total,
                           const uint32_t* __restrict__ ticks, const uint32_t* __restrict__ miss,
                           const uint64_t* __restrict__ since, uint64_t* __restrict__ nkey,
                           uint32_t* __restrict__ nticks, uint32_t* __restrict__ nmiss, uint64_t* __restrict__ nsince,
                           uint32_t* __restrict__ keep, uint32_t* __restrict__ pers, const uint32_t* __restrict__ thr,
                           const uint8_t* __restrict__ elem, const uint32_t* __restrict__ pos_of_slot,
                           uint32_t debounce, uint64_t now, unsigned long long* __restrict__ dc) {
    size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
    keep[s] = 0u;
    pers[s] = 0u;
    const uint64_t k = ck[s];
    if (s > 0 && ck[s - 1] == k) return;  // not the first entry of its key
    long long o = -1;
    bool cur = false;
    for (size_t t = s; t < total && ck[t] == k; ++t) {
        const uint32_t v = cv[t];
        if (v & kCurrent) cur = true;
        else o = v;
    }
    uint32_t tk, ms;
    uint64_t sn;
    if (cur) {  // pairs.rs:64-67: bound this tick
        tk = (o >= 0 ? ticks[o] : 0u) + 1u;
        ms = 0u;
        sn = o >= 0 ? since[o] : kNever;
    } else {  // pairs.rs:69-84: open but absent
        tk = ticks[o];
        ms = miss[o] + 1u;
        sn = since[o];
        if (ms >= debounce) {
            atomicAdd(&dc[1], 1ull);
            atomicAdd(&dc[2], (unsigned long long)tk);
            if (sn != kNever) {
                atomicAdd(&dc[3], 1ull);
                atomicAdd(&dc[4], (unsigned long long)(now - sn));
            }
            return;
        }
    }
    const uint32_t a = (uint32_t)(k >> 32), b = (uint32_t)k;
    const int ea = elem[pos_of_slot[a]], eb = elem[pos_of_slot[b]];
    const bool p = tk >= thr[ea * kNElem + eb];
    if (p && sn == kNever) sn = now;  // active_since.entry(p).or_insert(now), bonds.rs:169-171
    keep[s] = 1u;
    pers[s] = p ? 1u : 0u;
    nkey[s] = k;
    nticks[s] = tk;
    nmiss[s] = ms;
    nsince[s] = sn;
}

__global__ void k_bt_compact(size_t total, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ keep_pos,
                             const uint32_t* __restrict__ pers, const uint32_t* __restrict__ pers_pos,
                             const uint64_t* __restrict__ nkey, const uint32_t* __restrict__ nticks,
                             const uint32_t* __restrict__ nmiss, const uint64_t* __restrict__ nsince,
                             uint64_t* __restrict__ key, uint32_t* __restrict__ ticks, uint32_t* __restrict__ miss,
                             uint64_t* __restrict__ since, uint32_t* __restrict__ bonds, uint32_t* __restrict__ mark,
                             const uint8_t* __restrict__ elem, const uint32_t* __restrict__ pos_of_slot,
                             unsigned long long* __restrict__ dc) {
    size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total) return;
    if (s == total - 1) {
        dc[106] = keep_pos[s] + keep[s];
        dc[107] = pers_pos[s] + pers[s];
    }
    if (!keep[s]) return;
    const uint32_t q = keep_pos[s];
    key[q] = nkey[s];
    ticks[q] = nticks[s];
    miss[q] = nmiss[s];
    since[q] = nsince[s];
    if (!pers[s]) return;
    const uint32_t a = (uint32_t)(nkey[s] >> 32), b = (uint32_t)nkey[s];
    const uint32_t w = pers_pos[s];
    if (bonds) {
        bonds[2 * w] = a;
        bonds[2 * w + 1] = b;
    }
    const int ea = elem[pos_of_slot[a]], eb = elem[pos_of_slot[b]];
    atomicAdd(&dc[6 + ea * kNElem + eb], 1ull);  // bonds.rs:143-147
    atomicAdd(&dc[6 + eb * kNElem + ea], 1ull);
    if (atomicExch(&mark[a], 1u) == 0u) atomicAdd(&dc[5], 1ull);
    if (atomicExch(&mark[b], 1u) == 0u) atomicAdd(&dc[5], 1ull);
}

}  // namespace

struct BondTracker {
    size_t cap = 0;   // open episodes + bound pairs a merge can hold
    size_t bcap = 0;  // bound pairs of one tick
    size_t ncap = 0;  // atoms (marks)
    size_t M = 0;     // open episodes
    uint64_t *key = nullptr, *since = nullptr, *ck = nullptr, *ck2 = nullptr, *nkey = nullptr, *nsince = nullptr;
    uint32_t *ticks = nullptr, *miss = nullptr, *cv = nullptr, *cv2 = nullptr, *nticks = nullptr, *nmiss = nullptr;
    uint32_t *keep = nullptr, *keep_pos = nullptr, *pers = nullptr, *pers_pos = nullptr;
    uint32_t *bound = nullptr, *mark = nullptr, *thr = nullptr;
    unsigned long long* dc = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    double thr_min_periods = -1.0;
    uint64_t completed = 0, completed_ticks = 0, formed = 0, lifetime = 0;
};

void tracker_free(gx_handle* h) {
    if (!h || !h->tracker) return;
    BondTracker* t = static_cast<BondTracker*>(h->tracker);
    void* ps[] = {t->key, t->since, t->ck, t->ck2, t->nkey, t->nsince, t->ticks, t->miss, t->cv, t->cv2,
                  t->nticks, t->nmiss, t->keep, t->keep_pos, t->pers, t->pers_pos, t->bound, t->mark,
                  t->thr, t->dc, t->temp};
    for (void* p : ps) cudaFree(p);
    delete t;
    h->tracker = nullptr;
}

namespace {

// Grows the merge arrays to hold `need` entries, keeping the open episodes.
int ensure_merge(gx_handle* h, BondTracker* t, size_t need) {
    if (need <= t->cap) return GX_OK;
    size_t cap = need + need / 2 + 1024;
    auto grow = [&](void** p, size_t elem, bool keep_old) -> int {
        void* q = nullptr;
        GX_CUDA(h, cudaMalloc(&q, cap * elem));
        if (keep_old && *p && t->M) GX_CUDA(h, cudaMemcpyAsync(q, *p, t->M * elem, cudaMemcpyDeviceToDevice, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        cudaFree(*p);
        *p = q;
        return GX_OK;
    };
    int rc = 0;
    rc |= grow((void**)&t->key, 8, true);
    rc |= grow((void**)&t->since, 8, true);
    rc |= grow((void**)&t->ticks, 4, true);
    rc |= grow((void**)&t->miss, 4, true);
    rc |= grow((void**)&t->ck, 8, false);
    rc |= grow((void**)&t->ck2, 8, false);
    rc |= grow((void**)&t->nkey, 8, false);
    rc |= grow((void**)&t->nsince, 8, false);
    rc |= grow((void**)&t->cv, 4, false);
    rc |= grow((void**)&t->cv2, 4, false);
    rc |= grow((void**)&t->nticks, 4, false);
    rc |= grow((void**)&t->nmiss, 4, false);
    rc |= grow((void**)&t->keep, 4, false);
    rc |= grow((void**)&t->keep_pos, 4, false);
    rc |= grow((void**)&t->pers, 4, false);
    rc |= grow((void**)&t->pers_pos, 4, false);
    if (rc) return GX_ERR_OOM;
    t->cap = cap;
    // temporary storage for the sort and the two scans at this capacity
    size_t b1 = 0, b2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, t->ck, t->ck2, t->cv, t->cv2, (int)cap, 0, 64, h->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, t->keep, t->keep_pos, (int)cap, h->stream);
    size_t b = b1 > b2 ? b1 : b2;
    if (b > t->temp_bytes) {
        cudaFree(t->temp);
        t->temp = nullptr;
        GX_CUDA(h, cudaMalloc(&t->temp, b));
        t->temp_bytes = b;
    }
    return GX_OK;
}

int upload_thresholds(gx_handle* h, BondTracker* t, double min_periods) {
    if (t->thr_min_periods == min_periods && t->thr) return GX_OK;
    if (!t->thr) GX_CUDA(h, cudaMalloc(&t->thr, kNElem * kNElem * sizeof(uint32_t)));
    uint32_t thr[kNElem * kNElem];
    const double mp = std::fmax(min_periods, 0.1);  // bonds.rs:49
    for (int a = 0; a < kNElem; ++a)
        for (int b = 0; b < kNElem; ++b) {  // threshold_ticks, bonds.rs:94-99
            double mu = kElemMass[a] * kElemMass[b] / (kElemMass[a] + kElemMass[b]);
            double eps = h->p.thermal_constant * std::sqrt(h->p.epsilon_k[a] * h->p.epsilon_k[b]);
            double sig = 0.5 * (h->p.sigma[a] + h->p.sigma[b]);
            double k = 72.0 * std::pow(2.0, -1.0 / 3.0) * eps / (sig * sig);  // well_curvature, forces.rs:194-196
            double period = 2.0 * 3.14159265358979323846 * std::sqrt(mu / k);  // vib_period, forces.rs:201-203
            double v = std::ceil(mp * period / h->p.dt);
            thr[a * kNElem + b] = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
        }
    GX_CUDA(h, cudaMemcpy(t->thr, thr, sizeof thr, cudaMemcpyHostToDevice));
    t->thr_min_periods = min_periods;
    return GX_OK;
}

}  // namespace
}  // namespace gx

using namespace gx;

extern "C" {

int gx_bond_observe(gx_handle* h, double k_bind, double min_periods, int debounce, uint64_t tick, int apply_bonds,
                    gx_bond_observation* out) {
    if (!h || !out || debounce < 1 || !(k_bind > 0.0)) return GX_ERR_ARG;
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    if (!h->tracker) h->tracker = new BondTracker();
    BondTracker* t = static_cast<BondTracker*>(h->tracker);
    const size_t n = h->n;
    int rc = upload_thresholds(h, t, min_periods);
    if (rc) return rc;
    if (!t->dc) GX_CUDA(h, cudaMalloc(&t->dc, kNCount * sizeof(unsigned long long)));
    if (t->ncap < n || !t->mark) {
        cudaFree(t->mark);
        t->mark = nullptr;
        GX_CUDA(h, cudaMalloc(&t->mark, (n ? n : 1) * sizeof(uint32_t)));
        t->ncap = n;
    }
    if (t->bcap < 8 * n + 1024 || !t->bound) {
        cudaFree(t->bound);
        t->bound = nullptr;
        t->bcap = 8 * n + 1024;
        GX_CUDA(h, cudaMalloc(&t->bound, 2 * t->bcap * sizeof(uint32_t)));
    }
    // 1. bound pairs; grow and repeat once if this tick has more than fit
    unsigned long long C = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        GX_CUDA(h, cudaMemsetAsync(t->dc, 0, kNCount * sizeof(unsigned long long), h->stream));
        if ((rc = bound_pairs_device(h, k_bind, t->bound, t->bcap, t->dc))) return rc;
        GX_CUDA(h, cudaMemcpyAsync(&C, t->dc, sizeof C, cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        if (C <= t->bcap) break;
        cudaFree(t->bound);
        t->bound = nullptr;
        t->bcap = (size_t)C + C / 2;
        GX_CUDA(h, cudaMalloc(&t->bound, 2 * t->bcap * sizeof(uint32_t)));
    }
    if (C > t->bcap) return set_err(h, GX_ERR_CAPACITY, "bound-pair buffer");
    const size_t M = t->M, total = M + (size_t)C;
    if ((rc = ensure_merge(h, t, total))) return rc;
    // the bond list must hold every persistent pair (at most all of them)
    const bool grow_bonds = apply_bonds && total > h->bonds_cap;
    if (grow_bonds) {
        cudaFree(h->bonds);
        h->bonds = nullptr;
        size_t bc = total + total / 2 + 1024;
        GX_CUDA(h, cudaMalloc(&h->bonds, 2 * bc * sizeof(uint32_t)));
        h->bonds_cap = bc;
        h->nbonds = 0;
    }
    StateBuf& b = h->buf[h->cur];
    uint64_t persistent = 0, open_after = 0, counts[kNCount];
    std::memset(counts, 0, sizeof counts);
    if (total) {
        // 2. sort the open keys and this tick's keys together
        GX_LAUNCH(h, k_bt_keys, nblk(total, 256), 256, t->key, M, t->bound, (size_t)C, t->ck, t->cv);
        int bits = 1;
        while (bits < 32 && (1ull << bits) < (unsigned long long)n) ++bits;
        size_t tb = t->temp_bytes;
        GX_CUDA(h, cub::DeviceRadixSort::SortPairs(t->temp, tb, t->ck, t->ck2, t->cv, t->cv2, (int)total, 0, 32 + bits,
                                                    h->stream));
        // 3. advance every episode
        GX_LAUNCH(h, k_bt_merge, nblk(total, 256), 256, t->ck2, t->cv2, total, t->ticks, t->miss, t->since, t->nkey,
                  t->nticks, t->nmiss, t->nsince, t->keep, t->pers, t->thr, b.elem, h->pos_of_slot,
                  (uint32_t)debounce, tick, t->dc);
        // 4. compact the open set, emit the persistent pairs
        tb = t->temp_bytes;
        GX_CUDA(h, cub::DeviceScan::ExclusiveSum(t->temp, tb, t->keep, t->keep_pos, (int)total, h->stream));
        tb = t->temp_bytes;
        GX_CUDA(h, cub::DeviceScan::ExclusiveSum(t->temp, tb, t->pers, t->pers_pos, (int)total, h->stream));
        GX_CUDA(h, cudaMemsetAsync(t->mark, 0, (n ? n : 1) * sizeof(uint32_t), h->stream));
        GX_LAUNCH(h, k_bt_compact, nblk(total, 256), 256, total, t->keep, t->keep_pos, t->pers, t->pers_pos,
                  t->nkey, t->nticks, t->nmiss, t->nsince, t->key, t->ticks, t->miss, t->since,
                  apply_bonds ? h->bonds : nullptr, t->mark, b.elem, h->pos_of_slot, t->dc);
        GX_CUDA(h, cudaMemcpyAsync(counts, t->dc, sizeof counts, cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        GX_CUDA(h, cudaGetLastError());
        open_after = counts[106];
        persistent = counts[107];
    }
    t->M = (size_t)open_after;
    t->completed += counts[1];
    t->completed_ticks += counts[2];
    t->formed += counts[3];
    t->lifetime += counts[4];
    if (apply_bonds) bonds_changed(h, (size_t)persistent, grow_bonds);
    out->tick = tick;
    out->bound_pairs = C;
    out->bonded_pairs = persistent;
    out->bonded_entities = counts[5];
    out->mean_coordination = counts[5] ? 2.0 * (double)persistent / (double)counts[5] : 0.0;  // bonds.rs:173-177
    out->bonds_formed = t->formed;
    out->lifetime_sum_ticks = (double)t->lifetime;
    out->open_episodes = open_after;
    out->completed_episodes = t->completed;
    out->completed_ticks = t->completed_ticks;
    for (int k = 0; k < kNElem * kNElem; ++k) out->species_matrix[k] = counts[6 + k];
    return GX_OK;
}

int gx_bond_tracker_reset(gx_handle* h) {
    if (!h) return GX_ERR_ARG;
    tracker_free(h);
    return GX_OK;
}

int gx_get_bonds(gx_handle* h, uint32_t* pairs, size_t cap, size_t* nbonds) {
    if (!h || !nbonds || (cap && !pairs)) return GX_ERR_ARG;
    *nbonds = h->nbonds;
    size_t w = h->nbonds < cap ? h->nbonds : cap;
    if (w) {
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        GX_CUDA(h, cudaMemcpy(pairs, h->bonds, 2 * w * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    return h->nbonds > cap ? set_err(h, GX_ERR_CAPACITY, "bond buffer too small") : GX_OK;
}

}  // extern "C"
