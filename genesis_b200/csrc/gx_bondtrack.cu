// gx_bondtrack.cu -- bond observation on the device: BondObservationSystem::run
// (src/systems/bonds.rs:73-185) with its PairTracker (src/analysis/pairs.rs:38-94).
//
// The reference keeps the open episodes in hash maps on the host.  Here a
// pair (slot a < slot b; the slot-entity map is fixed for a handle) belongs
// to its lower slot, and the open episodes of slot a sit in column a of
// slabs laid out [k * stride + a], k < count[a], sorted by b, so that one
// thread per slot reads them coalesced.  One observation:
//
//   1. the tick's bound pairs (bound_pairs_with_grid, pairs.rs:132-174) are
//      appended to their owner's bucket, in the same column layout;
//   2. one thread per slot sorts its bucket and merges it with its open
//      episodes: each episode's new tick count, missing count and
//      persistence (track_tick, pairs.rs:61-85; threshold bonds.rs:94-99),
//      closing it after `debounce` absent ticks -- a closed persistent pair
//      is a formed bond with lifetime now - since (bonds.rs:155-167);
//   3. a scan of the per-slot persistent counts places the persistent pairs,
//      in (a, b) order, in the handle's bond list (the Bonds component the
//      next force pass reads, bonds.rs:116-121), with the species matrix and
//      the number of bonded atoms, and commits the new episodes.
// Every launch is sized by the atom count alone, so after a first eager
// observation the launches are captured as a CUDA graph (one per cell-buffer
// parity; the tick number is read from device memory), and the host
// synchronises once, for the summary.  A bucket, slab or bond list too shallow for the
// tick leaves the open episodes as they were: the host deepens it and
// observes the tick again.  Every count is an integer, so the result does
// not depend on scheduling.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstring>

#include "gx_internal.cuh"

namespace gx {

int bound_buckets_device(gx_handle* h, void** pool, double k_bind, uint32_t* bucket, uint32_t* bcnt, uint32_t depth,
                         size_t stride);
void aux_pool_free(void* pool);
void bound_list_key(const gx_handle* h, double k_bind, const void** list, const void** start);
void bonds_changed(gx_handle* h, size_t nbonds, bool realloc);

namespace {

constexpr uint64_t kNever = ~0ull;
// A new episode's missing-count word: the count in bits 0-15, and for a
// persistent pair the flag kPers with its rank among the column's
// persistent pairs in bits 16-30.
constexpr uint32_t kPers = 0x80000000u;
constexpr uint32_t kMissMask = 0xFFFFu;
constexpr uint32_t kMaxDebounce = 0xFFFFu, kMaxSlab = 0x7FFFu;
constexpr int kThreads = 64;  // 512 blocks at 32,768 atoms: every SM busy
// device counters: [0] bound pairs this tick, [1] completed episodes,
// [2] their ticks, [3] bonds formed, [4] lifetime sum, [5] bonded atoms,
// [6..105] species matrix, [106] open episodes after, [107] persistent pairs,
// [108] deepest bucket when deeper than allotted, [109] deepest slab column
// likewise, [110] nonzero when the tick was not committed
constexpr int kNCount = 112;
constexpr int kOpenAfter = 106, kPersistent = 107, kNeedBucket = 108, kNeedSlab = 109, kRedo = 110;
// AtomType::mass, src/components/atom_type.rs:80-93
const double kElemMass[kNElem] = {1.008, 4.0026, 12.011, 14.007, 15.999, 22.99, 28.085, 30.974, 32.06, 55.845};

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// Open episodes of every slot, column layout.
struct Slab {
    uint32_t* b = nullptr;      // partner slot
    uint32_t* ticks = nullptr;  // ticks bound (pairs.rs:64-67)
    uint32_t* miss = nullptr;   // consecutive absent ticks
    uint64_t* since = nullptr;  // tick the pair became persistent, or never
    uint32_t* cnt = nullptr;    // episodes per slot
};

namespace {

// A slot's column: this tick's partners and its open episodes, read from the
// bucket and slab (Global) or from per-thread copies when short (Local).
struct GlobalCol {
    uint32_t* bucket;
    const Slab* o;
    size_t S;
    uint32_t a;
    __device__ uint32_t cur(uint32_t i) const { return bucket[(size_t)i * S + a]; }
    __device__ void set_cur(uint32_t i, uint32_t v) const { bucket[(size_t)i * S + a] = v; }
    __device__ uint32_t b(uint32_t j) const { return o->b[(size_t)j * S + a]; }
    __device__ uint32_t ticks(uint32_t j) const { return o->ticks[(size_t)j * S + a]; }
    __device__ uint32_t miss(uint32_t j) const { return o->miss[(size_t)j * S + a]; }
    __device__ uint64_t since(uint32_t j) const { return o->since[(size_t)j * S + a]; }
};

constexpr uint32_t kLocal = 16;

struct LocalCol {
    uint32_t c_[kLocal], b_[kLocal], t_[kLocal], m_[kLocal];
    uint64_t s_[kLocal];
    __device__ uint32_t cur(uint32_t i) const { return c_[i]; }
    __device__ void set_cur(uint32_t i, uint32_t v) { c_[i] = v; }
    __device__ uint32_t b(uint32_t j) const { return b_[j]; }
    __device__ uint32_t ticks(uint32_t j) const { return t_[j]; }
    __device__ uint32_t miss(uint32_t j) const { return m_[j]; }
    __device__ uint64_t since(uint32_t j) const { return s_[j]; }
};

struct MergeOut {
    uint32_t nw, np;
    unsigned long long done, done_ticks, formed, life;
};

// Sorts the column's c partners and merges them with its oc open episodes:
// track_tick (pairs.rs:61-85) and the persistence and bond bookkeeping of
// BondObservationSystem::run (bonds.rs:130-171) for one slot.
template <class Col>
__device__ MergeOut merge_column(Col& col, uint32_t c, uint32_t oc, uint32_t a, int ea, size_t S, uint32_t slab,
                                 const Slab& w, const uint32_t* sthr, const uint8_t* __restrict__ eslot,
                                 uint32_t* __restrict__ mark, unsigned int* sm, uint32_t debounce, uint64_t now) {
    for (uint32_t i = 1; i < c; ++i) {  // ascending (a column holds a few)
        const uint32_t v = col.cur(i);
        uint32_t j = i;
        for (; j > 0; --j) {
            const uint32_t u = col.cur(j - 1);
            if (u <= v) break;
            col.set_cur(j, u);
        }
        col.set_cur(j, v);
    }
    MergeOut r = {0u, 0u, 0ull, 0ull, 0ull, 0ull};
    uint32_t i = 0, j = 0, last = 0xFFFFFFFFu;
    while (i < c || j < oc) {
        const uint32_t bc = i < c ? col.cur(i) : 0xFFFFFFFFu;
        if (i < c && bc == last) {  // the same pair twice (an axis of 2 cells)
            ++i;
            continue;
        }
        const uint32_t bo = j < oc ? col.b(j) : 0xFFFFFFFFu;
        uint32_t b, tk, ms;
        uint64_t sn;
        if (bc <= bo) {  // pairs.rs:64-67: bound this tick
            b = bc;
            last = bc;
            ++i;
            if (bc == bo) {
                tk = col.ticks(j) + 1u;
                sn = col.since(j);
                ++j;
            } else {
                tk = 1u;
                sn = kNever;
            }
            ms = 0u;
        } else {  // pairs.rs:69-84: open but absent
            b = bo;
            tk = col.ticks(j);
            ms = col.miss(j) + 1u;
            sn = col.since(j);
            ++j;
            if (ms >= debounce) {
                ++r.done;
                r.done_ticks += tk;
                if (sn != kNever) {
                    ++r.formed;
                    r.life += now - sn;
                }
                continue;
            }
        }
        const int eb = eslot[b];
        const bool p = tk >= sthr[ea * kNElem + eb];
        if (p && sn == kNever) sn = now;  // active_since.entry(p).or_insert(now), bonds.rs:169-171
        if (r.nw < slab) {
            const size_t q = (size_t)r.nw * S + a;
            w.b[q] = b;
            w.ticks[q] = tk;
            w.miss[q] = ms | (p ? kPers | (r.np << 16) : 0u);
            w.since[q] = sn;
        }
        ++r.nw;
        if (p) {
            ++r.np;
            mark[a] = 1u;
            mark[b] = 1u;
            atomicAdd(&sm[ea * kNElem + eb], 1u);  // bonds.rs:143-147
            atomicAdd(&sm[eb * kNElem + ea], 1u);
        }
    }
    return r;
}

__global__ void __launch_bounds__(kThreads)
    k_bt_merge(uint32_t n, size_t S, uint32_t depth, uint32_t slab, uint32_t* __restrict__ bucket,
               const uint32_t* __restrict__ bcnt, Slab o, Slab w, uint32_t* __restrict__ pcnt,
               uint32_t* __restrict__ mark, const uint32_t* __restrict__ thr, const uint8_t* __restrict__ eslot,
               uint32_t debounce, const uint64_t* __restrict__ now_p, unsigned long long* __restrict__ dc) {
    __shared__ unsigned long long sc[6];  // completed, their ticks, formed, lifetime, open after, bound pairs
    __shared__ unsigned int sm[kNElem * kNElem];
    __shared__ uint32_t sthr[kNElem * kNElem];
    for (int k = threadIdx.x; k < kNElem * kNElem; k += kThreads) {
        sm[k] = 0u;
        sthr[k] = thr[k];
    }
    if (threadIdx.x < 6) sc[threadIdx.x] = 0ull;
    __syncthreads();
    const uint32_t a = blockIdx.x * kThreads + threadIdx.x;
    if (a < n) {
        uint32_t c = bcnt[a];
        if (c) atomicAdd(&sc[5], (unsigned long long)c);  // every pair found, repeats included
        if (c > depth) {
            atomicMax(&dc[kNeedBucket], (unsigned long long)c);
            c = depth;
        }
        const uint32_t oc = o.cnt[a];
        const uint64_t now = *now_p;
        const int ea = eslot[a];
        MergeOut r;
        if (c <= kLocal && oc <= kLocal) {
            LocalCol col;  // independent loads, issued together
            for (uint32_t i = 0; i < c; ++i) col.c_[i] = bucket[(size_t)i * S + a];
            for (uint32_t j = 0; j < oc; ++j) {
                const size_t e = (size_t)j * S + a;
                col.b_[j] = o.b[e];
                col.t_[j] = o.ticks[e];
                col.m_[j] = o.miss[e];
                col.s_[j] = o.since[e];
            }
            r = merge_column(col, c, oc, a, ea, S, slab, w, sthr, eslot, mark, sm, debounce, now);
        } else {
            GlobalCol col{bucket, &o, S, a};
            r = merge_column(col, c, oc, a, ea, S, slab, w, sthr, eslot, mark, sm, debounce, now);
        }
        if (r.nw > slab) atomicMax(&dc[kNeedSlab], (unsigned long long)r.nw);
        w.cnt[a] = r.nw < slab ? r.nw : slab;
        pcnt[a] = r.np;
        if (r.done) {
            atomicAdd(&sc[0], r.done);
            atomicAdd(&sc[1], r.done_ticks);
        }
        if (r.formed) {
            atomicAdd(&sc[2], r.formed);
            atomicAdd(&sc[3], r.life);
        }
        if (r.nw) atomicAdd(&sc[4], (unsigned long long)r.nw);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kNElem * kNElem; k += kThreads)
        if (sm[k]) atomicAdd(&dc[6 + k], (unsigned long long)sm[k]);
    if (threadIdx.x < 4 && sc[threadIdx.x]) atomicAdd(&dc[1 + threadIdx.x], sc[threadIdx.x]);
    if (threadIdx.x == 4 && sc[4]) atomicAdd(&dc[kOpenAfter], sc[4]);
    if (threadIdx.x == 5 && sc[5]) atomicAdd(&dc[0], sc[5]);
}

// The element of every slot (fixed while the tracker lives).
__global__ void k_bt_eslot(uint32_t n, const uint8_t* __restrict__ elem, const uint32_t* __restrict__ pos_of_slot,
                           uint8_t* __restrict__ eslot) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < n) eslot[a] = elem[pos_of_slot[a]];
}

// One thread per slab entry (blockIdx.y = row): commits this tick's
// episodes and writes the persistent pairs at their column's offset plus
// their rank, so that no thread walks a column.
__global__ void __launch_bounds__(kThreads)
    k_bt_emit(uint32_t n, size_t S, uint32_t depth, uint32_t slab, size_t bonds_cap, Slab w, Slab o,
              const uint32_t* __restrict__ pcnt, const uint32_t* __restrict__ poff, const uint32_t* __restrict__ mark,
              uint32_t* __restrict__ bonds, unsigned long long* __restrict__ nbonds_dev,
              unsigned long long* __restrict__ dc) {
    __shared__ unsigned int smark;
    if (threadIdx.x == 0) smark = 0u;
    __syncthreads();
    // the same decision in every thread: the scan and the overflow maxima
    // are complete before this launch
    const unsigned long long total = n ? (unsigned long long)poff[n - 1] + pcnt[n - 1] : 0ull;
    const bool redo = dc[kNeedBucket] > depth || dc[kNeedSlab] > slab || (bonds && total > bonds_cap);
    const uint32_t a = blockIdx.x * kThreads + threadIdx.x;
    const uint32_t k = blockIdx.y;
    if (k == 0) {
        if (a < n && mark[a]) atomicAdd(&smark, 1u);
        if (a == 0) {
            dc[kPersistent] = total;
            if (redo) dc[kRedo] = 1ull;
            else if (bonds) *nbonds_dev = total;
        }
    }
    if (a < n && !redo) {
        const uint32_t c = w.cnt[a];
        if (k == 0) o.cnt[a] = c;
        if (k < c) {
            const size_t e = (size_t)k * S + a;
            const uint32_t b = w.b[e], m = w.miss[e];
            o.b[e] = b;
            o.ticks[e] = w.ticks[e];
            o.miss[e] = m & kMissMask;
            o.since[e] = w.since[e];
            if ((m & kPers) && bonds) {
                const size_t q = (size_t)poff[a] + ((m >> 16) & kMaxSlab);
                bonds[2 * q] = a;
                bonds[2 * q + 1] = b;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && smark) atomicAdd(&dc[5], (unsigned long long)smark);
}

}  // namespace

// What a captured observation depends on.
struct ObsKey {
    uint64_t n, depth, slab, apply, debounce, bonds_cap;
    double k_bind;
    const void *bonds, *pos_of_slot, *elem, *x, *bucket, *open, *next, *list, *list_start;
};

struct BondTracker {
    size_t S = 0;        // column stride: the handle's atom capacity
    uint32_t depth = 0;  // bucket rows
    uint32_t slab = 0;   // open-episode rows
    Slab open, next;     // committed episodes, this tick's
    uint32_t *bucket = nullptr, *bcnt = nullptr, *pcnt = nullptr, *poff = nullptr, *mark = nullptr;
    uint32_t* thr = nullptr;
    uint8_t* eslot = nullptr;  // element of each slot
    unsigned long long* dc = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    double thr_min_periods = -1.0;
    uint64_t completed = 0, completed_ticks = 0, formed = 0, lifetime = 0;
    void* aux = nullptr;                   // bond-grid staging (gx_lens.cu)
    uint64_t* dnow = nullptr;              // the tick observed (device)
    uint64_t* hnow = nullptr;              // its pinned host copy
    unsigned long long* hcounts = nullptr;  // pinned summary
    bool warm = false;                     // an eager observation has allocated everything
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    ObsKey gkey[2];
    uint64_t gkernels[2] = {0, 0};
};

static void slab_free(Slab& s) {
    void* ps[] = {s.b, s.ticks, s.miss, s.since, s.cnt};
    for (void* p : ps) cudaFree(p);
    s = Slab();
}

void tracker_free(gx_handle* h) {
    if (!h || !h->tracker) return;
    BondTracker* t = static_cast<BondTracker*>(h->tracker);
    slab_free(t->open);
    slab_free(t->next);
    void* ps[] = {t->bucket, t->bcnt, t->pcnt, t->poff, t->mark, t->thr, t->dc, t->temp, t->dnow, t->eslot};
    for (void* p : ps) cudaFree(p);
    cudaFreeHost(t->hnow);
    cudaFreeHost(t->hcounts);
    for (auto& g : t->gexec)
        if (g) cudaGraphExecDestroy(g);
    aux_pool_free(t->aux);
    delete t;
    h->tracker = nullptr;
}

namespace {

// A slab of `rows` rows into `s`; with `old`, its first `keep_rows` rows and
// its counts are carried over (same stride; `old` may be `s`).
int slab_alloc(gx_handle* h, Slab& s, size_t S, uint32_t rows, const Slab* old, uint32_t keep_rows) {
    Slab t;
    const size_t m = (size_t)rows * S;
    GX_CUDA(h, cudaMalloc(&t.b, m * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t.ticks, m * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t.miss, m * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t.since, m * sizeof(uint64_t)));
    GX_CUDA(h, cudaMalloc(&t.cnt, S * sizeof(uint32_t)));
    if (old && old->b) {
        const size_t k = (size_t)keep_rows * S;
        GX_CUDA(h, cudaMemcpyAsync(t.b, old->b, k * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(t.ticks, old->ticks, k * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(t.miss, old->miss, k * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(t.since, old->since, k * sizeof(uint64_t), cudaMemcpyDeviceToDevice, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(t.cnt, old->cnt, S * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
    } else {
        GX_CUDA(h, cudaMemsetAsync(t.cnt, 0, S * sizeof(uint32_t), h->stream));
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    slab_free(s);
    s = t;
    return GX_OK;
}

// First use: per-slot arrays at the handle's capacity, shallow bucket and slabs.
int tracker_init(gx_handle* h, BondTracker* t) {
    if (t->dc) return GX_OK;
    const size_t S = h->cap;
    t->S = S;
    t->depth = 8;
    t->slab = 8;
    GX_CUDA(h, cudaMalloc(&t->dc, kNCount * sizeof(unsigned long long)));
    GX_CUDA(h, cudaMalloc(&t->dnow, sizeof(uint64_t)));
    GX_CUDA(h, cudaMallocHost(&t->hnow, sizeof(uint64_t)));
    GX_CUDA(h, cudaMallocHost(&t->hcounts, kNCount * sizeof(unsigned long long)));
    GX_CUDA(h, cudaMalloc(&t->bucket, (size_t)t->depth * S * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t->bcnt, S * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t->pcnt, S * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t->poff, S * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t->mark, S * sizeof(uint32_t)));
    GX_CUDA(h, cudaMalloc(&t->eslot, S));
    if (h->n)
        GX_LAUNCH(h, k_bt_eslot, nblk(h->n, 256), 256, (uint32_t)h->n, h->buf[h->cur].elem, h->pos_of_slot, t->eslot);
    int rc = slab_alloc(h, t->open, S, t->slab, nullptr, 0);
    if (!rc) rc = slab_alloc(h, t->next, S, t->slab, nullptr, 0);
    if (rc) return rc;
    size_t tb = 0;
    GX_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, tb, t->pcnt, t->poff, (int)S, h->stream));
    GX_CUDA(h, cudaMalloc(&t->temp, tb ? tb : 1));
    t->temp_bytes = tb;
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

// The launches of one observation, from the tick number in t->dnow to the
// summary in t->hcounts.
int observe_launches(gx_handle* h, BondTracker* t, double k_bind, uint32_t debounce, bool apply) {
    const uint32_t n = (uint32_t)h->n;
    const size_t S = t->S;
    GX_CUDA(h, cudaMemsetAsync(t->dc, 0, kNCount * sizeof(unsigned long long), h->stream));
    if (n) {
        GX_CUDA(h, cudaMemsetAsync(t->bcnt, 0, n * sizeof(uint32_t), h->stream));
        GX_CUDA(h, cudaMemsetAsync(t->mark, 0, n * sizeof(uint32_t), h->stream));
        int rc = bound_buckets_device(h, &t->aux, k_bind, t->bucket, t->bcnt, t->depth, S);
        if (rc) return rc;
        prof_begin(h, "bond_merge");
        GX_LAUNCH(h, k_bt_merge, nblk(n, kThreads), kThreads, n, S, t->depth, t->slab, t->bucket, t->bcnt, t->open,
                  t->next, t->pcnt, t->mark, t->thr, t->eslot, debounce, t->dnow, t->dc);
        size_t tb = t->temp_bytes;
        GX_CUDA(h, cub::DeviceScan::ExclusiveSum(t->temp, tb, t->pcnt, t->poff, (int)n, h->stream));
        GX_LAUNCH(h, k_bt_emit, dim3(nblk(n, kThreads), t->slab), kThreads, n, S, t->depth, t->slab,
                  apply ? h->bonds_cap : 0,
                  t->next, t->open, t->pcnt, t->poff, t->mark, apply ? h->bonds : nullptr, dnbonds(h), t->dc);
        prof_end(h, "bond_merge");
    } else if (apply) {
        GX_CUDA(h, cudaMemsetAsync(dnbonds(h), 0, sizeof(unsigned long long), h->stream));
    }
    GX_CUDA(h, cudaMemcpyAsync(t->hcounts, t->dc, kNCount * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               h->stream));
    return GX_OK;
}

// One attempt at the tick, captured once its launches are known to need no
// allocation; the summary lands in t->hcounts.
int observe_once(gx_handle* h, BondTracker* t, double k_bind, uint32_t debounce, uint64_t tick, bool apply,
                 bool graph) {
    *t->hnow = tick;  // the previous observation synchronised: its copy has run
    GX_CUDA(h, cudaMemcpyAsync(t->dnow, t->hnow, sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream));
    if (!graph || !t->warm || h->prof_on) {
        int rc = observe_launches(h, t, k_bind, debounce, apply);
        if (rc) return rc;
    } else {
        ObsKey k;
        std::memset(&k, 0, sizeof k);
        k.n = h->n;
        k.depth = t->depth;
        k.slab = t->slab;
        k.apply = apply;
        k.debounce = debounce;
        k.bonds_cap = h->bonds_cap;
        k.k_bind = k_bind;
        k.bonds = h->bonds;
        k.pos_of_slot = h->pos_of_slot;
        k.elem = h->buf[h->cur].elem;
        k.x = h->buf[h->cur].x;
        k.bucket = t->bucket;
        k.open = t->open.b;
        k.next = t->next.b;
        bound_list_key(h, k_bind, &k.list, &k.list_start);
        const int par = h->cur & 1;
        if (!t->gexec[par] || std::memcmp(&k, &t->gkey[par], sizeof k) != 0) {
            if (t->gexec[par]) cudaGraphExecDestroy(t->gexec[par]);
            t->gexec[par] = nullptr;
            const uint64_t l0 = h->launches;
            GX_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            int rc = observe_launches(h, t, k_bind, debounce, apply);
            cudaGraph_t gr = nullptr;
            cudaError_t ce = cudaStreamEndCapture(h->stream, &gr);
            if (rc || ce != cudaSuccess) {
                if (gr) cudaGraphDestroy(gr);
                return rc ? rc : cuda_err(h, ce, "cudaStreamEndCapture");
            }
            cudaGraphExec_t ex = nullptr;
            ce = cudaGraphInstantiate(&ex, gr, 0);
            cudaGraphDestroy(gr);
            if (ce != cudaSuccess) return cuda_err(h, ce, "cudaGraphInstantiate");
            t->gexec[par] = ex;
            t->gkey[par] = k;
            t->gkernels[par] = h->launches - l0;
            h->launches = l0;
        }
        GX_CUDA(h, cudaGraphLaunch(t->gexec[par], h->stream));
        h->launches += t->gkernels[par];
    }
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return take_step_errors(h);  // an asynchronous step before this observation
}

}  // namespace
}  // namespace gx

using namespace gx;

extern "C" {

int gx_bond_observe(gx_handle* h, double k_bind, double min_periods, int debounce, uint64_t tick, int apply_bonds,
                    gx_bond_observation* out) {
    if (!h || !out || debounce < 1 || !(k_bind > 0.0)) return GX_ERR_ARG;
    if ((uint32_t)debounce > kMaxDebounce) return set_err(h, GX_ERR_ARG, "debounce above 65535 ticks");
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    if (!h->tracker) h->tracker = new BondTracker();
    BondTracker* t = static_cast<BondTracker*>(h->tracker);
    int rc = tracker_init(h, t);
    if (!rc) rc = upload_thresholds(h, t, min_periods);
    if (rc) return rc;
    bool grew_bonds = false;
    if (apply_bonds && !h->bonds) {  // a first bond list: the spring is on from now
        GX_CUDA(h, cudaMalloc(&h->bonds, 2 * 1024 * sizeof(uint32_t)));
        h->bonds_cap = 1024;
        h->nbonds = 0;
        grew_bonds = true;
    }
    const unsigned long long* counts = t->hcounts;
    for (int attempt = 0;; ++attempt) {
        if ((rc = observe_once(h, t, k_bind, (uint32_t)debounce, tick, apply_bonds != 0, attempt == 0))) return rc;
        if (!counts[kRedo]) break;
        if (attempt >= 3) return set_err(h, GX_ERR_CAPACITY, "bond observation did not fit after deepening");
        // nothing was committed: deepen what overflowed and observe again
        if (counts[kNeedBucket] > t->depth) {
            const uint32_t d = (uint32_t)(counts[kNeedBucket] + counts[kNeedBucket] / 2 + 2);
            cudaFree(t->bucket);
            t->bucket = nullptr;
            GX_CUDA(h, cudaMalloc(&t->bucket, (size_t)d * t->S * sizeof(uint32_t)));
            t->depth = d;
        }
        if (counts[kNeedSlab] > t->slab) {
            if (counts[kNeedSlab] > kMaxSlab)
                return set_err(h, GX_ERR_CAPACITY, "more than 32767 open bond episodes on one atom");
            uint32_t d = (uint32_t)(counts[kNeedSlab] + counts[kNeedSlab] / 2 + 2);
            if (d > kMaxSlab) d = kMaxSlab;
            if ((rc = slab_alloc(h, t->open, t->S, d, &t->open, t->slab))) return rc;
            if ((rc = slab_alloc(h, t->next, t->S, d, nullptr, 0))) return rc;
            t->slab = d;
        }
        if (apply_bonds && counts[kPersistent] > h->bonds_cap) {
            cudaFree(h->bonds);
            h->bonds = nullptr;
            h->nbonds = 0;
            const size_t bc = counts[kPersistent] + counts[kPersistent] / 2 + 1024;
            GX_CUDA(h, cudaMalloc(&h->bonds, 2 * bc * sizeof(uint32_t)));
            h->bonds_cap = bc;
            grew_bonds = true;
        }
    }
    t->warm = true;
    const uint64_t persistent = counts[kPersistent];
    t->completed += counts[1];
    t->completed_ticks += counts[2];
    t->formed += counts[3];
    t->lifetime += counts[4];
    if (apply_bonds) bonds_changed(h, (size_t)persistent, grew_bonds);
    out->tick = tick;
    out->bound_pairs = counts[0];
    out->bonded_pairs = persistent;
    out->bonded_entities = counts[5];
    out->mean_coordination = counts[5] ? 2.0 * (double)persistent / (double)counts[5] : 0.0;  // bonds.rs:173-177
    out->bonds_formed = t->formed;
    out->lifetime_sum_ticks = (double)t->lifetime;
    out->open_episodes = counts[kOpenAfter];
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
