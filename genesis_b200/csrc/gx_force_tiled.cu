// gx_force_tiled.cu -- staged mixed-precision pair passes for sm_100a.
//
// Both kernels here compute the same physics and the same fixed-point sums as
// k_force_mixed (gx_force.cu), bit for bit; they differ in how the work is
// laid out.  Both stage the block's neighbourhood into shared memory first:
//
//  * A block owns a run of home cells along x in one (y, z) row.  Its half
//    shell is the own row (cells x0 .. x0+run) and four forward rows
//    (dy, dz) in {(1,0), (-1,1), (0,1), (1,1)} (cells x0-1 .. x0+run).  Atoms
//    are sorted by cell, so each row span is one contiguous range of pos4
//    (two when it wraps in x): stage_rows copies them into shared memory with
//    cp.async.bulk, completing on one mbarrier (bounded wait).
//
//  k_force_mixed_tiled (variant 2): a warp per home cell walks the 14 tiles
//    (A,A) with j > i, (A, A+x) and the 12 forward-row cells, testing 32
//    (i, j) candidates per step and compacting the pairs in the cutoff into a
//    ring queue with __ballot_sync; 32 queued pairs are evaluated at a time.
//  k_force_mixed_rows (variant 3): a thread per home atom walks the same 14
//    cells, appends every candidate inside the cutoff to a private list in
//    shared memory and evaluates the list afterwards, so the pair law never
//    runs inside a divergent filter branch; the i-end sum stays in registers.
//
// The half shell here ({(+1,0,0)} and the 12 forward-row offsets) is a
// different half of the 26 offsets than the reference's canonical one
// (src/physics/grid.rs:275-296); with three or more cells on every axis each
// cell pair is visited exactly once either way, so the pair set is the same.
// Grids with fewer than three cells on an axis use k_force_mixed.
#include "gx_pair_f32.cuh"

namespace gx {

namespace {

constexpr int kRows = 5;                   // own row + 4 forward rows
constexpr int kTiles = 14;
constexpr uint32_t kWaitLimit = 1u << 20;  // bounded mbarrier wait

// forward rows r = 1..4: (dy, dz) = (1,0), (-1,1), (0,1), (1,1); r = 0 is the own row
__device__ __forceinline__ int row_dy(int r) { return (r == 1 || r == 4) ? 1 : (r == 2 ? -1 : 0); }
__device__ __forceinline__ int row_dz(int r) { return r >= 2 ? 1 : 0; }
// tile id -> (row, slot offset from the home slot, dx): tile 0 = own cell,
// 1 = own row +x, 2..13 = forward row 1 + (t-2)/3 at dx = (t-2)%3 - 1.
__device__ __forceinline__ void tile_geom(int t, int& r, int& dslot, int& dx) {
    if (t == 0) { r = 0; dslot = 0; dx = 0; }
    else if (t == 1) { r = 0; dslot = 1; dx = 1; }
    else { int q = t - 2; r = 1 + q / 3; dx = q % 3 - 1; dslot = dx + 1; }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

template <int SLOTS>
struct Stage {
    uint32_t g[kRows][SLOTS];  // first atom of each staged cell in pos4
    uint32_t s[kRows][SLOTS];  // its position in the shared-memory copy
    uint32_t c[kRows][SLOTS];  // atoms in the cell
    unsigned long long mbar;
    uint32_t total;
    int staged;
};

// Fills the cell table of the block's rows and copies their atoms into s_pos
// (when they fit in cap).  Every thread of the block must call it.  Returns
// false when the copy did not complete (the block must exit; err is set).
template <int SLOTS>
__device__ bool stage_rows(Stage<SLOTS>& S, float4* s_pos, uint32_t cap, const GridGeom& g, int run, int x0,
                           uint32_t cy, uint32_t cz, const float4* __restrict__ pos4,
                           const uint32_t* __restrict__ start, uint32_t* err) {
    const int tid = threadIdx.x, nth = blockDim.x;
    const int nsl = run + 2;
    for (int t = tid; t < kRows * nsl; t += nth) {
        int r = t / nsl, s = t - r * nsl;
        int nslots = r == 0 ? run + 1 : run + 2;
        uint32_t gs = 0, cnt = 0;
        if (s < nslots) {
            int xr = r == 0 ? x0 + s : x0 - 1 + s;
            uint32_t ux = (uint32_t)((xr % (int)g.n[0] + (int)g.n[0]) % (int)g.n[0]);
            uint32_t c = encode(g, ux, wrap_add(cy, row_dy(r), g.n[1]), wrap_add(cz, row_dz(r), g.n[2]));
            gs = start[c];
            cnt = start[c + 1] - gs;
        }
        S.g[r][s] = gs;
        S.c[r][s] = cnt;
    }
    __syncthreads();
    const uint32_t mbar = smem_addr(&S.mbar);
    if (tid == 0) {
        uint32_t total = 0;
        for (int r = 0; r < kRows; ++r)
            for (int s = 0; s < nsl; ++s) {
                S.s[r][s] = total;
                total += S.c[r][s];
            }
        S.total = total;
        int staged = total <= cap;
        S.staged = staged;
        if (staged && total) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(total * 16u)
                         : "memory");
            for (int r = 0; r < kRows; ++r) {
                int s = 0;
                while (s < nsl) {
                    uint32_t g0 = S.g[r][s], bytes = 0;
                    int e = s;
                    // merge slots whose atom ranges are adjacent in pos4
                    while (e < nsl && (e == s || S.g[r][e] == S.g[r][e - 1] + S.c[r][e - 1])) {
                        bytes += S.c[r][e] * 16u;
                        ++e;
                    }
                    if (bytes) {
                        uint32_t dst = smem_addr(s_pos + S.s[r][s]);
                        const float4* src = pos4 + g0;
                        asm volatile(
                            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                                dst),
                            "l"(src), "r"(bytes), "r"(mbar)
                            : "memory");
                    }
                    s = e;
                }
            }
        }
    }
    __syncthreads();
    if (S.staged && S.total) {
        auto wait = [&](uint32_t limit) -> bool {
            for (uint32_t it = 0; it < limit; ++it) {
                uint32_t done = 0;
                asm volatile(
                    "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                    : "=r"(done)
                    : "r"(mbar), "r"(0u)
                    : "memory");
                if (done) return true;
            }
            return false;
        };
        bool ok = wait(kWaitLimit);
        if (__syncthreads_or(!ok)) {  // every thread leaves together
            if (!ok) wait(kWaitLimit);  // let copies still in flight land before the block exits
            if (tid == 0) atomicOr(err, kErrTimeout);
            return false;
        }
    }
    return true;
}

// ------------------------------------------------------------------ variant 2

constexpr int kTWarps = 8;
constexpr int kTThreads = kTWarps * 32;
constexpr int kTRunMax = kTWarps;
constexpr int kTSlots = kTRunMax + 2;
constexpr int kTStageCap = 1536;
constexpr int kQ = 64;
constexpr int kHomeCap = 64;

struct TileInfo {
    uint32_t sbase, gbase, cnt, pad;
    float sx, sy, sz, pad2;
};

__global__ void __launch_bounds__(kTThreads, 4)
    k_force_mixed_tiled(GridGeom g, int run, int nbx, const float4* __restrict__ pos4,
                        const uint32_t* __restrict__ start, LawF32 L, const PairF* __restrict__ tab,
                        long long* __restrict__ F, size_t fstride, unsigned long long* __restrict__ vacc,
                        unsigned long long* __restrict__ npairs, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) float4 s_pos[];
    __shared__ PairF s_tab[kMaxKinds * kMaxKinds];
    __shared__ Stage<kTSlots> S;
    __shared__ TileInfo s_tile[kTWarps][kTiles];
    __shared__ uint2 s_q[kTWarps][kQ];
    __shared__ unsigned long long s_acc[kTWarps][kHomeCap * 3];
    __shared__ unsigned long long s_red[kTWarps][2];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t bx = blockIdx.x % nbx, yz = blockIdx.x / nbx;
    const uint32_t cy = yz % g.n[1], cz = yz / g.n[1];
    const int x0 = (int)bx * run;
    for (int t = tid; t < L.nkinds * L.nkinds; t += kTThreads) s_tab[t] = tab[t];
    if (!stage_rows<kTSlots>(S, s_pos, kTStageCap, g, run, x0, cy, cz, pos4, start, err)) return;
    const bool staged = S.staged != 0;
    const float4* P = staged ? (const float4*)s_pos : pos4;

    const bool home = w < run && x0 + w < (int)g.n[0];
    if (lane < kTiles) {
        int r, ds, dx;
        tile_geom(lane, r, ds, dx);
        int slot = w + (r == 0 ? ds : ds);
        TileInfo T;
        T.cnt = home ? S.c[r][slot] : 0u;
        T.gbase = S.g[r][slot];
        T.sbase = staged ? S.s[r][slot] : T.gbase;
        T.sx = -(float)dx * g.cellf[0];
        T.sy = -(float)row_dy(r) * g.cellf[1];
        T.sz = -(float)row_dz(r) * g.cellf[2];
        T.pad = 0;
        T.pad2 = 0.f;
        s_tile[w][lane] = T;
    }
    __syncwarp();
    const uint32_t nA = s_tile[w][0].cnt, sA = s_tile[w][0].sbase, gA = s_tile[w][0].gbase;
    const bool shared_i = nA <= (uint32_t)kHomeCap;
    for (uint32_t k = lane; k < 3 * kHomeCap; k += 32) s_acc[w][k] = 0ull;
    __syncwarp();

    long long vq = 0;
    unsigned long long pcount = 0;
    uint32_t head = 0, tail = 0;
    const int nk = L.nkinds;

    auto compute = [&](uint32_t np) {
        if ((uint32_t)lane < np) {
            uint2 e = s_q[w][(head + lane) & (kQ - 1)];
            uint32_t tl = e.x >> 24, i = e.x & 0xFFFFFFu, j = e.y;
            const TileInfo& T = s_tile[w][tl];
            float4 pi = P[sA + i], pj = P[T.sbase + j];
            float dx = delta1(pi.x, pj.x, T.sx), dy = delta1(pi.y, pj.y, T.sy), dz = delta1(pi.z, pj.z, T.sz);
            float d2 = dist2(dx, dy, dz);
            float fs, v;
            pair_f32(L, s_tab[__float_as_int(pi.w) * nk + __float_as_int(pj.w)], d2, fs, v);
            long long qx, qy, qz;
                quant3(fmul(dx, fs), fmul(dy, fs), fmul(dz, fs), qx, qy, qz, err);
            if (shared_i) {
                atomicAdd(&s_acc[w][3 * i], (unsigned long long)qx);
                atomicAdd(&s_acc[w][3 * i + 1], (unsigned long long)qy);
                atomicAdd(&s_acc[w][3 * i + 2], (unsigned long long)qz);
            } else {
                atomicAdd((unsigned long long*)&F[gA + i], (unsigned long long)qx);
                atomicAdd((unsigned long long*)&F[fstride + gA + i], (unsigned long long)qy);
                atomicAdd((unsigned long long*)&F[2 * fstride + gA + i], (unsigned long long)qz);
            }
            uint32_t gj = T.gbase + j;
            atomicAdd((unsigned long long*)&F[gj], (unsigned long long)(-qx));
            atomicAdd((unsigned long long*)&F[fstride + gj], (unsigned long long)(-qy));
            atomicAdd((unsigned long long*)&F[2 * fstride + gj], (unsigned long long)(-qz));
            vq += quant(v, err);
        }
        __syncwarp();
    };

    if (nA) {
        const unsigned lt_mask = (1u << lane) - 1u;
        for (int tl = 0; tl < kTiles; ++tl) {
            const uint32_t nB = s_tile[w][tl].cnt;
            if (!nB) continue;
            const uint32_t sB = s_tile[w][tl].sbase;
            const float sx = s_tile[w][tl].sx, sy = s_tile[w][tl].sy, sz = s_tile[w][tl].sz;
            const uint32_t total = nA * nB;
            const float inv_nB = 1.0f / (float)nB;
            for (uint32_t t0 = 0; t0 < total; t0 += 32) {
                uint32_t t = t0 + lane;
                bool ok = t < total;
                int i = (int)(((float)t + 0.5f) * inv_nB);
                int j = (int)t - i * (int)nB;
                if (j < 0) { --i; j += (int)nB; }
                else if (j >= (int)nB) { ++i; j -= (int)nB; }
                if (tl == 0) ok = ok && j > i;
                bool pass = false;
                if (ok) {
                    float4 pi = P[sA + i], pj = P[sB + j];
                    float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
                    float d2 = dist2(dx, dy, dz);
                    pass = d2 < L.rc2 && d2 > 0.f;
                }
                unsigned m = __ballot_sync(0xffffffffu, pass);
                if (m) {
                    if (pass)
                        s_q[w][(tail + __popc(m & lt_mask)) & (kQ - 1)] =
                            make_uint2(((uint32_t)tl << 24) | (uint32_t)i, (uint32_t)j);
                    tail += __popc(m);
                    pcount += __popc(m);
                    __syncwarp();
                    if (tail - head >= 32) {
                        compute(32);
                        head += 32;
                    }
                }
            }
        }
        while (tail != head) {
            uint32_t np = tail - head < 32 ? tail - head : 32;
            compute(np);
            head += np;
        }
        if (shared_i) {
            for (uint32_t a = lane; a < nA; a += 32) {
                unsigned long long fx = s_acc[w][3 * a], fy = s_acc[w][3 * a + 1], fz = s_acc[w][3 * a + 2];
                if (fx) atomicAdd((unsigned long long*)&F[gA + a], fx);
                if (fy) atomicAdd((unsigned long long*)&F[fstride + gA + a], fy);
                if (fz) atomicAdd((unsigned long long*)&F[2 * fstride + gA + a], fz);
            }
        }
    }
    unsigned long long u = (unsigned long long)vq;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) u += __shfl_down_sync(0xffffffffu, u, o);
    if (lane == 0) {
        s_red[w][0] = u;
        s_red[w][1] = pcount;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long a = 0, b = 0;
        for (int k = 0; k < kTWarps; ++k) {
            a += s_red[k][0];
            b += s_red[k][1];
        }
        if (a) atomicAdd(vacc, a);
        if (b) atomicAdd(npairs, b);
    }
}

// ------------------------------------------------------------------ variant 3

constexpr int kRThreads = 128;
constexpr int kRRunMax = 12;
constexpr int kRSlots = kRRunMax + 2;
constexpr int kRStageCap = 2048;
constexpr int kLCap = 40;    // per-thread candidate list (u32 entries)
constexpr int kLStep = 20;   // candidates a lane may append between capacity checks

__global__ void __launch_bounds__(kRThreads, 4)
    k_force_mixed_rows(GridGeom g, int run, int nbx, const float4* __restrict__ pos4,
                       const uint32_t* __restrict__ start, LawF32 L, const PairF* __restrict__ tab,
                       long long* __restrict__ F, size_t fstride, unsigned long long* __restrict__ vacc,
                       unsigned long long* __restrict__ npairs, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) float4 s_pos[];
    __shared__ PairF s_tab[kMaxKinds * kMaxKinds];
    __shared__ Stage<kRSlots> S;
    __shared__ uint32_t s_list[kLCap][kRThreads];
    __shared__ uint32_t s_home[kRRunMax + 1];  // prefix of home atoms per own-row slot
    __shared__ unsigned long long s_red[kRThreads / 32][2];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t bx = blockIdx.x % nbx, yz = blockIdx.x / nbx;
    const uint32_t cy = yz % g.n[1], cz = yz / g.n[1];
    const int x0 = (int)bx * run;
    for (int t = tid; t < L.nkinds * L.nkinds; t += kRThreads) s_tab[t] = tab[t];
    if (!stage_rows<kRSlots>(S, s_pos, kRStageCap, g, run, x0, cy, cz, pos4, start, err)) return;
    const bool staged = S.staged != 0;
    const float4* P = staged ? (const float4*)s_pos : pos4;
    const int nh = x0 + run <= (int)g.n[0] ? run : (int)g.n[0] - x0;  // home cells of this block
    if (tid == 0) {
        uint32_t acc = 0;
        for (int s = 0; s < nh; ++s) {
            s_home[s] = acc;
            acc += S.c[0][s];
        }
        s_home[nh] = acc;
    }
    __syncthreads();
    const uint32_t nhome = s_home[nh];
    const uint32_t hbase_s = staged ? S.s[0][0] : S.g[0][0];  // home atoms are contiguous
    const uint32_t hbase_g = S.g[0][0];
    const int nk = L.nkinds;
    long long vq = 0;
    unsigned long long pcount = 0;

    for (uint32_t a0 = 0; a0 < nhome; a0 += kRThreads) {
        const uint32_t a = a0 + tid;
        const bool act = a < nhome;
        int hs = 0;
        while (hs + 1 < nh && s_home[hs + 1] <= a) ++hs;
        const uint32_t ii = hbase_s + a;  // index of i in P
        float4 pi = act ? P[ii] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int ki = __float_as_int(pi.w);
        long long fx = 0, fy = 0, fz = 0;
        int cnt = 0;

        auto flush = [&]() {
            int m = __reduce_max_sync(0xffffffffu, cnt);
            for (int k = 0; k < m; ++k) {
                if (k < cnt) {
                    uint32_t e = s_list[k][tid];
                    int t = (int)(e >> 27);
                    uint32_t jidx = e & 0x07FFFFFFu;
                    int r, ds, ddx;
                    tile_geom(t, r, ds, ddx);
                    int slot = hs + ds;
                    float4 pj = P[jidx];
                    float dx = delta1(pi.x, pj.x, -(float)ddx * g.cellf[0]);
                    float dy = delta1(pi.y, pj.y, -(float)row_dy(r) * g.cellf[1]);
                    float dz = delta1(pi.z, pj.z, -(float)row_dz(r) * g.cellf[2]);
                    float d2 = dist2(dx, dy, dz);
                    float fs, v;
                    pair_f32(L, s_tab[ki * nk + __float_as_int(pj.w)], d2, fs, v);
                    long long qx, qy, qz;
                quant3(fmul(dx, fs), fmul(dy, fs), fmul(dz, fs), qx, qy, qz, err);
                    fx += qx;
                    fy += qy;
                    fz += qz;
                    uint32_t gj = S.g[r][slot] + (jidx - (staged ? S.s[r][slot] : S.g[r][slot]));
                    atomicAdd((unsigned long long*)&F[gj], (unsigned long long)(-qx));
                    atomicAdd((unsigned long long*)&F[fstride + gj], (unsigned long long)(-qy));
                    atomicAdd((unsigned long long*)&F[2 * fstride + gj], (unsigned long long)(-qz));
                    vq += quant(v, err);
                }
            }
            cnt = 0;
        };

        for (int t = 0; t < kTiles; ++t) {
            int r, ds, ddx;
            tile_geom(t, r, ds, ddx);
            const int slot = hs + ds;
            uint32_t lo = staged ? S.s[r][slot] : S.g[r][slot];
            uint32_t hi = lo + S.c[r][slot];
            if (t == 0) lo = ii + 1;
            if (!act) hi = lo;
            const float sx = -(float)ddx * g.cellf[0], sy = -(float)row_dy(r) * g.cellf[1],
                        sz = -(float)row_dz(r) * g.cellf[2];
            const int mine = (int)(hi > lo ? hi - lo : 0u);
            const int most = __reduce_max_sync(0xffffffffu, mine);
            for (int c0 = 0; c0 < most; c0 += kLStep) {
                if (__any_sync(0xffffffffu, cnt > kLCap - kLStep)) flush();
                int c1 = mine < c0 + kLStep ? mine : c0 + kLStep;
                for (int c = c0; c < c1; ++c) {
                    uint32_t j = lo + (uint32_t)c;
                    float4 pj = P[j];
                    float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
                    float d2 = dist2(dx, dy, dz);
                    if (d2 < L.rc2 && d2 > 0.f) {
                        s_list[cnt][tid] = ((uint32_t)t << 27) | j;
                        ++cnt;
                        ++pcount;
                    }
                }
            }
        }
        flush();
        if (act) {
            if (fx) atomicAdd((unsigned long long*)&F[hbase_g + a], (unsigned long long)fx);
            if (fy) atomicAdd((unsigned long long*)&F[fstride + hbase_g + a], (unsigned long long)fy);
            if (fz) atomicAdd((unsigned long long*)&F[2 * fstride + hbase_g + a], (unsigned long long)fz);
        }
    }
    unsigned long long u = (unsigned long long)vq;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u += __shfl_down_sync(0xffffffffu, u, o);
        pcount += __shfl_down_sync(0xffffffffu, pcount, o);
    }
    if (lane == 0) {
        s_red[w][0] = u;
        s_red[w][1] = pcount;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long s = 0, p = 0;
        for (int k = 0; k < kRThreads / 32; ++k) {
            s += s_red[k][0];
            p += s_red[k][1];
        }
        if (s) atomicAdd(vacc, s);
        if (p) atomicAdd(npairs, p);
    }
}

// ------------------------------------------------------------------ variant 4
// A thread per atom over the whole sorted array (like k_force_mixed), the
// reference's canonical half shell, L1-cached loads, and the per-thread
// candidate list of variant 3 so the pair law runs outside the filter loop.

constexpr int kLThreads = 128;
constexpr int kL4Cap = 32;
constexpr int kL4Step = 16;

__global__ void __launch_bounds__(kLThreads, 8)
    k_force_mixed_lists(GridGeom g, const float4* __restrict__ pos4, const uint32_t* __restrict__ key,
                        const uint32_t* __restrict__ start, uint32_t n, LawF32 L, const PairF* __restrict__ tab,
                        long long* __restrict__ F, size_t fstride, unsigned long long* __restrict__ vacc,
                        unsigned long long* __restrict__ npairs, uint32_t* __restrict__ err) {
    __shared__ PairF s_tab[kMaxKinds * kMaxKinds];
    __shared__ float s_shift[kTiles][3];
    __shared__ uint32_t s_list[kL4Cap][kLThreads];
    __shared__ unsigned long long s_red[kLThreads / 32][2];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int t = tid; t < L.nkinds * L.nkinds; t += kLThreads) s_tab[t] = tab[t];
    if (tid < kTiles) {
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (tid > 0 && tid - 1 < g.nhalf) {
            sx = -(float)g.half[tid - 1][0] * g.cellf[0];
            sy = -(float)g.half[tid - 1][1] * g.cellf[1];
            sz = -(float)g.half[tid - 1][2] * g.cellf[2];
        }
        s_shift[tid][0] = sx;
        s_shift[tid][1] = sy;
        s_shift[tid][2] = sz;
    }
    __syncthreads();
    const uint32_t i = blockIdx.x * kLThreads + tid;
    const bool act = i < n;
    float4 pi = act ? __ldg(pos4 + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    const int ki = __float_as_int(pi.w);
    uint32_t cx = 0, cy = 0, cz = 0, c = 0;
    if (act) {
        c = key[i];
        decode(g, c, cx, cy, cz);
    }
    const int nk = L.nkinds;
    long long fx = 0, fy = 0, fz = 0, vq = 0;
    unsigned long long pcount = 0;
    int cnt = 0;

    auto flush = [&]() {
        int m = __reduce_max_sync(0xffffffffu, cnt);
        for (int k = 0; k < m; ++k) {
            if (k < cnt) {
                uint32_t e = s_list[k][tid];
                int t = (int)(e >> 27);
                uint32_t j = e & 0x07FFFFFFu;
                float4 pj = __ldg(pos4 + j);
                float dx = delta1(pi.x, pj.x, s_shift[t][0]), dy = delta1(pi.y, pj.y, s_shift[t][1]),
                      dz = delta1(pi.z, pj.z, s_shift[t][2]);
                if (g.minimg_mask) {
                    if (g.minimg_mask & 1) dx = fsub(dx, fmul(g.Lf[0], rintf(fmul(dx, g.invLf[0]))));
                    if (g.minimg_mask & 2) dy = fsub(dy, fmul(g.Lf[1], rintf(fmul(dy, g.invLf[1]))));
                    if (g.minimg_mask & 4) dz = fsub(dz, fmul(g.Lf[2], rintf(fmul(dz, g.invLf[2]))));
                }
                float d2 = dist2(dx, dy, dz);
                float fs, v;
                pair_f32(L, s_tab[ki * nk + __float_as_int(pj.w)], d2, fs, v);
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
        cnt = 0;
    };

    for (int t = 0; t <= g.nhalf; ++t) {
        uint32_t lo = 0, hi = 0;
        if (act) {
            if (t == 0) {
                lo = i + 1;
                hi = start[c + 1];
            } else {
                uint32_t B = encode(g, wrap_add(cx, g.half[t - 1][0], g.n[0]), wrap_add(cy, g.half[t - 1][1], g.n[1]),
                                    wrap_add(cz, g.half[t - 1][2], g.n[2]));
                lo = start[B];
                hi = start[B + 1];
            }
        }
        const float sx = s_shift[t][0], sy = s_shift[t][1], sz = s_shift[t][2];
        const int mine = (int)(hi > lo ? hi - lo : 0u);
        const int most = __reduce_max_sync(0xffffffffu, mine);
        for (int c0 = 0; c0 < most; c0 += kL4Step) {
            if (__any_sync(0xffffffffu, cnt > kL4Cap - kL4Step)) flush();
            const int c1 = mine < c0 + kL4Step ? mine : c0 + kL4Step;
            for (int q = c0; q < c1; ++q) {
                const uint32_t j = lo + (uint32_t)q;
                float4 pj = __ldg(pos4 + j);
                float dx = delta1(pi.x, pj.x, sx), dy = delta1(pi.y, pj.y, sy), dz = delta1(pi.z, pj.z, sz);
                if (g.minimg_mask) {
                    if (g.minimg_mask & 1) dx = fsub(dx, fmul(g.Lf[0], rintf(fmul(dx, g.invLf[0]))));
                    if (g.minimg_mask & 2) dy = fsub(dy, fmul(g.Lf[1], rintf(fmul(dy, g.invLf[1]))));
                    if (g.minimg_mask & 4) dz = fsub(dz, fmul(g.Lf[2], rintf(fmul(dz, g.invLf[2]))));
                }
                float d2 = dist2(dx, dy, dz);
                if (d2 < L.rc2 && d2 > 0.f) {
                    s_list[cnt][tid] = ((uint32_t)t << 27) | j;
                    ++cnt;
                    ++pcount;
                }
            }
        }
    }
    flush();
    if (act) {
        if (fx) atomicAdd((unsigned long long*)&F[i], (unsigned long long)fx);
        if (fy) atomicAdd((unsigned long long*)&F[fstride + i], (unsigned long long)fy);
        if (fz) atomicAdd((unsigned long long*)&F[2 * fstride + i], (unsigned long long)fz);
    }
    unsigned long long u = (unsigned long long)vq;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u += __shfl_down_sync(0xffffffffu, u, o);
        pcount += __shfl_down_sync(0xffffffffu, pcount, o);
    }
    if (lane == 0) {
        s_red[w][0] = u;
        s_red[w][1] = pcount;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long s = 0, p = 0;
        for (int k = 0; k < kLThreads / 32; ++k) {
            s += s_red[k][0];
            p += s_red[k][1];
        }
        if (s) atomicAdd(vacc, s);
        if (p) atomicAdd(npairs, p);
    }
}

}  // namespace

void launch_force_mixed_lists(gx_handle* h, const GridGeom& g, const float4* pos4, const uint32_t* key,
                              const uint32_t* start, uint32_t n, const LawF32& L, const PairF* tab, long long* F,
                              size_t fstride, unsigned long long* vacc, unsigned long long* npairs, uint32_t* err) {
    k_force_mixed_lists<<<(n + kLThreads - 1) / kLThreads, kLThreads, 0, h->stream>>>(
        g, pos4, key, start, n, L, tab, F, fstride, vacc, npairs, err);
    ++h->launches;
}

void launch_force_mixed_tiled(gx_handle* h, const GridGeom& g, const float4* pos4, const uint32_t* start,
                              const LawF32& L, const PairF* tab, long long* F, size_t fstride,
                              unsigned long long* vacc, unsigned long long* npairs, uint32_t* err) {
    static bool attr_set[64][2] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    bool rows = h->kernel_variant == 3;
    const size_t dyn = (rows ? kRStageCap : kTStageCap) * sizeof(float4);
    if (dev < 0 || dev >= 64 || !attr_set[dev][rows]) {
        if (rows) cudaFuncSetAttribute(k_force_mixed_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        else cudaFuncSetAttribute(k_force_mixed_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        if (dev >= 0 && dev < 64) attr_set[dev][rows] = true;
    }
    int runmax = rows ? kRRunMax : kTRunMax;
    int nx = (int)g.n[0];
    int run = nx - 2 < runmax ? nx - 2 : runmax;
    int nbx = (nx + run - 1) / run;
    run = (nx + nbx - 1) / nbx;  // balance the runs of a row
    unsigned blocks = (unsigned)nbx * g.n[1] * g.n[2];
    if (rows)
        k_force_mixed_rows<<<blocks, kRThreads, dyn, h->stream>>>(g, run, nbx, pos4, start, L, tab, F, fstride, vacc,
                                                                 npairs, err);
    else
        k_force_mixed_tiled<<<blocks, kTThreads, dyn, h->stream>>>(g, run, nbx, pos4, start, L, tab, F, fstride,
                                                                  vacc, npairs, err);
    ++h->launches;
}

}  // namespace gx
