// gx_snapshot.cu -- the world section of Universe::save, encoded on the device.
//
// save_universe (src/serialization/mod.rs:85-104) writes
// bincode::serialize(&Snapshot { format, config, state, world }) where world
// is a Vec<EntitySnapshot> (mod.rs:38-56), one record per entity with every
// component as an Option.  bincode 1 with its default options encodes
// integers and floats little-endian at their full width, a sequence as a u64
// length followed by its items, an Option as a u8 tag (0 None, 1 Some)
// followed by the value, a unit enum variant as its u32 declaration index,
// and newtype and plain structs as their fields in order.  Every atom the
// reference spawns carries all seven components (src/universe/mod.rs:247-273),
// so one record is
//
//   index u32, generation u32,
//   1 + position (3 f64), 1 + velocity (3 f64), 1 + mass f64, 1 + charge f64,
//   1 + atom_type u32 (H, He, C, N, O, Na, Si, P, S, Fe = 0..9),
//   1 + bonds: u64 count + count x EntityId (index u32, generation u32),
//   1 + acceleration (3 f64)
//
// = 115 + 8 k bytes for an atom with k bonds.  The record of ECS slot s
// starts at 8 + 115 s + 8 (bonds of the slots before s), so one scan of the
// per-slot bond counts places every record.  The partners of a slot are
// listed in ascending slot order (the reference lists them in hash-map
// order, src/systems/bonds.rs:100-121, which no byte comparison can pin; any
// order loads the same world).  The configuration, clock, RNG and statistics
// that precede the world in the file stay with the host code that owns them.
#include <cub/cub.cuh>

#include <cstring>

#include "gx_internal.cuh"

namespace gx {

namespace {

constexpr int kSnapThreads = 256;
constexpr size_t kSnapFixed = 115;  // bytes of a record without its bonds

__global__ void k_snap_degree(const uint32_t* __restrict__ bonds, uint32_t nb, uint32_t n,
                              unsigned long long* __restrict__ deg, uint32_t* __restrict__ err) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const uint32_t a = bonds[2 * k], b = bonds[2 * k + 1];
    if (a >= n || b >= n) {
        atomicOr(err, kErrCapacity);
        return;
    }
    atomicAdd(&deg[a], 1ull);
    atomicAdd(&deg[b], 1ull);
}

__global__ void k_snap_fill(const uint32_t* __restrict__ bonds, uint32_t nb, uint32_t n,
                            const unsigned long long* __restrict__ off, uint32_t* __restrict__ fill,
                            uint32_t* __restrict__ adj) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const uint32_t a = bonds[2 * k], b = bonds[2 * k + 1];
    if (a >= n || b >= n) return;
    adj[off[a] + atomicAdd(&fill[a], 1u)] = b;
    adj[off[b] + atomicAdd(&fill[b], 1u)] = a;
}

// Each slot's partners in ascending order (rows are short: a few bonds).
__global__ void k_snap_sort_rows(const unsigned long long* __restrict__ off, uint32_t n, uint32_t* __restrict__ adj) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const unsigned long long lo = off[s], hi = off[s + 1];
    for (unsigned long long a = lo + 1; a < hi; ++a) {
        const uint32_t v = adj[a];
        unsigned long long b = a;
        while (b > lo && adj[b - 1] > v) {
            adj[b] = adj[b - 1];
            --b;
        }
        adj[b] = v;
    }
}

__device__ __forceinline__ unsigned char* put_u32(unsigned char* p, uint32_t v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = (unsigned char)(v >> (8 * k));
    return p + 4;
}
__device__ __forceinline__ unsigned char* put_u64(unsigned char* p, unsigned long long v) {
#pragma unroll
    for (int k = 0; k < 8; ++k) p[k] = (unsigned char)(v >> (8 * k));
    return p + 8;
}
__device__ __forceinline__ unsigned char* put_f64(unsigned char* p, double v) {
    return put_u64(p, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ unsigned char* put_vec3(unsigned char* p, double x, double y, double z) {
    *p++ = 1;  // Some
    p = put_f64(p, x);
    p = put_f64(p, y);
    return put_f64(p, z);
}

// One record per ECS slot at 8 + 115 s + 8 off[s]; the state is read through
// pos_of_slot (the device keeps it in cell order).
__global__ void __launch_bounds__(kSnapThreads) k_snap_write(StateBuf b, const uint32_t* __restrict__ pos_of_slot,
                                                             const uint32_t* __restrict__ entity,
                                                             const uint32_t* __restrict__ gen, uint32_t n,
                                                             const unsigned long long* __restrict__ off,
                                                             const uint32_t* __restrict__ adj,
                                                             unsigned char* __restrict__ out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) put_u64(out, (unsigned long long)n);  // Vec<EntitySnapshot> length
    if (s >= n) return;
    const uint32_t i = pos_of_slot[s];
    const unsigned long long lo = off[s], hi = off[s + 1];
    unsigned char* p = out + 8 + kSnapFixed * (unsigned long long)s + 8ull * lo;
    p = put_u32(p, entity ? entity[s] : s);
    p = put_u32(p, gen ? gen[s] : 0u);
    p = put_vec3(p, b.x[i], b.y[i], b.z[i]);
    p = put_vec3(p, b.vx[i], b.vy[i], b.vz[i]);
    *p++ = 1;
    p = put_f64(p, b.mass[i]);
    *p++ = 1;
    p = put_f64(p, b.charge[i]);
    *p++ = 1;
    p = put_u32(p, (uint32_t)b.elem[i]);
    *p++ = 1;
    p = put_u64(p, hi - lo);
    for (unsigned long long k = lo; k < hi; ++k) {
        const uint32_t q = adj[k];
        p = put_u32(p, entity ? entity[q] : q);
        p = put_u32(p, gen ? gen[q] : 0u);
    }
    put_vec3(p, b.ax[i], b.ay[i], b.az[i]);
}

struct SnapState {
    unsigned long long* deg = nullptr;  // n + 1: bonds per slot
    unsigned long long* off = nullptr;  // n + 1: exclusive scan of deg
    uint32_t* fill = nullptr;           // n: placement counters
    uint32_t* gen = nullptr;            // n
    uint32_t* adj = nullptr;            // 2 * nbonds partner slots
    uint32_t* err = nullptr;
    void* temp = nullptr;
    size_t cap = 0, adj_cap = 0, temp_bytes = 0;
    unsigned char* bytes = nullptr;
    size_t bytes_cap = 0;
};

inline unsigned nblk(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

SnapState& snap_of(gx_handle* h) {
    if (!h->snap) h->snap = new SnapState();
    return *static_cast<SnapState*>(h->snap);
}

}  // namespace

void snapshot_free(gx_handle* h) {
    if (!h->snap) return;
    SnapState* s = static_cast<SnapState*>(h->snap);
    cudaFree(s->deg);
    cudaFree(s->off);
    cudaFree(s->fill);
    cudaFree(s->gen);
    cudaFree(s->adj);
    cudaFree(s->err);
    cudaFree(s->temp);
    cudaFree(s->bytes);
    delete s;
    h->snap = nullptr;
}

}  // namespace gx

using namespace gx;

extern "C" int gx_snapshot_world(gx_handle* h, const uint32_t* generation, uint8_t* out, size_t cap, size_t* len) {
    if (!h || !len) return GX_ERR_ARG;
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    int rc = settle_step_errors(h);
    if (rc) return rc;
    rc = commit_pending_lambda(h);  // v as the host would read it
    if (rc) return rc;
    const uint32_t n = (uint32_t)h->n;
    const size_t nb = h->nbonds;
    const size_t total = 8 + kSnapFixed * (size_t)n + 16 * nb;
    *len = total;
    if (!out || cap < total) return set_err(h, GX_ERR_CAPACITY, "gx_snapshot_world: out holds fewer than *len bytes");
    if (!n) {
        std::memset(out, 0, 8);
        return GX_OK;
    }
    SnapState& S = snap_of(h);
    if (S.cap < (size_t)n + 1) {
        cudaFree(S.deg);
        cudaFree(S.off);
        cudaFree(S.fill);
        cudaFree(S.gen);
        cudaFree(S.temp);
        S.deg = S.off = nullptr;
        S.fill = S.gen = nullptr;
        S.temp = nullptr;
        S.cap = 0;
        const size_t c = (size_t)n + 1;
        GX_CUDA(h, cudaMalloc(&S.deg, c * sizeof(unsigned long long)));
        GX_CUDA(h, cudaMalloc(&S.off, c * sizeof(unsigned long long)));
        GX_CUDA(h, cudaMalloc(&S.fill, c * sizeof(uint32_t)));
        GX_CUDA(h, cudaMalloc(&S.gen, c * sizeof(uint32_t)));
        if (!S.err) GX_CUDA(h, cudaMalloc(&S.err, sizeof(uint32_t)));
        size_t tb = 0;
        GX_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, tb, S.deg, S.off, (int)c, h->stream));
        GX_CUDA(h, cudaMalloc(&S.temp, tb));
        S.temp_bytes = tb;
        S.cap = c;
    }
    if (2 * nb > S.adj_cap) {
        cudaFree(S.adj);
        S.adj = nullptr;
        S.adj_cap = 0;
        GX_CUDA(h, cudaMalloc(&S.adj, 2 * nb * sizeof(uint32_t)));
        S.adj_cap = 2 * nb;
    }
    if (total > S.bytes_cap) {
        cudaFree(S.bytes);
        S.bytes = nullptr;
        S.bytes_cap = 0;
        GX_CUDA(h, cudaMalloc(&S.bytes, total));
        S.bytes_cap = total;
    }
    if (generation)
        GX_CUDA(h, cudaMemcpyAsync(S.gen, generation, (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
    GX_CUDA(h, cudaMemsetAsync(S.deg, 0, ((size_t)n + 1) * sizeof(unsigned long long), h->stream));
    GX_CUDA(h, cudaMemsetAsync(S.err, 0, sizeof(uint32_t), h->stream));
    prof_begin(h, "snapshot");
    if (nb) GX_LAUNCH(h, k_snap_degree, nblk(nb, kSnapThreads), kSnapThreads, h->bonds, (uint32_t)nb, n, S.deg, S.err);
    size_t tb = S.temp_bytes;
    GX_CUDA(h, cub::DeviceScan::ExclusiveSum(S.temp, tb, S.deg, S.off, (int)(n + 1), h->stream));
    if (nb) {
        GX_CUDA(h, cudaMemsetAsync(S.fill, 0, (size_t)n * sizeof(uint32_t), h->stream));
        GX_LAUNCH(h, k_snap_fill, nblk(nb, kSnapThreads), kSnapThreads, h->bonds, (uint32_t)nb, n, S.off, S.fill,
                  S.adj);
        GX_LAUNCH(h, k_snap_sort_rows, nblk(n, kSnapThreads), kSnapThreads, S.off, n, S.adj);
    }
    GX_LAUNCH(h, k_snap_write, nblk(n, kSnapThreads), kSnapThreads, h->buf[h->cur], h->pos_of_slot,
              h->has_entity ? h->entity : nullptr, generation ? S.gen : nullptr, n, S.off, S.adj, S.bytes);
    prof_end(h, "snapshot");
    uint32_t herr = 0;
    GX_CUDA(h, cudaMemcpyAsync(&herr, S.err, sizeof herr, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaMemcpyAsync(out, S.bytes, total, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    if (herr) return set_err(h, GX_ERR_STATE, "gx_snapshot_world: a bond names a slot beyond the atom count");
    return GX_OK;
}
