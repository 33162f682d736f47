// gx_noalloc.cu -- g(r) for callers that cannot allocate device memory.
//
// gx_radial_distribution builds its grid in buffers the handle allocates.
// Some callers cannot do that: code that runs under a fixed device-memory
// budget, or code that must not call cudaMalloc/cudaFree because those
// calls can synchronise the whole device while other work is in flight.
// gx_radial_distribution_noalloc serves them.  It takes host positions and
// returns host counts, and keeps every intermediate (the sample, its cell
// list and the bin counters) in one file-scope __device__ array of fixed
// size.  It calls no cudaMalloc, cudaFree or other allocating routine.
//
// Limits (kept modest so every GPU that loads the library can hold the
// array until exit, ~1.9 MB):
//   * at most 8192 sampled atoms -- always true, because the reference's
//     subsample (src/analysis/mod.rs:32-46) never keeps more than 8192;
//   * at most 65536 cells in the g(r) grid (floor(L/r_max) per axis);
//   * at most 65536 bins (the reference's own clamp, mod.rs:93).
// A larger grid is rejected with GX_ERR_CAPACITY before any GPU work.
//
// The array is shared by every call on a device and keeps the last call's
// contents; the call clears what must start at zero.  Calls that overlap on
// the GPU (two host threads at once on one device) race on it.  The first
// call on a device looks up the array's device address with
// cudaGetSymbolAddress while that device is current; make that first call
// before any stream capture begins.  The address is kept for the life of the
// process (a device reset after the first call is not supported).  Each call
// runs on the legacy default stream and waits for it.
#include <cmath>
#include <cstring>

#include "gx_internal.cuh"

namespace {

using namespace gx;

constexpr uint32_t kNaAtoms = 8192;
constexpr uint32_t kNaCells = 65536;
constexpr uint32_t kNaBins = 65536;
constexpr int kNaScanThreads = 1024;
constexpr int kNaScanItems = 4;
constexpr uint32_t kNaTile = kNaScanThreads * kNaScanItems;  // 65537 counters -> 17 tiles

// Byte offsets of the regions carved out of the scratch array.
constexpr size_t kOffAos = 0;                                      // 3 f64 per sampled atom
constexpr size_t kOffX = kOffAos + 3 * 8 * kNaAtoms;               // sorted x, y, z
constexpr size_t kOffKey = kOffX + 3 * 8 * kNaAtoms;               // key per sampled atom
constexpr size_t kOffSKey = kOffKey + 4 * kNaAtoms;                // key, sorted
constexpr size_t kOffPerm = kOffSKey + 4 * kNaAtoms;               // sample index per slot, unordered in a cell
constexpr size_t kOffOrder = kOffPerm + 4 * kNaAtoms;              // the same, ascending in each cell
constexpr size_t kOffCount = kOffOrder + 4 * kNaAtoms;             // kNaCells + 1
constexpr size_t kOffStart = kOffCount + 4 * (kNaCells + 64);      // kNaCells + 1
constexpr size_t kOffFill = kOffStart + 4 * (kNaCells + 64);       // kNaCells
constexpr size_t kOffSums = kOffFill + 4 * (kNaCells + 64);        // scan tile sums
constexpr size_t kOffErr = kOffSums + 4 * 64;
constexpr size_t kOffBins = kOffErr + 256;                          // u64 per bin
constexpr size_t kScratchBytes = kOffBins + 8 * (size_t)kNaBins;

static __device__ __align__(256) unsigned char g_gr_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};

struct NaView {
    double* aos;
    double *x, *y, *z;
    uint32_t *key, *skey, *perm, *order, *count, *start, *fill, *sums, *err;
    unsigned long long* bins;
};

NaView view(unsigned char* s) {
    NaView v;
    v.aos = (double*)(s + kOffAos);
    v.x = (double*)(s + kOffX);
    v.y = v.x + kNaAtoms;
    v.z = v.y + kNaAtoms;
    v.key = (uint32_t*)(s + kOffKey);
    v.skey = (uint32_t*)(s + kOffSKey);
    v.perm = (uint32_t*)(s + kOffPerm);
    v.order = (uint32_t*)(s + kOffOrder);
    v.count = (uint32_t*)(s + kOffCount);
    v.start = (uint32_t*)(s + kOffStart);
    v.fill = (uint32_t*)(s + kOffFill);
    v.sums = (uint32_t*)(s + kOffSums);
    v.err = (uint32_t*)(s + kOffErr);
    v.bins = (unsigned long long*)(s + kOffBins);
    return v;
}

__global__ void na_keys(GridGeom g, NaView v, uint32_t m) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    uint32_t c = cell_of(g, v.aos[3 * q], v.aos[3 * q + 1], v.aos[3 * q + 2]);
    v.key[q] = c;
    atomicAdd(&v.count[c], 1u);
}

__global__ void __launch_bounds__(kNaScanThreads) na_scan(const uint32_t* in, uint32_t* out, uint32_t n,
                                                          uint32_t* sums) {
    __shared__ uint32_t warp_tot[kNaScanThreads / 32];
    uint32_t base = blockIdx.x * kNaTile + threadIdx.x * kNaScanItems;
    uint32_t val[kNaScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kNaScanItems; ++k) {
        val[k] = (base + k < n) ? in[base + k] : 0u;
        local += val[k];
    }
    uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += t;
    }
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = warp_tot[lane];
        uint32_t winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= (uint32_t)o) winc += t;
        }
        warp_tot[lane] = winc - w;
        if (lane == 31 && sums) sums[blockIdx.x] = winc;
    }
    __syncthreads();
    uint32_t run = warp_tot[wid] + inc - local;
#pragma unroll
    for (int k = 0; k < kNaScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += val[k];
    }
}

__global__ void na_scan_add(uint32_t* out, uint32_t n, const uint32_t* sums) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kNaTile];
}

__global__ void na_scatter(NaView v, uint32_t m) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    uint32_t c = v.key[q];
    v.perm[v.start[c] + atomicAdd(&v.fill[c], 1u)] = q;
}

// Makes the scatter deterministic: sample q goes to start[c] + (the number of
// samples of its cell with a smaller index), so each cell lists its samples
// in ascending order.  One thread per sample reads its cell's segment, which
// keeps a cell that holds most of the sample (a droplet) parallel: the work
// is the sum of the squared cell sizes spread over all samples.
__global__ void na_rank(NaView v, uint32_t m) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    uint32_t c = v.key[q];
    uint32_t lo = v.start[c], hi = v.start[c + 1], r = 0;
    for (uint32_t b = lo; b < hi; ++b) r += v.perm[b] < q ? 1u : 0u;
    v.order[lo + r] = q;
}

__global__ void na_gather(NaView v, uint32_t m) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    uint32_t q = v.order[p];
    v.x[p] = v.aos[3 * q];
    v.y[p] = v.aos[3 * q + 1];
    v.z[p] = v.aos[3 * q + 2];
    v.skey[p] = v.key[q];
}

// Canonical half shell with the exact check_pair test (grid.rs:201-225),
// then counts[(d / dr) as usize] += 1 for d < r_max (analysis/mod.rs:109-117).
__global__ void na_pairs(GridGeom g, NaView v, uint32_t m, double cd2, double r_max, double dr, uint32_t nbins) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t c = v.skey[i];
    uint32_t cx, cy, cz;
    decode(g, c, cx, cy, cz);
    double xi = v.x[i], yi = v.y[i], zi = v.z[i];
    for (int k = -1; k < g.nhalf; ++k) {
        uint32_t B, lo;
        if (k < 0) {
            B = c;
            lo = i + 1;
        } else {
            B = encode(g, wrap_add(cx, g.half[k][0], g.n[0]), wrap_add(cy, g.half[k][1], g.n[1]),
                       wrap_add(cz, g.half[k][2], g.n[2]));
            lo = v.start[B];
        }
        uint32_t hi = v.start[B + 1];
        for (uint32_t j = lo; j < hi; ++j) {
            double dx = min_image1(xsub(xi, v.x[j]), g.L[0]);
            double dy = min_image1(xsub(yi, v.y[j]), g.L[1]);
            double dz = min_image1(xsub(zi, v.z[j]), g.L[2]);
            double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
            if (d2 >= cd2) continue;
            double d = xsqrt(d2);
            if (d <= kEpsF64 || d >= r_max) continue;
            double f = xdiv(d, dr);
            uint32_t bi = f >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)f;
            if (bi >= nbins) {
                atomicOr(v.err, kErrBinRange);
                continue;
            }
            atomicAdd(&v.bins[bi], 1ull);
        }
    }
}

inline unsigned nb(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

extern "C" int gx_radial_distribution_noalloc(size_t n, const double* pos, const double box[3], double r_max_in,
                                              size_t nbins_in, uint64_t* counts, double* bins, double* r_max_out,
                                              double* dr_out) {
    if (!box || !counts || (n && !pos)) return GX_ERR_ARG;
    size_t nbins = nbins_in < 1 ? 1 : (nbins_in > kNaBins ? kNaBins : nbins_in);  // analysis/mod.rs:93
    double half_min = std::fmin(std::fmin(box[0], box[1]), box[2]) * 0.5;
    double r_max = std::fmin(std::fmax(r_max_in, 1e-9), half_min);
    double dr = r_max / (double)nbins;
    double vol = box[0] * box[1] * box[2];
    int ok = 0;
    GridGeom g = make_grid(box, r_max, &ok);
    if (!ok) return GX_ERR_ARG;
    if (g.ncell > kNaCells) return GX_ERR_CAPACITY;  // limit stated in the header
    // The reference's evenly spaced subsample (analysis/mod.rs:32-46): never more than 8192.
    size_t step = 1, m = n;
    if (n > 8192) {
        step = n / 8192 + 1;
        m = n / step;
    }
    // A non-sticky error an earlier, unrelated CUDA call left on this thread
    // is dropped here, so that the checks below see only this call's errors.
    cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GX_ERR_CUDA;
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_gr_scratch);
        if (e != cudaSuccess || !p) return GX_ERR_CUDA;
        g_scratch_addr[dev] = (unsigned char*)p;
    }
    NaView v = view(g_scratch_addr[dev]);
    cudaStream_t s = 0;
    uint32_t um = (uint32_t)m, nc = g.ncell;
    // Every enqueue is checked; after a failed one the call waits for what it
    // already queued on the stream before it returns.
    bool bad = false;
    auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess) bad = true;
        return !bad;
    };
    auto fail = [&]() {
        cudaStreamSynchronize(s);
        cudaGetLastError();
        return GX_ERR_CUDA;
    };
    chk(cudaMemsetAsync(v.count, 0, 4 * ((size_t)nc + 1), s)) && chk(cudaMemsetAsync(v.fill, 0, 4 * (size_t)nc, s)) &&
        chk(cudaMemsetAsync(v.err, 0, 4, s)) && chk(cudaMemsetAsync(v.bins, 0, 8 * nbins, s));
    if (bad) return fail();
    if (m) {
        // every step-th AoS record of the host array into the scratch sample
        if (!chk(cudaMemcpy2DAsync(v.aos, 24, pos, 24 * step, 24, m, cudaMemcpyHostToDevice, s))) return fail();
        na_keys<<<nb(m, 256), 256, 0, s>>>(g, v, um);
        if (!chk(cudaGetLastError())) return fail();
    }
    uint32_t nscan = nc + 1;
    unsigned tiles = (nscan + kNaTile - 1) / kNaTile;
    na_scan<<<tiles, kNaScanThreads, 0, s>>>(v.count, v.start, nscan, tiles > 1 ? v.sums : nullptr);
    if (tiles > 1) {
        na_scan<<<1, kNaScanThreads, 0, s>>>(v.sums, v.sums, tiles, nullptr);
        na_scan_add<<<nb(nscan, 256), 256, 0, s>>>(v.start, nscan, v.sums);
    }
    if (!chk(cudaGetLastError())) return fail();
    if (m) {
        na_scatter<<<nb(m, 256), 256, 0, s>>>(v, um);
        na_rank<<<nb(m, 128), 128, 0, s>>>(v, um);
        na_gather<<<nb(m, 256), 256, 0, s>>>(v, um);
        na_pairs<<<nb(m, 128), 128, 0, s>>>(g, v, um, r_max * r_max, r_max, dr, (uint32_t)nbins);
        if (!chk(cudaGetLastError())) return fail();
    }
    uint32_t err = 0;
    chk(cudaMemcpyAsync(counts, v.bins, 8 * nbins, cudaMemcpyDeviceToHost, s)) &&
        chk(cudaMemcpyAsync(&err, v.err, 4, cudaMemcpyDeviceToHost, s));
    if (bad) return fail();
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return GX_ERR_CUDA;
    if (r_max_out) *r_max_out = r_max;
    if (dr_out) *dr_out = dr;
    if (bins) {  // ideal-gas normalisation, analysis/mod.rs:119-132
        for (size_t i = 0; i < nbins; ++i) bins[i] = 0.0;
        if (m >= 2) {
            const double pi = 3.141592653589793;
            for (size_t i = 0; i < nbins; ++i) {
                double r_lo = (double)i * dr;
                double r_hi = r_lo + dr;
                double shell = 4.0 / 3.0 * pi * (r_hi * r_hi * r_hi - r_lo * r_lo * r_lo);
                double expected = (double)(m * (m - 1)) * 0.5 * shell / vol;
                bins[i] = (double)counts[i] / std::fmax(expected, 2.2250738585072014e-308);
            }
        }
    }
    return (err & kErrBinRange) ? GX_ERR_CAPACITY : GX_OK;
}
