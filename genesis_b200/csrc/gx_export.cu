// XYZ position frames written on the device: export::write_frame
// (src/export/mod.rs:152-172).  The frame is the text
//
//   "{N}\nframe {tick}\n" then, per atom in slot order,
//   "{symbol} {x:.6} {y:.6} {z:.6}\n"
//
// with every coordinate the exact binary value of the double rounded to six
// decimals, ties to even, as Rust's `{:.6}` prints it: a leading '-' whenever
// the sign bit is set (-0.0 and values that round to zero included), "NaN"
// for NaN, "inf" / "-inf" for infinities.
//
// Two passes over the atoms, both one thread per slot:
//   k_xyz_measure  the byte length of each line, summed per block
//   [scan]         exclusive sum of the block lengths (CUB)
//   k_xyz_write    the lines again, a block scan gives each its offset; the
//                  block formats its lines into shared memory laid out at the
//                  output's 16-byte phase and stores them as aligned 16-byte
//                  words (bytes only at the two ragged ends)
// The text goes to a device buffer and from there in one copy to the
// caller's host buffer.  Integer and byte work only: HBM-bound, 25 bytes
// read per atom per pass plus the text written once.
//
// Exact decimal conversion: x = m 2^e with m < 2^53.  For e >= 0, x is an
// integer (< 2^100 here); otherwise n = round(m 10^6 2^e) comes from 128-bit
// shifts (m 10^6 < 2^73) with the remainder compared against one half, and
// the integer part is m >> -e plus a possible carry of the rounding: no
// division.  Digits come from 32-bit divisions by 10 whenever the integer
// part is below 2^32.  Magnitudes up to 2^100 are formatted; larger ones
// make the call fail with GX_ERR_UNSUPPORTED.
#include <cub/cub.cuh>

#include <cstdio>
#include <cstring>

#include "gx_internal.cuh"

namespace gx {
namespace {

constexpr int kXyzThreads = 256;
constexpr int kMaxBinExp = 100;  // |x| < 2^100 formatted
// symbol (2) + 3 x (sign, 31 integer digits, '.', 6 decimals) + 3 blanks + '\n'
constexpr int kXyzMaxLine = 2 + 3 * (1 + 31 + 1 + 6) + 3 + 1;
constexpr unsigned long long kE19 = 10000000000000000000ull;

__constant__ char kSymbol[kNElem][2] = {{'H', 0},   {'H', 'e'}, {'C', 0},   {'N', 0},   {'O', 0},
                                        {'N', 'a'}, {'S', 'i'}, {'P', 0},   {'S', 0},   {'F', 'e'}};

__constant__ unsigned long long kPow10[20] = {1ull,
                                              10ull,
                                              100ull,
                                              1000ull,
                                              10000ull,
                                              100000ull,
                                              1000000ull,
                                              10000000ull,
                                              100000000ull,
                                              1000000000ull,
                                              10000000000ull,
                                              100000000000ull,
                                              1000000000000ull,
                                              10000000000000ull,
                                              100000000000000ull,
                                              1000000000000000ull,
                                              10000000000000000ull,
                                              100000000000000000ull,
                                              1000000000000000000ull,
                                              10000000000000000000ull};

// Decimal digits of v (1 for 0): log10 from the bit length, corrected by
// one comparison with a power of ten.
__device__ __forceinline__ int ndig64(unsigned long long v) {
    const int t = ((64 - __clzll(v | 1ull)) * 1233) >> 12;  // <= 19
    const int d = t + 1 - (v < kPow10[t] ? 1 : 0);
    return d > 1 ? d : 1;
}

// |x| rounded to 6 decimals, ties to even: integer part ip and the six
// decimals frac, nd = the digits of ip.
struct Fixed6 {
    unsigned __int128 ip;
    unsigned frac;
    int nd;
    int neg;   // sign bit
    int kind;  // 0 finite, 1 NaN, 2 infinite, 3 out of range
};

__device__ __forceinline__ Fixed6 to_fixed6(double x) {
    Fixed6 r;
    r.ip = 0;
    r.frac = 0;
    r.nd = 1;
    r.kind = 0;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
    r.neg = (int)(bits >> 63);
    const int ex = (int)((bits >> 52) & 0x7ff);
    const unsigned long long fr = bits & ((1ull << 52) - 1);
    if (ex == 0x7ff) {
        r.kind = fr ? 1 : 2;
        return r;
    }
    if (ex >= 1023 + kMaxBinExp) {
        r.kind = 3;
        return r;
    }
    const unsigned long long m = ex ? (fr | (1ull << 52)) : fr;
    const int e = (ex ? ex : 1) - 1075;  // |x| = m 2^e
    if (e >= 0) {  // an integer: m 2^e < 2^100
        r.ip = (unsigned __int128)m << e;
        if ((r.ip >> 64) == 0) {
            r.nd = ndig64((unsigned long long)r.ip);
        } else {
            const unsigned long long hi = (unsigned long long)(r.ip / kE19);
            r.nd = ndig64(hi) + 19;
        }
        return r;
    }
    const int s = -e;
    if (s > 74) return r;  // m 10^6 < 2^73 <= half an ulp of 2^-s: rounds to 0
    // n = round(m 10^6 / 2^s); the integer part before rounding is m >> s
    // and n - (m >> s) 10^6 lies in [0, 10^6], 10^6 being a carry
    const unsigned __int128 p = (unsigned __int128)m * 1000000u;
    const unsigned __int128 q = p >> s;
    const unsigned __int128 rem = p - (q << s);
    const unsigned __int128 half = (unsigned __int128)1 << (s - 1);
    const unsigned __int128 n = q + ((rem > half || (rem == half && (q & 1))) ? 1 : 0);
    unsigned long long ip = s < 64 ? (m >> s) : 0ull;  // < 2^52
    unsigned f = (unsigned)(n - (unsigned __int128)ip * 1000000u);
    if (f >= 1000000u) {
        ++ip;
        f -= 1000000u;
    }
    r.ip = ip;
    r.frac = f;
    r.nd = ndig64(ip);
    return r;
}

__device__ __forceinline__ int fixed6_len(const Fixed6& f) {
    if (f.kind == 1) return 3;
    if (f.kind == 2) return 3 + f.neg;
    if (f.kind == 3) return 0;
    return f.neg + f.nd + 7;
}

// Writes the text of f at out (fixed6_len(f) bytes).
__device__ __forceinline__ char* fixed6_put(const Fixed6& f, char* out) {
    if (f.kind == 1) {
        out[0] = 'N';
        out[1] = 'a';
        out[2] = 'N';
        return out + 3;
    }
    if (f.neg) *out++ = '-';
    if (f.kind == 2) {
        out[0] = 'i';
        out[1] = 'n';
        out[2] = 'f';
        return out + 3;
    }
    char* p = out + f.nd;
    if ((f.ip >> 32) == 0) {  // every coordinate of a simulation box
        unsigned v = (unsigned)f.ip;
        do {
            const unsigned q = v / 10u;
            *--p = (char)('0' + (v - q * 10u));
            v = q;
        } while (v);
    } else {
        unsigned long long lo, hi = 0;
        if ((f.ip >> 64) == 0) {
            lo = (unsigned long long)f.ip;
        } else {
            hi = (unsigned long long)(f.ip / kE19);
            lo = (unsigned long long)(f.ip - (unsigned __int128)hi * kE19);
        }
        const int nlo = hi ? 19 : f.nd;
        for (int k = 0; k < nlo; ++k) {
            const unsigned long long q = lo / 10u;
            *--p = (char)('0' + (unsigned)(lo - q * 10u));
            lo = q;
        }
        while (hi) {
            const unsigned long long q = hi / 10u;
            *--p = (char)('0' + (unsigned)(hi - q * 10u));
            hi = q;
        }
    }
    out += f.nd;
    *out++ = '.';
    unsigned fr = f.frac;
    for (int k = 5; k >= 0; --k) {
        const unsigned q = fr / 10u;
        out[k] = (char)('0' + (fr - q * 10u));
        fr = q;
    }
    return out + 6;
}

struct Line {
    Fixed6 c[3];
    int elem;
    int len;
};

__device__ __forceinline__ Line load_line(const StateBuf& b, const uint32_t* __restrict__ pos_of_slot, uint32_t s,
                                          uint32_t* err) {
    Line L;
    const uint32_t i = pos_of_slot[s];
    L.c[0] = to_fixed6(b.x[i]);
    L.c[1] = to_fixed6(b.y[i]);
    L.c[2] = to_fixed6(b.z[i]);
    L.elem = b.elem[i];
    if (L.c[0].kind == 3 || L.c[1].kind == 3 || L.c[2].kind == 3 || L.elem >= kNElem) atomicOr(err, 1u);
    L.len = (L.elem < kNElem && kSymbol[L.elem][1] ? 2 : 1) + 3 + fixed6_len(L.c[0]) + fixed6_len(L.c[1]) +
            fixed6_len(L.c[2]) + 1;
    return L;
}

__global__ void __launch_bounds__(kXyzThreads) k_xyz_measure(StateBuf b, const uint32_t* __restrict__ pos_of_slot,
                                                             uint32_t n, unsigned long long* __restrict__ block_len,
                                                             uint32_t* err) {
    using Reduce = cub::BlockReduce<unsigned long long, kXyzThreads>;
    __shared__ typename Reduce::TempStorage tmp;
    const uint32_t s = blockIdx.x * kXyzThreads + threadIdx.x;
    unsigned long long len = 0;
    if (s < n) len = (unsigned long long)load_line(b, pos_of_slot, s, err).len;
    const unsigned long long tot = Reduce(tmp).Sum(len);
    if (threadIdx.x == 0) block_len[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kXyzThreads) k_xyz_write(StateBuf b, const uint32_t* __restrict__ pos_of_slot,
                                                           uint32_t n, const unsigned long long* __restrict__ block_off,
                                                           char* __restrict__ text, uint32_t* err) {
    using Scan = cub::BlockScan<unsigned, kXyzThreads>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ __align__(16) char stage[kXyzThreads * kXyzMaxLine + 16];
    __shared__ unsigned block_total;
    const uint32_t s = blockIdx.x * kXyzThreads + threadIdx.x;
    Line L;
    L.len = 0;
    if (s < n) L = load_line(b, pos_of_slot, s, err);
    unsigned off, tot;
    Scan(tmp).ExclusiveSum((unsigned)L.len, off, tot);
    if (threadIdx.x == 0) block_total = tot;
    const unsigned long long base = block_off[blockIdx.x];
    const unsigned pad = (unsigned)(base & 15);
    if (s < n && L.elem < kNElem) {
        char* p = stage + pad + off;
        *p++ = kSymbol[L.elem][0];
        if (kSymbol[L.elem][1]) *p++ = kSymbol[L.elem][1];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            *p++ = ' ';
            p = fixed6_put(L.c[k], p);
        }
        *p = '\n';
    }
    __syncthreads();
    // stage[k] holds the byte for text[base - pad + k]; base - pad is 16-aligned
    const unsigned end = pad + block_total;
    char* dst = text + (base - pad);
    const unsigned words = (end + 15) >> 4;
    for (unsigned w = threadIdx.x; w < words; w += kXyzThreads) {
        const unsigned lo = w << 4, hi = lo + 16;
        if (lo >= pad && hi <= end) {
            *reinterpret_cast<uint4*>(dst + lo) = *reinterpret_cast<const uint4*>(stage + lo);
        } else {
            for (unsigned k = (lo > pad ? lo : pad); k < (hi < end ? hi : end); ++k) dst[k] = stage[k];
        }
    }
}

struct ExportState {
    unsigned long long* block = nullptr;  // [nblocks + 1]: lengths, then offsets
    unsigned long long* off = nullptr;    // [nblocks + 1]
    uint32_t* err = nullptr;
    size_t cap_blocks = 0;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    char* text = nullptr;
    size_t text_cap = 0;
};

int require_state(gx_handle* h) {
    if (!h) return GX_ERR_ARG;
    if (!h->cap) return set_err(h, GX_ERR_STATE, "no state uploaded (call gx_set_state first)");
    return GX_OK;
}

ExportState& export_of(gx_handle* h) {
    if (!h->xport) h->xport = new ExportState();
    return *static_cast<ExportState*>(h->xport);
}

}  // namespace

void export_free(gx_handle* h) {
    if (!h->xport) return;
    ExportState* e = static_cast<ExportState*>(h->xport);
    cudaFree(e->block);
    cudaFree(e->off);
    cudaFree(e->err);
    cudaFree(e->temp);
    cudaFree(e->text);
    delete e;
    h->xport = nullptr;
}

}  // namespace gx

using namespace gx;

extern "C" int gx_xyz_frame(gx_handle* h, uint64_t tick, char* out, size_t cap, size_t* len) {
    int rc = require_state(h);
    if (rc) return rc;
    if (!len) return set_err(h, GX_ERR_ARG, "gx_xyz_frame: len is null");
    char head[64];
    const int hl = std::snprintf(head, sizeof head, "%zu\nframe %llu\n", h->n, (unsigned long long)tick);
    const uint32_t n = (uint32_t)h->n;
    const uint32_t nb = (uint32_t)((n + kXyzThreads - 1) / kXyzThreads);
    ExportState& E = export_of(h);
    if (nb + 1 > E.cap_blocks || !E.err) {
        cudaFree(E.block);
        cudaFree(E.off);
        cudaFree(E.temp);
        E.block = E.off = nullptr;
        E.temp = nullptr;
        E.cap_blocks = 0;
        const size_t c = nb + 1;
        GX_CUDA(h, cudaMalloc(&E.block, c * sizeof(unsigned long long)));
        GX_CUDA(h, cudaMalloc(&E.off, c * sizeof(unsigned long long)));
        if (!E.err) GX_CUDA(h, cudaMalloc(&E.err, sizeof(uint32_t)));
        size_t tb = 0;
        GX_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, tb, E.block, E.off, (int)c, h->stream));
        GX_CUDA(h, cudaMalloc(&E.temp, tb));
        E.temp_bytes = tb;
        E.cap_blocks = c;
    }
    const StateBuf& b = h->buf[h->cur];
    unsigned long long total = 0;
    if (n) {
        GX_CUDA(h, cudaMemsetAsync(E.err, 0, sizeof(uint32_t), h->stream));
        GX_CUDA(h, cudaMemsetAsync(E.block + nb, 0, sizeof(unsigned long long), h->stream));
        prof_begin(h, "xyz_measure");
        GX_LAUNCH(h, k_xyz_measure, nb, kXyzThreads, b, h->pos_of_slot, n, E.block, E.err);
        prof_end(h, "xyz_measure");
        size_t tb = E.temp_bytes;
        GX_CUDA(h, cub::DeviceScan::ExclusiveSum(E.temp, tb, E.block, E.off, (int)(nb + 1), h->stream));
        uint32_t herr = 0;
        GX_CUDA(h, cudaMemcpyAsync(&total, E.off + nb, sizeof total, cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaMemcpyAsync(&herr, E.err, sizeof herr, cudaMemcpyDeviceToHost, h->stream));
        GX_CUDA(h, cudaStreamSynchronize(h->stream));
        if (herr)
            return set_err(h, GX_ERR_UNSUPPORTED,
                           "gx_xyz_frame: a coordinate of magnitude >= 2^100 or an unknown element");
    }
    *len = (size_t)hl + (size_t)total;
    if (!out || cap < *len) return set_err(h, GX_ERR_CAPACITY, "gx_xyz_frame: out holds fewer than *len bytes");
    std::memcpy(out, head, (size_t)hl);
    if (!n) return GX_OK;
    if (total > E.text_cap) {
        cudaFree(E.text);
        E.text = nullptr;
        E.text_cap = 0;
        GX_CUDA(h, cudaMalloc(&E.text, (size_t)total));
        E.text_cap = (size_t)total;
    }
    prof_begin(h, "xyz_write");
    GX_LAUNCH(h, k_xyz_write, nb, kXyzThreads, b, h->pos_of_slot, n, E.off, E.text, E.err);
    prof_end(h, "xyz_write");
    GX_CUDA(h, cudaMemcpyAsync(out + hl, E.text, (size_t)total, cudaMemcpyDeviceToHost, h->stream));
    GX_CUDA(h, cudaStreamSynchronize(h->stream));
    GX_CUDA(h, cudaGetLastError());
    return GX_OK;
}
