// oracle_grid.h -- shared pieces of the CPU oracle (TEST INFRASTRUCTURE
// ONLY): Vec3 arithmetic with the reference's rounding, rem_euclid,
// min_image and the SpatialGrid cell list (src/physics/grid.rs:37-306).
// Included by oracle.cpp (FP64 restatement) and oracle_dual.cpp (the
// dual-number adjoint reference).
#ifndef GENESIS_ORACLE_GRID_H
#define GENESIS_ORACLE_GRID_H

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace orcg {


const double kEps = 2.220446049250313e-16;  // f64::EPSILON
const uint32_t kEmpty = 0xFFFFFFFFu;        // grid.rs:34

struct V3 {
    double x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }  // math/mod.rs:47-49
inline double len2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }   // math/mod.rs:29-31
inline V3 at(const double* p, size_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

// f64::rem_euclid (Rust std): r = a % b; if r < 0 { r + |b| } else { r }.
inline double rem_euclid(double a, double b) {
    double r = std::fmod(a, b);
    return r < 0.0 ? r + std::fabs(b) : r;
}

// grid.rs:300-306
inline V3 min_image(V3 d, const double* L) {
    return {d.x - L[0] * std::round(d.x / L[0]), d.y - L[1] * std::round(d.y / L[1]),
            d.z - L[2] * std::round(d.z / L[2])};
}

// grid.rs:37-47
const int kOffsets[27][3] = {
    {-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, -1}, {-1, 0, 0}, {-1, 0, 1},
    {-1, 1, -1},  {-1, 1, 0},  {-1, 1, 1},  {0, -1, -1}, {0, -1, 0}, {0, -1, 1},
    {0, 0, -1},   {0, 0, 0},   {0, 0, 1},   {0, 1, -1},  {0, 1, 0},  {0, 1, 1},
    {1, -1, -1},  {1, -1, 0},  {1, -1, 1},  {1, 0, -1},  {1, 0, 0},  {1, 0, 1},
    {1, 1, -1},   {1, 1, 0},   {1, 1, 1}};

// SpatialGrid, grid.rs:50-296.
struct Grid {
    uint32_t dims[3];
    double cell[3];
    double L[3];
    std::vector<uint32_t> heads, touched, next, chain, nchain;

    Grid(const double* box, double min_cell) {  // grid.rs:67-86
        for (int k = 0; k < 3; ++k) {
            double c = std::floor(box[k] / min_cell);
            if (c < 1.0) c = 1.0;  // .max(1.0)
            dims[k] = (uint32_t)c;
            L[k] = box[k];
        }
        for (int k = 0; k < 3; ++k) cell[k] = box[k] / (double)dims[k];
        heads.assign((size_t)dims[0] * dims[1] * dims[2], kEmpty);
    }
    uint32_t axis(double v, double period, double c, uint32_t n) const {  // grid.rs:229-232
        double u = rem_euclid(v + 0.5 * period, period);
        double f = std::floor(u / c);
        uint32_t i = f <= 0.0 ? 0u : (f >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)f);
        return std::min(i, n - 1);
    }
    size_t cell_index(V3 p) const {  // grid.rs:228-246
        uint32_t ix = axis(p.x, L[0], cell[0], dims[0]);
        uint32_t iy = axis(p.y, L[1], cell[1], dims[1]);
        uint32_t iz = axis(p.z, L[2], cell[2], dims[2]);
        return encode(ix, iy, iz);
    }
    size_t encode(uint32_t ix, uint32_t iy, uint32_t iz) const {
        return (size_t)(ix + dims[0] * (iy + dims[1] * iz));
    }
    void decode(uint32_t idx, uint32_t* cx, uint32_t* cy, uint32_t* cz) const {  // grid.rs:248-256
        uint32_t nxny = dims[0] * dims[1];
        *cz = idx / nxny;
        uint32_t rem = idx % nxny;
        *cy = rem / dims[0];
        *cx = rem % dims[0];
    }
    size_t neighbor(uint32_t cx, uint32_t cy, uint32_t cz, int dx, int dy, int dz) const {
        auto w = [](int64_t v, int64_t n) { int64_t r = v % n; return r < 0 ? r + n : r; };
        return encode((uint32_t)w((int64_t)cx + dx, dims[0]), (uint32_t)w((int64_t)cy + dy, dims[1]),
                      (uint32_t)w((int64_t)cz + dz, dims[2]));
    }
    bool is_canonical(const int* o) const {  // grid.rs:275-296 compared with the offset itself
        int d[3] = {o[0], o[1], o[2]};
        for (int k = 0; k < 3; ++k)
            if (dims[k] <= 1) d[k] = 0;
        int first = 0;
        for (int k = 0; k < 3; ++k)
            if (d[k] != 0) { first = d[k]; break; }
        int c[3];
        if (first == 1) { c[0] = d[0]; c[1] = d[1]; c[2] = d[2]; }
        else if (first == -1) { c[0] = -d[0]; c[1] = -d[1]; c[2] = -d[2]; }
        else { c[0] = c[1] = c[2] = 0; }
        return c[0] == o[0] && c[1] == o[1] && c[2] == o[2];
    }
    void build(const double* pos, size_t n) {  // grid.rs:99-113
        for (uint32_t ci : touched) heads[ci] = kEmpty;
        touched.clear();
        next.assign(n, kEmpty);
        for (size_t slot = 0; slot < n; ++slot) {
            size_t ci = cell_index(at(pos, slot));
            if (heads[ci] == kEmpty) touched.push_back((uint32_t)ci);
            next[slot] = heads[ci];
            heads[ci] = (uint32_t)slot;
        }
    }
    static void gather(const std::vector<uint32_t>& nx, uint32_t head, std::vector<uint32_t>& buf) {
        buf.clear();
        for (uint32_t cur = head; cur != kEmpty; cur = nx[cur]) buf.push_back(cur);
    }
    // grid.rs:119-153 with check_pair (grid.rs:201-225) inlined; emit(a, b, delta, d).
    template <class F>
    void neighbors(const double* pos, double cutoff, F&& emit) {
        double cd2 = cutoff * cutoff;
        auto check = [&](uint32_t sa, uint32_t sb) {
            V3 delta = min_image(sub(at(pos, sa), at(pos, sb)), L);
            double d2 = len2(delta);
            if (d2 >= cd2) return;
            double d = std::sqrt(d2);
            if (d <= kEps) return;
            emit(sa, sb, delta, d);
        };
        for (uint32_t ci : touched) {
            gather(next, heads[ci], chain);
            uint32_t cx, cy, cz;
            decode(ci, &cx, &cy, &cz);
            for (size_t i = 0; i < chain.size(); ++i)
                for (size_t j = i + 1; j < chain.size(); ++j) check(chain[i], chain[j]);
            for (const auto& o : kOffsets) {
                if (o[0] == 0 && o[1] == 0 && o[2] == 0) continue;
                size_t nc = neighbor(cx, cy, cz, o[0], o[1], o[2]);
                if (nc == ci || heads[nc] == kEmpty) continue;
                if (!is_canonical(o)) continue;
                gather(next, heads[nc], nchain);
                for (uint32_t sa : chain)
                    for (uint32_t sb : nchain) check(sa, sb);
            }
        }
    }
};

}  // namespace orcg

#endif
