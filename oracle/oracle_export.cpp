// Test infrastructure only: the XYZ frame text of export::write_frame
// (src/export/mod.rs:152-172) restated with the C library's printf, the
// checker of gx_xyz_frame and the CPU baseline of its bench leg.  Nothing in
// the product links it.
//
// "{n}\nframe {tick}\n", then "{symbol} {x:.6} {y:.6} {z:.6}\n" per atom.
// printf's %.6f is the exact binary value rounded to 6 decimals in the
// current rounding mode (round to nearest, ties to even), which is what
// Rust's {:.6} prints; only the non-finite spellings differ and are mapped
// to Rust's ("NaN", "inf", "-inf").  One thread, like the reference's loop.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "oracle.h"

namespace {

const char* const kSymbols[10] = {"H", "He", "C", "N", "O", "Na", "Si", "P", "S", "Fe"};

void put_fixed6(std::string& s, double x) {
    char buf[400];
    if (std::isnan(x)) {
        s += "NaN";
    } else if (std::isinf(x)) {
        s += x > 0 ? "inf" : "-inf";
    } else {
        int k = std::snprintf(buf, sizeof buf, "%.6f", x);
        s.append(buf, (size_t)k);
    }
}

}  // namespace

extern "C" size_t orc_xyz_frame(size_t n, uint64_t tick, const double* pos, const uint8_t* elem, char* out,
                                size_t cap) {
    std::string s;
    s.reserve(n * 40 + 64);
    s += std::to_string(n);
    s += "\nframe ";
    s += std::to_string((unsigned long long)tick);
    s += "\n";
    for (size_t i = 0; i < n; ++i) {
        s += elem[i] < 10 ? kSymbols[elem[i]] : "?";
        for (int k = 0; k < 3; ++k) {
            s += ' ';
            put_fixed6(s, pos[3 * i + k]);
        }
        s += '\n';
    }
    if (out && cap >= s.size()) std::memcpy(out, s.data(), s.size());
    return s.size();
}
