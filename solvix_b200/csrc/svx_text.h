// Text helpers shared by the host writers and readers.
#pragma once

#include <charconv>
#include <cmath>
#include <string>

namespace svx {

// Rust's `{}` Display of an f64 (core::fmt): the shortest digits that read
// back to the same bits (std::to_chars' shortest scientific form supplies
// them with their decimal exponent), laid out positionally with zeros,
// never an exponent; "-0" for negative zero, "NaN", "inf" and "-inf".
inline void rust_display_f64(std::string& out, double v) {
    if (std::isnan(v)) {
        out += "NaN";
        return;
    }
    if (std::isinf(v)) {
        out += v > 0 ? "inf" : "-inf";
        return;
    }
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    const char* p = buf;
    if (*p == '-') {
        out += '-';
        ++p;
    }
    char digits[32];
    int nd = 0;
    for (; p < r.ptr && *p != 'e'; ++p)
        if (*p != '.') digits[nd++] = *p;
    int e = 0;  // the exponent after "e+" / "e-", read up to the end of the output
    const bool neg_e = (p + 1 < r.ptr && p[1] == '-');
    for (const char* q = p + 2; q < r.ptr; ++q) e = 10 * e + (*q - '0');
    if (neg_e) e = -e;
    if (e >= nd - 1) {  // integer: the digits, then zeros
        out.append(digits, size_t(nd));
        out.append(size_t(e - (nd - 1)), '0');
    } else if (e >= 0) {
        out.append(digits, size_t(e + 1));
        out += '.';
        out.append(digits + e + 1, size_t(nd - e - 1));
    } else {
        out += "0.";
        out.append(size_t(-e - 1), '0');
        out.append(digits, size_t(nd));
    }
}

}  // namespace svx
