// On-disk formats of MDFF and their streaming from the device.
//
// Formats (one frame each; the reference's writers are cited per kind):
//   TRAJFF  write_trajff_xyz (src/config.f90:539-628): formatted (itraj_format
//           != 0) or Fortran unformatted sequential (== 0); trajff_data rvf /
//           rvn / rnf / rnn; positions folded into the cell first (kardir,
//           periodicbc, dirkar).
//   CONTFF  write_CONTFF (src/config.f90:206-250): formatted, positions,
//           velocities and forces, the file rewritten at every call.
//   EFGALL  write_EFGALL (src/field.f90:4140-4195): formatted (six
//           components per site) or unformatted (the full 3x3 efg_t array).
//   DIPFF   write_DIPFF (src/field.f90:4051-4083), EFALL write_EFALL
//           (src/field.f90:4205-4240): formatted.
// Explicit edit descriptors (I, F, E, A) are reproduced as the Fortran
// runtime prints them; list-directed lines (the "*" format, whose layout is
// processor dependent) follow the Intel runtime for integers and character
// items (I12; a blank before each character item) and print reals in a
// fixed 1PE24.16 layout that any list-directed READ accepts.  Unformatted
// records carry 4-byte little-endian length markers before and after, as both
// common Fortran runtimes write them.
//
// Streaming: a frame is a snapshot taken on the engine's stream (device
// copies of the arrays the format needs, positions folded into the cell on
// the device), copied to pinned host memory on a separate copy stream and
// formatted and written by a writer thread, so the time loop never waits for
// the disk unless every slot of the ring is still in flight.
#pragma once
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mdff_engine.h"

namespace mdff {
namespace io {

// ---- Fortran edit descriptors ---------------------------------------------
inline void pad_left(std::string& o, const std::string& s, int w) {
    if ((int)s.size() > w) {
        o.append(w, '*');
        return;
    }
    o.append(w - s.size(), ' ');
    o += s;
}

// Exact powers of ten in x87 extended precision (10^k = 5^k 2^k, 5^27 < 2^64).
inline long double pow10_exact(int k) {
    static const long double t[28] = {1e0L,  1e1L,  1e2L,  1e3L,  1e4L,  1e5L,  1e6L,  1e7L,  1e8L,  1e9L,
                                      1e10L, 1e11L, 1e12L, 1e13L, 1e14L, 1e15L, 1e16L, 1e17L, 1e18L, 1e19L,
                                      1e20L, 1e21L, 1e22L, 1e23L, 1e24L, 1e25L, 1e26L, 1e27L};
    return t[k];
}

// The d significant decimal digits of a > 0 (d <= 17) and its decimal
// exponent (a = 0.digits x 10^e), correctly rounded, without the general
// conversion: a times an exact power of ten in extended precision carries a
// relative error below 2^-64, far less than the distance of its fractional
// part from 1/2 except near a tie; near one (or outside the exact range)
// returns false and the caller converts exactly.
inline bool digits_fast(double a, int d, char* out, int& e) {
    if (!(a > 1e-25 && a < 1e25) || d > 17) return false;
    int e10 = (int)std::floor(std::log10(a));           // a in [10^e10, 10^(e10+1)), up to one off
    const long double top = pow10_exact(d);
    for (int attempt = 0; attempt < 3; ++attempt) {
        const int k = d - 1 - e10;                        // scale a by 10^k into [10^(d-1), 10^d)
        if (k > 27 || k < -27) return false;
        const long double m = k >= 0 ? (long double)a * pow10_exact(k) : (long double)a / pow10_exact(-k);
        if (m >= top) { ++e10; continue; }
        if (m < pow10_exact(d - 1)) { --e10; continue; }
        long double ip = std::floor(m);
        const long double frac = m - ip;
        if (std::fabs(frac - 0.5L) < 1e-3L) return false;
        if (frac > 0.5L) ip += 1.0L;
        if (ip >= top) { ip = pow10_exact(d - 1); ++e10; }
        unsigned long long u = (unsigned long long)ip;
        for (int j = d - 1; j >= 0; --j) {
            out[j] = (char)('0' + u % 10);
            u /= 10;
        }
        e = e10 + 1;
        return true;
    }
    return false;
}

// Ew.d: [-]0.d1..dd E+ee (|exponent| <= 99) or [-]0.d1..dd+eee; the optional
// leading zero is dropped only when the field is too narrow for it.
inline void fmt_E(std::string& o, double v, int w, int d) {
    if (std::isnan(v)) { pad_left(o, "NaN", w); return; }
    if (std::isinf(v)) { pad_left(o, v < 0 ? "-Infinity" : "Infinity", w); return; }
    char s[96];
    int k = 0, e = 0;
    if (std::signbit(v)) s[k++] = '-';
    const int zero_at = k;
    s[k++] = '0';
    s[k++] = '.';
    if (v == 0.0) {
        for (int j = 0; j < d && k < 80; ++j) s[k++] = '0';
    } else if (d <= 17 && digits_fast(std::fabs(v), d, s + k, e)) {
        k += d;
    } else {
        // d significant digits of the binary value, correctly rounded (as
        // the Fortran runtime prints them)
        char buf[64];
        const auto r = std::to_chars(buf, buf + sizeof buf, std::fabs(v), std::chars_format::scientific, d - 1);
        const char* p = buf;
        for (; p < r.ptr && *p != 'e' && k < 80; ++p)
            if (*p != '.') s[k++] = *p;
        int ex = 0;
        const char* q = p + 1;
        if (q < r.ptr && *q == '+') ++q;
        std::from_chars(q, (const char*)r.ptr, ex);
        e = ex + 1;
    }
    const int ae = std::abs(e);
    if (ae <= 99) {
        s[k++] = 'E';
        s[k++] = e < 0 ? '-' : '+';
    } else {
        s[k++] = e < 0 ? '-' : '+';
        s[k++] = (char)('0' + ae / 100 % 10);
    }
    s[k++] = (char)('0' + ae / 10 % 10);
    s[k++] = (char)('0' + ae % 10);
    const char* beg = s;
    if (k > w) {   // drop the optional leading zero
        std::memmove(s + zero_at, s + zero_at + 1, k - zero_at - 1);
        --k;
    }
    if (k > w) {
        o.append(w, '*');
        return;
    }
    o.append(w - k, ' ');
    o.append(beg, k);
}

inline void fmt_F(std::string& o, double v, int w, int d) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%.*f", d, v);
    pad_left(o, buf, w);
}

inline void fmt_I(std::string& o, long long v, int w) {
    char buf[32];
    const auto r = std::to_chars(buf, buf + sizeof buf, v);
    const int k = (int)(r.ptr - buf);
    if (k > w) {
        o.append(w, '*');
        return;
    }
    o.append(w - k, ' ');
    o.append(buf, k);
}

// character variable of declared length len (blank padded)
inline void fmt_A(std::string& o, const char* s, int len) {
    int k = 0;
    for (; k < len && s[k]; ++k) o.push_back(s[k]);
    o.append(len - k, ' ');
}

// list-directed items
inline void ld_ints(std::string& o, const int* v, int n) {
    for (int k = 0; k < n; ++k) fmt_I(o, v[k], 12);
    o.push_back('\n');
}
inline void ld_chars(std::string& o, const char (*s)[3], int n) {
    for (int k = 0; k < n; ++k) {
        o.push_back(' ');
        fmt_A(o, s[k], 3);
    }
    o.push_back('\n');
}
inline void ld_reals(std::string& o, const double* v, int n) {
    for (int k = 0; k < n; ++k) {
        o.push_back(' ');
        char buf[64];
        std::snprintf(buf, sizeof buf, "%24.16E", v[k]);
        o += buf;
    }
    o.push_back('\n');
}

// ---- unformatted sequential records ----------------------------------------
inline void rec(std::string& o, const void* p, size_t bytes) {
    const uint32_t m = (uint32_t)bytes;
    o.append((const char*)&m, 4);
    o.append((const char*)p, bytes);
    o.append((const char*)&m, 4);
}

// Number of data columns of a frame of each kind ([ncol][natm] doubles).
inline int frame_cols(int file, int data) {
    switch (file) {
        case MDFF_FILE_TRAJFF: return 3 + ((data & MDFF_DATA_V) ? 3 : 0) + ((data & MDFF_DATA_F) ? 3 : 0);
        case MDFF_FILE_CONTFF: return 9;
        case MDFF_FILE_EFGALL: return 6;
        case MDFF_FILE_DIPFF: return 3;
        case MDFF_FILE_EFALL: return 3;
        default: return -1;
    }
}

// One frame into o.  h: header; itype: 1-based type per atom; cols:
// [ncol][natm] (positions already folded into the cell for TRAJFF / CONTFF).
inline int format_frame(int file, int iformat, int data, const mdff_frame_header& h, const int* itype,
                        const double* cols, std::string& o) {
    const int n = h.natm, nt = h.ntype;
    if (n < 0 || nt < 1 || nt > MDFF_NTYPE_MAX) return MDFF_E_ARG;
    const int ncol = frame_cols(file, data);
    if (ncol < 0) return MDFF_E_ARG;
    for (int i = 0; i < n; ++i)
        if (itype[i] < 1 || itype[i] > nt) return MDFF_E_ARG;
    auto col = [&](int c, int i) { return cols[(size_t)c * n + i]; };
    const double* A = h.A;   // column-major: A[i + 3 j] = simu_cell%A(i+1, j+1)
    const bool bin = iformat == 0;
    if (bin && (file == MDFF_FILE_CONTFF || file == MDFF_FILE_DIPFF || file == MDFF_FILE_EFALL))
        return MDFF_E_UNSUPPORTED;   // the reference writes these formatted only
    if (!bin) {
        if (file == MDFF_FILE_TRAJFF) {
            fmt_I(o, n, 6); o.push_back('\n');
            fmt_A(o, h.system, 60); o.push_back('\n');
            for (int i = 0; i < 3; ++i) {   // rows of A, as write_trajff_xyz writes them
                for (int j = 0; j < 3; ++j) fmt_F(o, A[i + 3 * j], 20, 12);
                o.push_back('\n');
            }
            fmt_I(o, nt, 4); o.push_back('\n');
        } else if (file == MDFF_FILE_CONTFF) {
            fmt_I(o, n, 12); o.push_back('\n');
            fmt_A(o, h.system, 60); o.push_back('\n');
            for (int j = 0; j < 3; ++j) {   // columns of A (lattice vectors)
                for (int i = 0; i < 3; ++i) fmt_F(o, A[i + 3 * j], 20, 12);
                o.push_back('\n');
            }
            fmt_I(o, nt, 4); o.push_back('\n');
        } else {
            ld_ints(o, &n, 1);
            o.push_back(' ');
            fmt_A(o, h.system, 60); o.push_back('\n');
            for (int j = 0; j < 3; ++j) ld_reals(o, A + 3 * j, 3);
            ld_ints(o, &nt, 1);
        }
        ld_chars(o, h.atypei, nt);
        ld_ints(o, h.natmi, nt);
        // per-atom lines: chunks formatted on host threads, joined in order
        const bool traj = file == MDFF_FILE_TRAJFF || file == MDFF_FILE_CONTFF;
        auto line = [&](std::string& s, int i) {
            if (traj) {
                fmt_A(s, h.atypei[itype[i] - 1], 3);
                for (int c = 0; c < ncol; ++c) fmt_E(s, col(c, i), 20, 12);
            } else {
                fmt_I(s, i + 1, 8);
                s += "  ";
                fmt_A(s, h.atypei[itype[i] - 1], 3);
                for (int c = 0; c < ncol; ++c) fmt_E(s, col(c, i), 24, 16);
            }
            s.push_back('\n');
        };
        auto lines = [&](std::string& s) {
            const int nth = n < 4096 ? 1 : (int)std::min<unsigned>(8u, std::max(1u, std::thread::hardware_concurrency()));
            if (nth == 1) {
                for (int i = 0; i < n; ++i) line(s, i);
                return;
            }
            std::vector<std::string> part(nth);
            std::vector<std::thread> th;
            for (int t = 0; t < nth; ++t)
                th.emplace_back([&, t] {
                    const int i0 = (int)((long long)n * t / nth), i1 = (int)((long long)n * (t + 1) / nth);
                    part[t].reserve((size_t)(i1 - i0) * (traj ? 4 + 20 * ncol : 14 + 24 * ncol));
                    for (int i = i0; i < i1; ++i) line(part[t], i);
                });
            for (auto& x : th) x.join();
            for (auto& x : part) s += x;
        };
        if (traj) {
            o += "Cartesian\n";
            lines(o);
        } else {
            const char* head =
                file == MDFF_FILE_EFGALL
                    ? "      ia type                   vxx                     vyy                     vzz          "
                      "           vxy                     vxz                     vyz"
                    : file == MDFF_FILE_DIPFF
                          ? "      ia type                   mux                       muy                      muz"
                          : "      ia type                   Ex                      Ey                      Ez";
            o += head;
            o.push_back('\n');
            lines(o);
        }
        return MDFF_OK;
    }
    // unformatted
    const int32_t n32 = n, nt32 = nt;
    rec(o, &n32, 4);
    rec(o, h.system, 60);
    for (int i = 0; i < 3; ++i) {
        double row[3];
        for (int j = 0; j < 3; ++j)   // TRAJFF: rows of A; EFGALL: columns (lattice vectors)
            row[j] = file == MDFF_FILE_TRAJFF ? A[i + 3 * j] : A[j + 3 * i];
        rec(o, row, sizeof row);
    }
    rec(o, &nt32, 4);
    rec(o, h.atypei, (size_t)3 * nt);
    std::vector<int32_t> ni(h.natmi, h.natmi + nt);
    rec(o, ni.data(), sizeof(int32_t) * nt);
    if (file == MDFF_FILE_TRAJFF) {
        rec(o, "C", 1);
        rec(o, cols, sizeof(double) * (size_t)ncol * n);
    } else {   // EFGALL: efg_t(natm, 3, 3), column-major
        std::vector<double> t((size_t)9 * n);
        const int comp[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i)
                for (int a = 0; a < n; ++a) t[(size_t)a + (size_t)n * (i + 3 * j)] = col(comp[i][j], a);
        rec(o, t.data(), sizeof(double) * t.size());
    }
    return MDFF_OK;
}

}  // namespace io
}  // namespace mdff
