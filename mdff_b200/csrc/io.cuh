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
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
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

// Ew.d: [-]0.d1..dd E+ee (|exponent| <= 99) or [-]0.d1..dd+eee; the optional
// leading zero is dropped only when the field is too narrow for it.
inline void fmt_E(std::string& o, double v, int w, int d) {
    if (std::isnan(v)) { pad_left(o, "NaN", w); return; }
    if (std::isinf(v)) { pad_left(o, v < 0 ? "-Infinity" : "Infinity", w); return; }
    const bool neg = std::signbit(v);
    std::string digits;
    int e = 0;
    if (v == 0.0) {
        digits.assign(d, '0');
    } else {
        char buf[64];
        std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(v));
        const char* p = buf;
        for (; *p && *p != 'e'; ++p)
            if (*p != '.') digits.push_back(*p);
        e = std::atoi(p + 1) + 1;
    }
    char ex[16];
    if (std::abs(e) <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
    else std::snprintf(ex, sizeof ex, "%c%03d", e < 0 ? '-' : '+', std::abs(e));
    std::string s = std::string(neg ? "-" : "") + "0." + digits + ex;
    if ((int)s.size() > w) s = std::string(neg ? "-" : "") + "." + digits + ex;
    pad_left(o, s, w);
}

inline void fmt_F(std::string& o, double v, int w, int d) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%.*f", d, v);
    pad_left(o, buf, w);
}

inline void fmt_I(std::string& o, long long v, int w) {
    char buf[32];
    std::snprintf(buf, sizeof buf, "%lld", v);
    pad_left(o, buf, w);
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
        if (file == MDFF_FILE_TRAJFF || file == MDFF_FILE_CONTFF) {
            o += "Cartesian\n";
            for (int i = 0; i < n; ++i) {
                fmt_A(o, h.atypei[itype[i] - 1], 3);
                for (int c = 0; c < ncol; ++c) fmt_E(o, col(c, i), 20, 12);
                o.push_back('\n');
            }
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
            for (int i = 0; i < n; ++i) {
                fmt_I(o, i + 1, 8);
                o += "  ";
                fmt_A(o, h.atypei[itype[i] - 1], 3);
                for (int c = 0; c < ncol; ++c) fmt_E(o, col(c, i), 24, 16);
                o.push_back('\n');
            }
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
