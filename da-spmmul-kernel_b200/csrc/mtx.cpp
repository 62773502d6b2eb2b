// mtx.cpp -- Matrix Market coordinate files to sorted CSR.
//
// The reference reads a file with mmio's banner and size parsers and fscanf
// per entry (util/spmatrix.hpp:286-333), turns a symmetric file into both
// triangles with makeSymmetric (spmatrix.hpp:219-284) -- which drops
// diagonal entries and repeated (row, col) pairs but compacts only the row
// and column arrays, so values after the first dropped entry belong to other
// positions -- and sorts by (row, col) (customSort, spmatrix.hpp:62-97).
//
// Here: the same structure (a general file keeps every entry, a symmetric
// file is mirrored and, by default, loses its diagonal and repeated pairs as
// in the reference), with every value kept beside its own (row, col).  The
// order is (row, col, position in the file), so repeated pairs of a general
// file come out in file order.  The whole file is read at once and parsed
// with strtol / strtof.
#include "daspmm.h"

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

struct Header {
    int nr = 0, nc = 0;
    long long entries = 0;
    int field = 0;     // 0 real, 1 integer, 2 pattern, 3 complex
    int symmetry = 0;  // 0 general, 1 symmetric, 2 skew-symmetric, 3 hermitian
    size_t body = 0;   // offset of the first entry
};

bool read_file(const char *path, std::string *out)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) {
        std::fclose(f);
        return false;
    }
    out->resize((size_t)n);
    const size_t got = n ? std::fread(&(*out)[0], 1, (size_t)n, f) : 0;
    std::fclose(f);
    return got == (size_t)n;
}

std::string lower(std::string s)
{
    for (char &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Banner, comments and size line.
daspmm_status parse_header(const std::string &t, Header *h)
{
    size_t eol = t.find('\n');
    const std::string banner = lower(t.substr(0, eol));
    char mm[64], obj[64], fmt[64], field[64], sym[64];
    if (std::sscanf(banner.c_str(), "%63s %63s %63s %63s %63s", mm, obj, fmt, field, sym) != 5)
        return DASPMM_ERR_BAD_MATRIX;
    if (std::strcmp(mm, "%%matrixmarket") != 0 || std::strcmp(obj, "matrix") != 0)
        return DASPMM_ERR_BAD_MATRIX;
    if (std::strcmp(fmt, "coordinate") != 0) return DASPMM_ERR_UNSUPPORTED;  // dense "array"
    if (!std::strcmp(field, "real") || !std::strcmp(field, "double")) h->field = 0;
    else if (!std::strcmp(field, "integer")) h->field = 1;
    else if (!std::strcmp(field, "pattern")) h->field = 2;
    else if (!std::strcmp(field, "complex")) h->field = 3;
    else return DASPMM_ERR_BAD_MATRIX;
    if (!std::strcmp(sym, "general")) h->symmetry = 0;
    else if (!std::strcmp(sym, "symmetric")) h->symmetry = 1;
    else if (!std::strcmp(sym, "skew-symmetric")) h->symmetry = 2;
    else if (!std::strcmp(sym, "hermitian")) h->symmetry = 3;
    else return DASPMM_ERR_BAD_MATRIX;
    size_t p = eol == std::string::npos ? t.size() : eol + 1;
    for (;;) {  // comment and blank lines
        if (p >= t.size()) return DASPMM_ERR_BAD_MATRIX;
        size_t e = t.find('\n', p);
        if (e == std::string::npos) e = t.size();
        const char *q = t.c_str() + p;
        while (q < t.c_str() + e && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
        if (q == t.c_str() + e || *q == '%') {
            p = e + 1;
            continue;
        }
        long long nr, nc, nz;
        if (std::sscanf(t.substr(p, e - p).c_str(), "%lld %lld %lld", &nr, &nc, &nz) != 3)
            return DASPMM_ERR_BAD_MATRIX;
        if (nr < 0 || nc < 0 || nz < 0 || nr > INT_MAX - 1 || nc > INT_MAX) return DASPMM_ERR_BAD_MATRIX;
        h->nr = (int)nr;
        h->nc = (int)nc;
        h->entries = nz;
        h->body = e + 1;
        return DASPMM_OK;
    }
}

struct Entry {
    int row, col;
    long long seq;
    float val;
};

daspmm_status parse_entries(const std::string &t, const Header &h, std::vector<Entry> *out)
{
    out->clear();
    out->reserve((size_t)h.entries);
    const char *p = t.c_str() + std::min(h.body, t.size());
    for (long long i = 0; i < h.entries; ++i) {
        char *e = nullptr;
        errno = 0;
        const long r = std::strtol(p, &e, 10);
        if (e == p) return DASPMM_ERR_BAD_MATRIX;  // fewer entries than the size line says
        p = e;
        const long c = std::strtol(p, &e, 10);
        if (e == p) return DASPMM_ERR_BAD_MATRIX;
        p = e;
        float v = 1.0f;
        if (h.field == 0 || h.field == 1) {
            v = std::strtof(p, &e);
            if (e == p) return DASPMM_ERR_BAD_MATRIX;
            p = e;
        }
        if (r < 1 || r > h.nr || c < 1 || c > h.nc) return DASPMM_ERR_BAD_MATRIX;
        out->push_back(Entry{(int)r - 1, (int)c - 1, i, v});
        // the rest of the line (a complex part, trailing text) is ignored
        while (*p && *p != '\n') ++p;
    }
    return DASPMM_OK;
}

}  // namespace

extern "C" {

daspmm_status daspmm_mtx_info(const char *path, daspmm_mtx_header *out)
{
    if (!path || !out) return DASPMM_ERR_INVALID;
    std::string t;
    if (!read_file(path, &t)) return DASPMM_ERR_INVALID;
    Header h;
    const daspmm_status s = parse_header(t, &h);
    if (s != DASPMM_OK) return s;
    out->nr = h.nr;
    out->nc = h.nc;
    out->entries = h.entries;
    out->field = h.field;
    out->symmetry = h.symmetry;
    out->nnz_max = h.symmetry == 1 ? 2 * h.entries : h.entries;
    return DASPMM_OK;
}

daspmm_status daspmm_mtx_read(const char *path, int flags, long long cap, int *rowPtr,
                              int *rowIdx, int *colIdx, float *values, int *nnz_out)
{
    if (!path || !rowPtr || !nnz_out || cap < 0) return DASPMM_ERR_INVALID;
    *nnz_out = 0;
    std::string t;
    if (!read_file(path, &t)) return DASPMM_ERR_INVALID;
    Header h;
    daspmm_status s = parse_header(t, &h);
    if (s != DASPMM_OK) return s;
    if (h.field == 3) return DASPMM_ERR_UNSUPPORTED;  // complex values
    std::vector<Entry> ent;
    s = parse_entries(t, h, &ent);
    if (s != DASPMM_OK) return s;
    t.clear();
    t.shrink_to_fit();
    const bool mirror = h.symmetry == 1;
    if (mirror) {
        const size_t n = ent.size();
        for (size_t i = 0; i < n; ++i)
            if (ent[i].row != ent[i].col)
                ent.push_back(Entry{ent[i].col, ent[i].row, h.entries + (long long)i, ent[i].val});
    }
    std::sort(ent.begin(), ent.end(), [](const Entry &a, const Entry &b) {
        if (a.row != b.row) return a.row < b.row;
        if (a.col != b.col) return a.col < b.col;
        return a.seq < b.seq;
    });
    if (mirror) {  // the reference's makeSymmetric: no diagonal, no repeated pairs
        const bool keep_diag = (flags & DASPMM_MTX_KEEP_DIAGONAL) != 0;
        size_t w = 0;
        for (size_t i = 0; i < ent.size(); ++i) {
            const Entry &e = ent[i];
            if (!keep_diag && e.row == e.col) continue;
            if (w > 0 && ent[w - 1].row == e.row && ent[w - 1].col == e.col) continue;
            ent[w++] = e;
        }
        ent.resize(w);
    }
    if ((long long)ent.size() > INT_MAX) return DASPMM_ERR_UNSUPPORTED;
    if ((long long)ent.size() > cap) return DASPMM_ERR_WORKSPACE;
    if (!ent.empty() && (!colIdx || !values)) return DASPMM_ERR_INVALID;
    std::fill(rowPtr, rowPtr + h.nr + 1, 0);
    for (size_t i = 0; i < ent.size(); ++i) {
        ++rowPtr[ent[i].row + 1];
        colIdx[i] = ent[i].col;
        values[i] = ent[i].val;
        if (rowIdx) rowIdx[i] = ent[i].row;
    }
    for (int r = 0; r < h.nr; ++r) rowPtr[r + 1] += rowPtr[r];
    *nnz_out = (int)ent.size();
    return DASPMM_OK;
}

}  // extern "C"
