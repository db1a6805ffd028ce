// Matrix Market input (host), after the reference's matrix_market_istream
// (boost/numeric/mtl/io/matrix_market.hpp:44-214):
//   header     "%%MatrixMarket matrix <coordinate|array> <real|integer|
//              complex|pattern> <general|symmetric|skew-symmetric|hermitian>";
//              the marker and "matrix" are compared as written, the sparsity
//              and symmetry words in lower case (matrix_market.hpp:90-101,
//              177-186); then comment lines starting with '%'
//   sizes      rows cols [entries] (coordinate: entries)
//   entries    coordinate: "r c [value]" (1-based) for each entry, stopping
//              early when the input runs out (matrix_market.hpp:109-115);
//              array: every value, column by column (:117-119)
//   insertion  ins[r][c] << v with the inserter's default store update: a
//              later entry at the same position replaces an earlier one;
//              off-diagonal entries of symmetric / skew-symmetric / Hermitian
//              files are mirrored as v / -v / conj(v) (:122-137)
//   values     pattern entries are stored as 0.0 (which_value(pattern_type),
//              :147); integers are converted to double; complex values cannot
//              go into a real matrix (runtime_error, :148)
// The result is CSR with the entries of each row sorted by column, as the
// reference's compressed2D inserter leaves them.
#pragma once
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace mtlg {

struct MmCsr {
    int64_t n_rows = 0, n_cols = 0;
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> val;
};

class MmParser {
  public:
    explicit MmParser(std::string text) : s_(std::move(text)), p_(s_.c_str()), end_(s_.c_str() + s_.size()) {}

    bool token(std::string& out)
    {
        skip_space();
        if (p_ >= end_) return false;
        const char* b = p_;
        while (p_ < end_ && !isspace((unsigned char)*p_)) ++p_;
        out.assign(b, p_);
        return true;
    }
    // the reference reads one non-blank character and, if it is '%', drops
    // the rest of the line
    void skip_comments()
    {
        for (;;) {
            skip_space();
            if (p_ < end_ && *p_ == '%') {
                while (p_ < end_ && *p_ != '\n') ++p_;
            } else {
                return;
            }
        }
    }
    bool read_int(long long& v)
    {
        skip_space();
        if (p_ >= end_) return false;
        char* e = nullptr;
        errno = 0;
        v = strtoll(p_, &e, 10);
        if (e == p_ || errno) return false;
        p_ = e;
        return true;
    }
    bool read_double(double& v)
    {
        skip_space();
        if (p_ >= end_) return false;
        char* e = nullptr;
        v = strtod(p_, &e);
        if (e == p_) return false;
        p_ = e;
        return true;
    }

  private:
    void skip_space()
    {
        while (p_ < end_ && isspace((unsigned char)*p_)) ++p_;
    }
    std::string s_;
    const char* p_;
    const char* end_;
};

inline std::string lower(std::string s)
{
    for (char& ch : s) ch = char(tolower((unsigned char)ch));
    return s;
}

// Parses a Matrix Market file into host CSR.  Status codes:
// MTLG_ERR_FILE_NOT_FOUND (mtl::io::file_not_found), MTLG_ERR_FORMAT
// (mtl::runtime_error of the reader), MTLG_ERR_TOO_LARGE.
inline int mm_read_file(const char* path, MmCsr& out)
{
    FILE* f = path ? fopen(path, "rb") : nullptr;
    if (!f) {
        set_error("matrix_market_istream: Error in input stream! Probably file %s not found.", path ? path : "(null)");
        return MTLG_ERR_FILE_NOT_FOUND;
    }
    std::string text;
    char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, k);
    fclose(f);
    MmParser in(std::move(text));
    std::string marker, type, sparsity, format, symmetry;
    if (!in.token(marker) || !in.token(type) || !in.token(sparsity) || !in.token(format) || !in.token(symmetry)) {
        set_error("File not in Matrix Market format");
        return MTLG_ERR_FORMAT;
    }
    if (marker != "%%MatrixMarket") {
        set_error("File not in Matrix Market format");
        return MTLG_ERR_FORMAT;
    }
    if (type != "matrix") {
        set_error("Try to read matrix from non-matrix file");
        return MTLG_ERR_FORMAT;
    }
    sparsity = lower(sparsity);
    symmetry = lower(symmetry);
    const bool coordinate = sparsity == "coordinate";
    if (!coordinate && sparsity != "array") {
        set_error("unknown sparsity '%s'", sparsity.c_str());
        return MTLG_ERR_FORMAT;
    }
    enum { GENERAL, SYMMETRIC, SKEW, HERMITIAN } sym;
    if (symmetry == "general") sym = GENERAL;
    else if (symmetry == "symmetric") sym = SYMMETRIC;
    else if (symmetry == "skew-symmetric") sym = SKEW;
    else if (symmetry == "hermitian") sym = HERMITIAN;
    else {
        set_error("unknown symmetry '%s'", symmetry.c_str());
        return MTLG_ERR_FORMAT;
    }
    enum { REAL, INTEGER, PATTERN } fmt;
    if (format == "real") fmt = REAL;
    else if (format == "integer") fmt = INTEGER;
    else if (format == "pattern") fmt = PATTERN;
    else if (format == "complex") {
        set_error("Cannot convert complex value in real");
        return MTLG_ERR_FORMAT;
    } else {
        set_error("Unknown tag for matrix value type in file");
        return MTLG_ERR_FORMAT;
    }
    in.skip_comments();
    long long nr = 0, nc = 0, nz = 0;
    if (!in.read_int(nr) || !in.read_int(nc) || nr < 0 || nc < 0 || (coordinate && (!in.read_int(nz) || nz < 0))) {
        set_error("bad size line");
        return MTLG_ERR_FORMAT;
    }
    if (nr > INT32_MAX || nc > INT32_MAX) {
        set_error("%lld x %lld exceeds int32 indexing", nr, nc);
        return MTLG_ERR_TOO_LARGE;
    }
    struct Ent {
        int32_t r, c;
        int64_t seq;
        double v;
    };
    std::vector<Ent> ents;
    int64_t seq = 0;
    auto read_value = [&](double& v) -> bool {
        if (fmt == PATTERN) { v = 0.0; return true; }
        if (fmt == INTEGER) {
            long long iv;
            if (!in.read_int(iv)) return false;
            v = double(iv);
            return true;
        }
        return in.read_double(v);
    };
    auto insert = [&](long long r, long long c, double v) -> int {
        if (r < 0 || r >= nr || c < 0 || c >= nc) {
            set_error("entry (%lld, %lld) outside the %lld x %lld matrix", r + 1, c + 1, nr, nc);
            return MTLG_ERR_FORMAT;
        }
        ents.push_back({int32_t(r), int32_t(c), seq++, v});
        if (r != c && sym != GENERAL) {
            if (c >= nr || r >= nc) {
                set_error("mirrored entry (%lld, %lld) outside the matrix", c + 1, r + 1);
                return MTLG_ERR_FORMAT;
            }
            ents.push_back({int32_t(c), int32_t(r), seq++, sym == SKEW ? -v : v});
        }
        return MTLG_OK;
    };
    if (coordinate) {
        ents.reserve(size_t(sym == GENERAL ? nz : 2 * nz));
        for (long long i = 0; i < nz; ++i) {
            long long r, c;
            if (!in.read_int(r) || !in.read_int(c)) break;   // input ran out
            double v;
            if (!read_value(v)) break;
            MTLG_TRY(insert(r - 1, c - 1, v));
        }
    } else {
        for (long long c = 0; c < nc; ++c)
            for (long long r = 0; r < nr; ++r) {
                double v;
                if (!read_value(v)) {
                    set_error("array file ends before its %lld x %lld values", nr, nc);
                    return MTLG_ERR_FORMAT;
                }
                MTLG_TRY(insert(r, c, v));
            }
    }
    // row-major, columns sorted; the last write to a position wins
    std::sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) {
        return a.r != b.r ? a.r < b.r : a.c != b.c ? a.c < b.c : a.seq < b.seq;
    });
    out.n_rows = nr;
    out.n_cols = nc;
    out.rp.assign(size_t(nr) + 1, 0);
    out.ci.clear();
    out.val.clear();
    for (size_t i = 0; i < ents.size(); ++i) {
        if (i + 1 < ents.size() && ents[i + 1].r == ents[i].r && ents[i + 1].c == ents[i].c) continue;
        out.ci.push_back(ents[i].c);
        out.val.push_back(ents[i].v);
        out.rp[size_t(ents[i].r) + 1]++;
    }
    for (int64_t i = 0; i < nr; ++i) out.rp[size_t(i) + 1] += out.rp[size_t(i)];
    if (out.ci.size() > size_t(INT32_MAX)) {
        set_error("%zu entries exceed int32 indexing", out.ci.size());
        return MTLG_ERR_TOO_LARGE;
    }
    return MTLG_OK;
}

}  // namespace mtlg
