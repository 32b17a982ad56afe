// Host input/output around the solve phase: a Matrix Market reader that gives the same CSR
// arrays as the reference's readers, a dense right-hand-side reader, and a binary factor file
// (G, D^-1, H) so that a factor construction need not be repeated.
//
// Matrix Market (the NIST exchange format: a "%%MatrixMarket matrix coordinate real
// general|symmetric" banner, '%' comment lines, a "rows cols entries" line, then one
// "row col value" line per entry, 1-based). The reference's readers and what they produce:
//   * AFIIM/src/rw_matrix.cpp:62-216 (also ACIFIM): real coordinate matrices, general or
//     symmetric, square; a symmetric file is expanded to general by appending the mirror of
//     every off-diagonal entry after the entries as read; rows are bucketed in input order
//     (counting sort) and each row is then sorted by column with the reference's quicksort
//     (AFIIM/src/qsort.cpp:52-86), which is restated here so that repeated entries come out
//     in the same order.
//   * PDFIIM/src/rw_matrix.cpp:60-150 (CSR form): a symmetric file is kept as its mirror
//     image, (row, col) read as (col, row), i.e. the upper triangle of a lower-stored file,
//     and flagged symmetric; general files as above.
// Values are parsed with std::from_chars, correctly rounded like the C library's strtod that
// the reference's fscanf("%lg") uses.

#include <omp.h>

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <system_error>
#include <vector>

#include "fiim_b200.h"

namespace fiim {
int set_error(int code, const char *fmt, ...);
}

namespace {

// The reference's quicksort of (column, value) pairs, ascending by column (qSort2 with
// ascdes = 0): middle-element pivot, Hoare-style partition, recursion left then right.
void qsort_pairs(int *col, double *val, int left, int right) {
    int i = left, j = right;
    const int pivot = col[(left + right) / 2];
    while (i <= j) {
        while (col[i] < pivot) i++;
        while (col[j] > pivot) j--;
        if (i <= j) {
            std::swap(col[i], col[j]);
            std::swap(val[i], val[j]);
            i++;
            j--;
        }
    }
    if (left < j) qsort_pairs(col, val, left, j);
    if (i < right) qsort_pairs(col, val, i, right);
}

struct MtxBuf {
    int n = 0, issym = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};
thread_local MtxBuf g_mtx;

// Token readers over [p, e): whitespace (space, tab, newline, carriage return) separates
// tokens, as for fscanf. A real may carry a leading '+', which from_chars does not take.
inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }
inline void skip_space(const char *&p, const char *e) {
    while (p < e && is_space(*p)) p++;
}
inline bool tok_integer(const char *&p, const char *e, long &x) {
    skip_space(p, e);
    auto r = std::from_chars(p, e, x);
    if (r.ec != std::errc()) return false;
    p = r.ptr;
    return true;
}
inline bool tok_real(const char *&p, const char *e, double &x) {
    skip_space(p, e);
    const char *b = p;
    if (b < e && *b == '+') ++b;
    auto r = std::from_chars(b, e, x, std::chars_format::general);
    if (r.ec != std::errc()) return false;
    p = r.ptr;
    return true;
}

struct Reader {
    std::string text;
    size_t pos = 0;
    bool line(std::string &out) {
        if (pos >= text.size()) return false;
        size_t e = text.find('\n', pos);
        if (e == std::string::npos) e = text.size();
        out.assign(text, pos, e - pos);
        pos = e + 1;
        if (!out.empty() && out.back() == '\r') out.pop_back();
        return true;
    }
    template <typename T, bool (*F)(const char *&, const char *, T &)>
    bool token(T &x) {
        const char *p = text.data() + pos;
        if (!F(p, text.data() + text.size(), x)) return false;
        pos = p - text.data();
        return true;
    }
    bool integer(long &x) { return token<long, tok_integer>(x); }
    bool real(double &x) { return token<double, tok_real>(x); }
};

// Files with fewer entries are read on one thread.
constexpr long kParallelEntries = 1 << 16;

// The coordinate entries of a large file, parsed in pieces on all host threads. The text
// after the size line is cut at line starts into pieces; each piece is read as whole
// (row, col, value) triples, and the pieces are joined in file order. It returns false, and
// the caller reads the entries on one thread, when any piece is not a run of whole triples
// (an entry broken across a cut, or anything that is not an entry) or when the pieces hold
// fewer than Z entries: the one-thread reader then gives its own result or error. Otherwise
// I, J and val hold the first Z triples as read (1-based, unchecked).
bool parse_entries_parallel(const char *b, const char *e, long Z, std::vector<int> &I, std::vector<int> &J,
                            std::vector<double> &val) {
    const int T = std::max(1, omp_get_max_threads());
    const int P = 4 * T;
    std::vector<const char *> cut(P + 1);
    cut[0] = b;
    cut[P] = e;
    for (int q = 1; q < P; ++q) {
        const char *c = b + (size_t)(e - b) * q / P;
        if (c < cut[q - 1]) c = cut[q - 1];
        while (c < e && c[-1] != '\n') c++;
        cut[q] = c;
    }
    struct Piece {
        std::vector<int> ij;   // row, col pairs; 0 stands for a value outside 1..INT_MAX
        std::vector<double> v;
        bool ok = true;
    };
    std::vector<Piece> pc(P);
#pragma omp parallel for schedule(dynamic, 1) num_threads(T)
    for (int q = 0; q < P; ++q) {
        Piece &k = pc[q];
        const char *p = cut[q], *end = cut[q + 1];
        size_t lines = 1;   // one entry per line, as written: sizes the piece's arrays
        for (const char *c = p; (c = static_cast<const char *>(std::memchr(c, '\n', end - c))); ++c) lines++;
        k.ij.reserve(2 * lines);
        k.v.reserve(lines);
        auto as_index = [](long a) { return (a < 1 || a > 0x7fffffffL) ? 0 : (int)a; };
        for (;;) {
            skip_space(p, end);
            if (p >= end) break;
            long a = 0, c = 0;
            double x = 0.0;
            if (!tok_integer(p, end, a) || !tok_integer(p, end, c) || !tok_real(p, end, x) ||
                (p < end && !is_space(*p))) {
                k.ok = false;
                break;
            }
            k.ij.push_back(as_index(a));
            k.ij.push_back(as_index(c));
            k.v.push_back(x);
        }
    }
    std::vector<long> at(P + 1, 0);
    for (int q = 0; q < P; ++q) {
        if (!pc[q].ok) return false;
        at[q + 1] = at[q] + (long)pc[q].v.size();
    }
    if (at[P] < Z) return false;
#pragma omp parallel for schedule(dynamic, 1) num_threads(T)
    for (int q = 0; q < P; ++q) {
        const long lo = at[q], hi = std::min(at[q + 1], Z);
        for (long k = lo; k < hi; ++k) {
            I[k] = pc[q].ij[2 * (k - lo)];
            J[k] = pc[q].ij[2 * (k - lo) + 1];
            val[k] = pc[q].v[k - lo];
        }
    }
    return true;
}

int slurp(const char *path, std::string &out) {
    std::FILE *f = std::fopen(path, "rb");
    if (!f) return fiim::set_error(FIIM_EARG, "file %s does not exist", path);
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    const size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if ((long)got != sz) return fiim::set_error(FIIM_EARG, "could not read %s", path);
    return FIIM_OK;
}

std::string lower(std::string s) {
    for (char &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Banner words: object, format, field, symmetry. Returns FIIM_OK or FIIM_EARG.
int banner(Reader &rd, std::string w[4]) {
    std::string l;
    if (!rd.line(l)) return fiim::set_error(FIIM_EARG, "empty file");
    char a[64] = {0}, b[64] = {0}, c[64] = {0}, d[64] = {0}, e[64] = {0};
    if (std::sscanf(l.c_str(), "%63s %63s %63s %63s %63s", a, b, c, d, e) != 5 ||
        std::string(a) != "%%MatrixMarket")
        return fiim::set_error(FIIM_EARG, "could not process the Matrix Market banner");
    w[0] = lower(b);
    w[1] = lower(c);
    w[2] = lower(d);
    w[3] = lower(e);
    if (w[0] != "matrix") return fiim::set_error(FIIM_EARG, "Matrix Market object '%s' is not a matrix", b);
    return FIIM_OK;
}

void skip_comments(Reader &rd) {
    while (rd.pos < rd.text.size()) {
        size_t p = rd.pos;
        while (p < rd.text.size() && (rd.text[p] == ' ' || rd.text[p] == '\t')) p++;
        if (p < rd.text.size() && (rd.text[p] == '%' || rd.text[p] == '\n' || rd.text[p] == '\r')) {
            std::string dummy;
            rd.line(dummy);
        } else {
            break;
        }
    }
}

}  // namespace

extern "C" {

int fiim_read_mtx(const char *path, int form, int *n, int *nnz, int *issym, int *Ai, int *Aj, double *Av) {
    if (!n || !nnz) return fiim::set_error(FIIM_EARG, "n and nnz are required");
    if (Ai) {   // second call: copy out the matrix the first call read
        if (g_mtx.rp.empty()) return fiim::set_error(FIIM_EARG, "no matrix was read on this thread");
        if (*n != g_mtx.n || *nnz != (int)g_mtx.ci.size())
            return fiim::set_error(FIIM_EARG, "sizes differ from the ones the first call returned");
        std::memcpy(Ai, g_mtx.rp.data(), sizeof(int) * (g_mtx.n + 1));
        if (Aj) std::memcpy(Aj, g_mtx.ci.data(), sizeof(int) * g_mtx.ci.size());
        if (Av) std::memcpy(Av, g_mtx.v.data(), sizeof(double) * g_mtx.v.size());
        if (issym) *issym = g_mtx.issym;
        g_mtx = MtxBuf{};
        return FIIM_OK;
    }
    if (!path) return fiim::set_error(FIIM_EARG, "path is required");
    if (form != 0 && form != 1) return fiim::set_error(FIIM_EARG, "form is 0 (AFIIM/ACIFIM) or 1 (PDFIIM)");
    Reader rd;
    int rc = slurp(path, rd.text);
    if (rc != FIIM_OK) return rc;
    std::string w[4];
    if ((rc = banner(rd, w)) != FIIM_OK) return rc;
    // AFIIM/src/rw_matrix.cpp:98-104: only real coordinate matrices, general or symmetric.
    if (w[1] != "coordinate" || w[2] != "real" || (w[3] != "general" && w[3] != "symmetric"))
        return fiim::set_error(FIIM_EARG, "Matrix Market type [%s %s %s] is not supported (real coordinate "
                                          "general or symmetric only)", w[1].c_str(), w[2].c_str(), w[3].c_str());
    const bool sym = (w[3] == "symmetric");
    skip_comments(rd);
    long M = 0, N = 0, Z = 0;
    if (!rd.integer(M) || !rd.integer(N) || !rd.integer(Z) || M <= 0 || N <= 0 || Z < 0)
        return fiim::set_error(FIIM_EARG, "problem at reading dimensions and nonzero elements");
    if (M != N) return fiim::set_error(FIIM_EARG, "matrix is not square");
    if (M > 0x7ffffffeL || Z > 0x3fffffffL) return fiim::set_error(FIIM_EARG, "matrix too large for int32 CSR");
    std::vector<int> I(Z), J(Z);
    std::vector<double> val(Z);
    bool par = Z >= kParallelEntries &&
               parse_entries_parallel(rd.text.data() + rd.pos, rd.text.data() + rd.text.size(), Z, I, J, val);
    if (par) {
        bool ok = true;
#pragma omp parallel for reduction(&& : ok)
        for (long k = 0; k < Z; ++k) {
            const int a = I[k], b = J[k];
            if (a < 1 || a > M || b < 1 || b > N) {
                ok = false;
            } else if (sym && form == 1) {
                I[k] = b - 1;
                J[k] = a - 1;
            } else {
                I[k] = a - 1;
                J[k] = b - 1;
            }
        }
        par = ok;   // otherwise the one-thread reader below reports the first bad entry
    }
    for (long k = 0; !par && k < Z; ++k) {
        long a = 0, b = 0;
        double x = 0.0;
        if (!rd.integer(a) || !rd.integer(b) || !rd.real(x))
            return fiim::set_error(FIIM_EARG, "entry %ld is malformed", k + 1);
        if (a < 1 || a > M || b < 1 || b > N)
            return fiim::set_error(FIIM_EARG, "entry %ld (%ld, %ld) is outside the %ld x %ld matrix", k + 1, a, b, M, N);
        if (sym && form == 1) {   // PDFIIM/src/rw_matrix.cpp:108-113: read as (col, row)
            I[k] = (int)b - 1;
            J[k] = (int)a - 1;
        } else {
            I[k] = (int)a - 1;
            J[k] = (int)b - 1;
        }
        val[k] = x;
    }
    if (sym && form == 0) {   // AFIIM/src/rw_matrix.cpp:144-183: append the mirror entries
        const long z0 = Z;
        for (long k = 0; k < z0; ++k)
            if (I[k] != J[k]) {
                I.push_back(J[k]);
                J.push_back(I[k]);
                val.push_back(val[k]);
            }
        Z = (long)I.size();
        if (Z > 0x3fffffffL) return fiim::set_error(FIIM_EARG, "matrix too large for int32 CSR");
    }
    MtxBuf m;
    m.n = (int)N;
    m.issym = (sym && form == 1) ? 1 : 0;
    m.rp.assign(N + 1, 0);
    m.ci.resize(Z);
    m.v.resize(Z);
    for (long k = 0; k < Z; ++k) m.rp[I[k] + 1]++;                 // counts
    for (long i = 0; i < N; ++i) m.rp[i + 1] += m.rp[i];           // offsets
    std::vector<int> next(m.rp.begin(), m.rp.end() - 1);
    for (long k = 0; k < Z; ++k) {                                 // bucket in input order
        const int at = next[I[k]]++;
        m.ci[at] = J[k];
        m.v[at] = val[k];
    }
#pragma omp parallel for schedule(dynamic, 4096) if (Z >= kParallelEntries)
    for (long i = 0; i < N; ++i)
        if (m.rp[i + 1] - 1 > m.rp[i]) qsort_pairs(m.ci.data(), m.v.data(), m.rp[i], m.rp[i + 1] - 1);
    *n = m.n;
    *nnz = (int)Z;
    if (issym) *issym = m.issym;
    g_mtx = std::move(m);
    return FIIM_OK;
}

int fiim_read_rhs(const char *path, int cap, double *b, int *n) {
    if (!path || !n) return fiim::set_error(FIIM_EARG, "path and n are required");
    Reader rd;
    int rc = slurp(path, rd.text);
    if (rc != FIIM_OK) return rc;
    std::string w[4];
    if ((rc = banner(rd, w)) != FIIM_OK) return rc;
    // AFIIM/src/rw_matrix.cpp:266-272: a real general dense (array) vector.
    if (w[1] != "array" || w[2] != "real" || w[3] != "general")
        return fiim::set_error(FIIM_EARG, "Matrix Market type [%s %s %s] is not a real general array",
                               w[1].c_str(), w[2].c_str(), w[3].c_str());
    skip_comments(rd);
    long M = 0, N = 0;
    if (!rd.integer(M) || !rd.integer(N) || M < 0) return fiim::set_error(FIIM_EARG, "problem at reading dimensions");
    if (N != 1) return fiim::set_error(FIIM_EARG, "the input file does not contain a vector");
    *n = (int)M;
    if (!b) return FIIM_OK;   // size query
    if (M > cap) return fiim::set_error(FIIM_EARG, "vector has %ld entries, room for %d", M, cap);
    for (long i = 0; i < M; ++i)
        if (!rd.real(b[i])) return fiim::set_error(FIIM_EARG, "entry %ld is malformed", i + 1);
    return FIIM_OK;
}

// ---------------------------------------------------------------- binary factor file
// Layout (little-endian): 8-byte magic "FIIMFAC1"; int64 n, nnz(G), nnz(H); then Gi[n+1],
// Gj[nnzG] (int32), Gv[nnzG] (f64), IDv[n] (f64), Hi[n+1], Hj[nnzH] (int32), Hv[nnzH] (f64);
// then a 64-bit checksum of everything after the magic (the same mixing sum the drop-in
// cache uses for its stamps: splitmix64-mixed 8-byte words tagged by position).

namespace {

inline uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

struct Sum {
    uint64_t acc = 0, words = 0;
    unsigned char tail[8];
    int nt = 0;
    void add(const void *p, size_t bytes) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        for (size_t k = 0; k < bytes; ++k) {
            tail[nt++] = c[k];
            if (nt == 8) {
                uint64_t w;
                std::memcpy(&w, tail, 8);
                acc += mix64(w ^ (0x9e3779b97f4a7c15ULL * ++words));
                nt = 0;
            }
        }
    }
    uint64_t value() const {
        uint64_t w = 0;
        std::memcpy(&w, tail, (size_t)nt);
        return acc + mix64(w ^ 0xd1b54a32d192ed03ULL) + mix64(words * 8 + (uint64_t)nt);
    }
};

struct FacBuf {
    long n = 0;
    std::vector<int> Gi, Gj, Hi, Hj;
    std::vector<double> Gv, Hv, IDv;
};
thread_local FacBuf g_fac;

}  // namespace

int fiim_factors_save(const char *path, int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                      const int *Hi, const int *Hj, const double *Hv) {
    if (!path || n <= 0 || !Gi || !Gj || !Gv || !IDv || !Hi || !Hj || !Hv)
        return fiim::set_error(FIIM_EARG, "null argument or n <= 0");
    const int64_t hdr[3] = {n, Gi[n], Hi[n]};
    if (hdr[1] < 0 || hdr[2] < 0) return fiim::set_error(FIIM_EARG, "negative entry count");
    std::FILE *f = std::fopen(path, "wb");
    if (!f) return fiim::set_error(FIIM_EARG, "cannot open %s for writing", path);
    Sum sum;
    bool ok = std::fwrite("FIIMFAC1", 1, 8, f) == 8;
    auto put = [&](const void *p, size_t bytes) {
        if (!ok || bytes == 0) return;
        ok = std::fwrite(p, 1, bytes, f) == bytes;
        sum.add(p, bytes);
    };
    put(hdr, sizeof hdr);
    put(Gi, sizeof(int) * (n + 1));
    put(Gj, sizeof(int) * hdr[1]);
    put(Gv, sizeof(double) * hdr[1]);
    put(IDv, sizeof(double) * n);
    put(Hi, sizeof(int) * (n + 1));
    put(Hj, sizeof(int) * hdr[2]);
    put(Hv, sizeof(double) * hdr[2]);
    const uint64_t cs = sum.value();
    ok = ok && std::fwrite(&cs, 1, 8, f) == 8;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fiim::set_error(FIIM_EARG, "writing %s failed", path);
    return FIIM_OK;
}

int fiim_factors_load(const char *path, int *n, int *nnzG, int *nnzH, int *Gi, int *Gj, double *Gv, double *IDv,
                      int *Hi, int *Hj, double *Hv) {
    if (!n || !nnzG || !nnzH) return fiim::set_error(FIIM_EARG, "n, nnzG and nnzH are required");
    if (Gi) {   // second call: copy out the factors the first call read
        if (g_fac.n == 0) return fiim::set_error(FIIM_EARG, "no factor file was read on this thread");
        if (*n != g_fac.n || *nnzG != (int)g_fac.Gj.size() || *nnzH != (int)g_fac.Hj.size())
            return fiim::set_error(FIIM_EARG, "sizes differ from the ones the first call returned");
        if (!Gj || !Gv || !IDv || !Hi || !Hj || !Hv) return fiim::set_error(FIIM_EARG, "null output array");
        std::memcpy(Gi, g_fac.Gi.data(), sizeof(int) * g_fac.Gi.size());
        std::memcpy(Gj, g_fac.Gj.data(), sizeof(int) * g_fac.Gj.size());
        std::memcpy(Gv, g_fac.Gv.data(), sizeof(double) * g_fac.Gv.size());
        std::memcpy(IDv, g_fac.IDv.data(), sizeof(double) * g_fac.IDv.size());
        std::memcpy(Hi, g_fac.Hi.data(), sizeof(int) * g_fac.Hi.size());
        std::memcpy(Hj, g_fac.Hj.data(), sizeof(int) * g_fac.Hj.size());
        std::memcpy(Hv, g_fac.Hv.data(), sizeof(double) * g_fac.Hv.size());
        g_fac = FacBuf{};
        return FIIM_OK;
    }
    if (!path) return fiim::set_error(FIIM_EARG, "path is required");
    std::FILE *f = std::fopen(path, "rb");
    if (!f) return fiim::set_error(FIIM_EARG, "file %s does not exist", path);
    char magic[8];
    int64_t hdr[3];
    Sum sum;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "FIIMFAC1", 8) == 0;
    if (!ok) {
        std::fclose(f);
        return fiim::set_error(FIIM_EARG, "%s is not a factor file", path);
    }
    auto get = [&](void *p, size_t bytes) {
        if (!ok || bytes == 0) return;
        ok = std::fread(p, 1, bytes, f) == bytes;
        if (ok) sum.add(p, bytes);
    };
    get(hdr, sizeof hdr);
    if (!ok || hdr[0] <= 0 || hdr[0] > 0x7ffffffeL || hdr[1] < 0 || hdr[1] > 0x7fffffffL || hdr[2] < 0 ||
        hdr[2] > 0x7fffffffL) {
        std::fclose(f);
        return fiim::set_error(FIIM_EARG, "%s has a damaged header", path);
    }
    FacBuf b;
    b.n = hdr[0];
    b.Gi.resize(b.n + 1);
    b.Gj.resize(hdr[1]);
    b.Gv.resize(hdr[1]);
    b.IDv.resize(b.n);
    b.Hi.resize(b.n + 1);
    b.Hj.resize(hdr[2]);
    b.Hv.resize(hdr[2]);
    get(b.Gi.data(), sizeof(int) * b.Gi.size());
    get(b.Gj.data(), sizeof(int) * b.Gj.size());
    get(b.Gv.data(), sizeof(double) * b.Gv.size());
    get(b.IDv.data(), sizeof(double) * b.IDv.size());
    get(b.Hi.data(), sizeof(int) * b.Hi.size());
    get(b.Hj.data(), sizeof(int) * b.Hj.size());
    get(b.Hv.data(), sizeof(double) * b.Hv.size());
    uint64_t cs = 0;
    ok = ok && std::fread(&cs, 1, 8, f) == 8;
    std::fclose(f);
    if (!ok) return fiim::set_error(FIIM_EARG, "%s is truncated", path);
    if (cs != sum.value()) return fiim::set_error(FIIM_EARG, "%s fails its checksum", path);
    if (b.Gi[0] != 0 || b.Gi[b.n] != hdr[1] || b.Hi[0] != 0 || b.Hi[b.n] != hdr[2])
        return fiim::set_error(FIIM_EARG, "%s has inconsistent row offsets", path);
    *n = (int)b.n;
    *nnzG = (int)hdr[1];
    *nnzH = (int)hdr[2];
    g_fac = std::move(b);
    return FIIM_OK;
}

}  // extern "C"
