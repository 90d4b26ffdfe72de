// mmio.cu - Matrix Market reader of the host-buffer drop-ins (host code only).
//
// Semantics of the reference's mmio_allinone (src/mmio_highlevel.h:593-760),
// which its benchmark uses to load SuiteSparse inputs: a coordinate file
// becomes CSR with 0-based indices; pattern entries get 1.0, integer entries
// their value, complex entries their real part; a symmetric or hermitian file
// also stores every off-diagonal entry (i, j) at (j, i) with the same value.
// Entries are neither sorted nor merged: a row holds its entries in file
// order, and for symmetric files an entry's mirror is placed when the entry
// is read, so the rows interleave the two.  Unlike the reference, every
// index is checked against the declared shape and every short or unreadable
// line is an error (the reference reads on regardless).  value_mode 1 gives
// entry i (in CSR order) the value i % 10, as the reference's load_matrix
// does after reading (src/main.cu:1109-1110).
#include "rtt_internal.cuh"

#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace
{

struct File
{
    FILE *f = nullptr;
    ~File()
    {
        if (f != nullptr)
            std::fclose(f);
    }
};

// next line into buf (without the newline); false at end of file
bool next_line(FILE *f, std::string &buf)
{
    buf.clear();
    int ch;
    while ((ch = std::fgetc(f)) != EOF && ch != '\n')
        buf.push_back((char)ch);
    return ch != EOF || !buf.empty();
}

std::string lower(std::string s)
{
    for (char &c : s)
        c = (char)std::tolower((unsigned char)c);
    return s;
}

} // namespace

extern "C" {

int rtt_mmio_read(const char *path, int value_mode, SMatrix *out)
{
    using rtt::fail;
    if (path == nullptr || out == nullptr || value_mode < 0 || value_mode > 1)
        return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: bad arguments");
    File file;
    file.f = std::fopen(path, "r");
    if (file.f == nullptr)
        return fail(RTT_ERR_INVALID_ARGUMENT, std::string("mmio_read: cannot open ") + path);
    std::string line;
    if (!next_line(file.f, line))
        return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: empty file");
    char t[5][64] = {};
    if (std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", t[0], t[1], t[2], t[3], t[4]) != 5 ||
        std::strcmp(t[0], "%%MatrixMarket") != 0)
        return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: no Matrix Market banner");
    const std::string object = lower(t[1]), format = lower(t[2]), field = lower(t[3]),
                      symmetry = lower(t[4]);
    if (object != "matrix" || format != "coordinate")
        return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: only coordinate matrices are read");
    const bool pattern = field == "pattern", complex_ = field == "complex",
               integer = field == "integer", real = field == "real" || field == "double";
    if (!pattern && !complex_ && !integer && !real)
        return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: unknown field " + field);
    const bool mirror = symmetry == "symmetric" || symmetry == "hermitian";
    if (!mirror && symmetry != "general" && symmetry != "skew-symmetric")
        return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: unknown symmetry " + symmetry);
    // size line after the comments
    long long m = 0, n = 0, stored = 0;
    for (;;)
    {
        if (!next_line(file.f, line))
            return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: no size line");
        if (!line.empty() && line[0] == '%')
            continue;
        if (std::sscanf(line.c_str(), "%lld %lld %lld", &m, &n, &stored) == 3)
            break;
        if (line.find_first_not_of(" \t\r") != std::string::npos)
            return fail(RTT_ERR_INVALID_ARGUMENT, "mmio_read: bad size line");
    }
    if (m < 0 || n < 0 || stored < 0 || m > INT_MAX - 1 || n > INT_MAX || stored > INT_MAX)
        return fail(RTT_ERR_UNREPRESENTABLE, "mmio_read: shape beyond int32");
    std::vector<int> ri((size_t)stored), ci((size_t)stored);
    std::vector<double> vv((size_t)stored);
    std::vector<long long> cnt((size_t)m + 1, 0);
    for (long long i = 0; i < stored; ++i)
    {
        if (!next_line(file.f, line))
            return fail(RTT_ERR_INVALID_CSR, "mmio_read: fewer entries than declared");
        const char *p = line.c_str();
        char *end = nullptr;
        errno = 0;
        const long long r = std::strtoll(p, &end, 10);
        if (end == p)
        {
            if (line.find_first_not_of(" \t\r") == std::string::npos)
            {
                --i; // blank line between entries
                continue;
            }
            return fail(RTT_ERR_INVALID_CSR, "mmio_read: unreadable entry line");
        }
        p = end;
        const long long c = std::strtoll(p, &end, 10);
        if (end == p)
            return fail(RTT_ERR_INVALID_CSR, "mmio_read: unreadable entry line");
        p = end;
        double v = 1.0;
        if (!pattern)
        {
            v = std::strtod(p, &end); // real part for complex entries
            if (end == p)
                return fail(RTT_ERR_INVALID_CSR, "mmio_read: entry without a value");
        }
        if (r < 1 || r > m || c < 1 || c > n)
            return fail(RTT_ERR_INVALID_CSR, "mmio_read: entry outside the declared shape");
        ri[(size_t)i] = (int)(r - 1);
        ci[(size_t)i] = (int)(c - 1);
        vv[(size_t)i] = v;
        cnt[(size_t)(r - 1)]++;
        if (mirror && r != c)
        {
            if (c - 1 >= m)
                return fail(RTT_ERR_INVALID_CSR, "mmio_read: symmetric entry outside a square");
            cnt[(size_t)(c - 1)]++;
        }
    }
    // exclusive scan into the row pointer
    long long total = 0;
    for (long long r = 0; r <= m; ++r)
    {
        const long long k = cnt[(size_t)r];
        cnt[(size_t)r] = total;
        total += k;
    }
    if (total > INT_MAX)
        return fail(RTT_ERR_UNREPRESENTABLE, "mmio_read: more than INT32_MAX entries");
    int *rp = static_cast<int *>(std::malloc(sizeof(int) * ((size_t)m + 1)));
    int *col = static_cast<int *>(std::malloc(sizeof(int) * (size_t)(total > 0 ? total : 1)));
    double *val = static_cast<double *>(std::malloc(sizeof(double) * (size_t)(total > 0 ? total : 1)));
    if (rp == nullptr || col == nullptr || val == nullptr)
    {
        std::free(rp);
        std::free(col);
        std::free(val);
        return fail(RTT_ERR_OUT_OF_MEMORY, "mmio_read: host malloc failed");
    }
    for (long long r = 0; r <= m; ++r)
        rp[r] = (int)cnt[(size_t)r];
    // entries (and their mirrors) in file order
    std::vector<long long> fill(cnt.begin(), cnt.end());
    for (long long i = 0; i < stored; ++i)
    {
        const int r = ri[(size_t)i], c = ci[(size_t)i];
        long long at = fill[(size_t)r]++;
        col[at] = c;
        val[at] = vv[(size_t)i];
        if (mirror && r != c)
        {
            at = fill[(size_t)c]++;
            col[at] = r;
            val[at] = vv[(size_t)i];
        }
    }
    if (value_mode == 1)
        for (long long i = 0; i < total; ++i)
            val[i] = (double)(i % 10);
    std::memset(out, 0, sizeof(*out));
    out->m = (int)m;
    out->n = (int)n;
    out->nnz = (int)total;
    out->isSymmetric = mirror ? 1 : 0;
    out->rowpointer = rp;
    out->columnindex = col;
    out->value = val;
    return RTT_OK;
}

} // extern "C"
