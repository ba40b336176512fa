// Matrix Market input (clsparseHeaderfromFile, clsparse{S,D}{Coo,Csr}MatrixfromFile
// and the host-side clsparseB200ReadMatrixMarketHost), following the
// reference reader's behaviour (src/library/io/mm-reader.cpp:140-760):
//
// * only ".mtx" paths (otherwise clsparseInvalidFileFormat), only the
//   coordinate format with real, integer or pattern entries (array or complex
//   files, or a malformed banner, size line or entry: clsparseInvalidFile);
// * indices are 1-based in the file and 0-based in memory;
// * a "symmetric" file stores each off-diagonal entry once; it is mirrored
//   (mm-reader.cpp:225-255), and the header reports twice the stored count as
//   the capacity to allocate (mm-reader.cpp:189-191);
// * explicit zeros are dropped unless read_explicit_zeroes is set;
// * pattern entries get values in [0, 5) (the reference draws them with
//   rand(), mm-reader.cpp:306-308; here a fixed-seed generator, so a file
//   always loads to the same matrix);
// * entries are ordered by (row, column) (mm-reader.cpp:66-72, 637); the sort
//   is stable, so duplicate entries stay as separate entries in file order;
// * the CSR row pointer is built from the sorted rows (mm-reader.cpp:639-652).
//
// Device variants write into caller-allocated device buffers (sized from
// clsparseHeaderfromFile; a CUDA pointer carries no size to check, unlike the
// reference's cl_mem) with element offsets, then wait for the copies.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace clsp {
namespace {

struct MMHeader {
    bool symmetric = false;
    bool pattern = false;
    uint64_t rows = 0, cols = 0, stored = 0;
};

bool has_mtx_extension(const char* path) {
    if (!path) return false;
    const std::string s(path);
    const size_t dot = s.find_last_of('.');
    return dot != std::string::npos && s.substr(dot + 1) == "mtx";
}

std::string lower(std::string s) {
    for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return s;
}

// Reads the banner and size line; `rest` is left at the first entry line.
bool read_header(FILE* f, MMHeader& h) {
    char line[4096];
    if (!std::fgets(line, sizeof(line), f)) return false;
    char banner[64] = {}, object[64] = {}, format[64] = {}, field[64] = {}, sym[64] = {};
    if (std::sscanf(line, "%63s %63s %63s %63s %63s", banner, object, format, field, sym) != 5) return false;
    if (std::string(banner) != "%%MatrixMarket" || lower(object) != "matrix") return false;
    if (lower(format) != "coordinate") return false;
    const std::string fld = lower(field), sy = lower(sym);
    if (fld != "real" && fld != "double" && fld != "integer" && fld != "pattern") return false;
    if (sy != "general" && sy != "symmetric" && sy != "skew-symmetric" && sy != "hermitian") return false;
    h.pattern = fld == "pattern";
    h.symmetric = sy == "symmetric";
    // comments, then the size line
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '%') continue;
        bool blank = true;
        for (const char* p = line; *p; ++p)
            if (!std::isspace(static_cast<unsigned char>(*p))) blank = false;
        if (blank) continue;
        unsigned long long r = 0, c = 0, z = 0;
        if (std::sscanf(line, "%llu %llu %llu", &r, &c, &z) != 3) return false;
        h.rows = r;
        h.cols = c;
        h.stored = z;
        return true;
    }
    return false;
}

template <typename T>
struct Entry {
    uint32_t r, c;
    T v;
};

// SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014), for the values of pattern entries.
struct Mix64 {
    uint64_t s = 0x2545F4914F6CDD1Dull;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

template <typename T>
clsparseStatus read_entries(const char* path, bool keep_zeros, MMHeader& h, std::vector<Entry<T>>& out) {
    if (!has_mtx_extension(path)) return clsparseInvalidFileFormat;
    FILE* f = std::fopen(path, "r");
    if (!f) return clsparseInvalidFile;
    if (!read_header(f, h) || h.rows > 0xFFFFFFFFull || h.cols > 0xFFFFFFFFull) {
        std::fclose(f);
        return clsparseInvalidFile;
    }
    out.clear();
    out.reserve(h.symmetric ? 2 * h.stored : h.stored);
    Mix64 rng;
    char line[4096];
    uint64_t read = 0;
    while (read < h.stored && std::fgets(line, sizeof(line), f)) {
        char* p = line;
        while (std::isspace(static_cast<unsigned char>(*p))) ++p;
        if (*p == '\0' || *p == '%') continue;
        char* e = nullptr;
        const unsigned long long i = std::strtoull(p, &e, 10);
        if (e == p) break;
        p = e;
        const unsigned long long j = std::strtoull(p, &e, 10);
        if (e == p) break;
        p = e;
        T v;
        if (h.pattern) {
            v = static_cast<T>(5.0 * rng.uniform());
        } else {
            if constexpr (sizeof(T) == 4)
                v = std::strtof(p, &e);
            else
                v = std::strtod(p, &e);
            if (e == p) break;
        }
        ++read;
        if (i < 1 || j < 1 || i > h.rows || j > h.cols) {
            std::fclose(f);
            return clsparseInvalidFile;
        }
        if (!keep_zeros && v == T(0)) continue;
        out.push_back({static_cast<uint32_t>(i - 1), static_cast<uint32_t>(j - 1), v});
        if (h.symmetric && i != j) out.push_back({static_cast<uint32_t>(j - 1), static_cast<uint32_t>(i - 1), v});
    }
    std::fclose(f);
    if (read != h.stored) return clsparseInvalidFile;
    std::stable_sort(out.begin(), out.end(), [](const Entry<T>& a, const Entry<T>& b) {
        return a.r != b.r ? a.r < b.r : a.c < b.c;
    });
    return clsparseSuccess;
}

template <typename T>
void to_csr(const std::vector<Entry<T>>& en, uint32_t nrows, std::vector<uint32_t>& rp, std::vector<uint32_t>& col,
            std::vector<T>& val) {
    rp.assign(static_cast<size_t>(nrows) + 1, 0);
    col.resize(en.size());
    val.resize(en.size());
    for (size_t k = 0; k < en.size(); ++k) {
        ++rp[en[k].r + 1];
        col[k] = en[k].c;
        val[k] = en[k].v;
    }
    for (uint32_t r = 0; r < nrows; ++r) rp[r + 1] += rp[r];
}

clsparseStatus upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return clsparseSuccess;
    if (!dst) return clsparseInvalidMemObject;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) == cudaSuccess ? clsparseSuccess
                                                                                      : clsparseInvalidMemObject;
}

template <typename T>
clsparseStatus csr_from_file(clsparseCsrMatrix* m, const char* path, clsparseControl control, cl_bool keep) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!m) return clsparseInvalidValue;
    MMHeader h;
    std::vector<Entry<T>> en;
    st = read_entries<T>(path, keep != 0, h, en);
    if (st != clsparseSuccess) return st;
    std::vector<uint32_t> rp, col;
    std::vector<T> val;
    to_csr(en, static_cast<uint32_t>(h.rows), rp, col, val);
    DeviceGuard g(control->device);
    m->num_rows = static_cast<clsparseIdx_t>(h.rows);
    m->num_cols = static_cast<clsparseIdx_t>(h.cols);
    m->num_nonzeros = static_cast<clsparseIdx_t>(en.size());
    cudaStream_t s = control->stream;
    if ((st = upload(dev_ptr<T>(m->values, m->off_values), val.data(), val.size() * sizeof(T), s)) != clsparseSuccess ||
        (st = upload(dev_ptr<uint32_t>(m->col_indices, m->off_col_indices), col.data(), col.size() * 4, s)) !=
            clsparseSuccess ||
        (st = upload(dev_ptr<uint32_t>(m->row_pointer, m->off_row_pointer), rp.data(), rp.size() * 4, s)) !=
            clsparseSuccess)
        return st;
    return cudaStreamSynchronize(s) == cudaSuccess ? clsparseSuccess : clsparseInvalidMemObject;
}

template <typename T>
clsparseStatus coo_from_file(clsparseCooMatrix* m, const char* path, clsparseControl control, cl_bool keep) {
    clsparseStatus st = check_entry(control);
    if (st != clsparseSuccess) return st;
    if (!m) return clsparseInvalidValue;
    MMHeader h;
    std::vector<Entry<T>> en;
    st = read_entries<T>(path, keep != 0, h, en);
    if (st != clsparseSuccess) return st;
    std::vector<uint32_t> ri(en.size()), ci(en.size());
    std::vector<T> val(en.size());
    for (size_t k = 0; k < en.size(); ++k) {
        ri[k] = en[k].r;
        ci[k] = en[k].c;
        val[k] = en[k].v;
    }
    DeviceGuard g(control->device);
    m->num_rows = static_cast<clsparseIdx_t>(h.rows);
    m->num_cols = static_cast<clsparseIdx_t>(h.cols);
    m->num_nonzeros = static_cast<clsparseIdx_t>(en.size());
    cudaStream_t s = control->stream;
    if ((st = upload(dev_ptr<T>(m->values, m->off_values), val.data(), val.size() * sizeof(T), s)) != clsparseSuccess ||
        (st = upload(dev_ptr<uint32_t>(m->col_indices, m->off_col_indices), ci.data(), ci.size() * 4, s)) !=
            clsparseSuccess ||
        (st = upload(dev_ptr<uint32_t>(m->row_indices, m->off_row_indices), ri.data(), ri.size() * 4, s)) !=
            clsparseSuccess)
        return st;
    return cudaStreamSynchronize(s) == cudaSuccess ? clsparseSuccess : clsparseInvalidMemObject;
}

}  // namespace
}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus clsparseHeaderfromFile(clsparseIdx_t* nnz, clsparseIdx_t* row, clsparseIdx_t* col,
                                      const char* filePath) {
    if (!nnz || !row || !col) return clsparseInvalidValue;
    if (!has_mtx_extension(filePath)) return clsparseInvalidFileFormat;
    FILE* f = std::fopen(filePath, "r");
    if (!f) return clsparseInvalidFile;
    MMHeader h;
    const bool ok = read_header(f, h);
    std::fclose(f);
    if (!ok || h.rows > 0xFFFFFFFFull || h.cols > 0xFFFFFFFFull) return clsparseInvalidFile;
    *row = static_cast<clsparseIdx_t>(h.rows);
    *col = static_cast<clsparseIdx_t>(h.cols);
    *nnz = static_cast<clsparseIdx_t>(h.symmetric ? 2 * h.stored : h.stored);
    return clsparseSuccess;
}

clsparseStatus clsparseSCooMatrixfromFile(clsparseCooMatrix* cooMatx, const char* filePath, clsparseControl control,
                                          cl_bool read_explicit_zeroes) {
    return coo_from_file<float>(cooMatx, filePath, control, read_explicit_zeroes);
}

clsparseStatus clsparseDCooMatrixfromFile(clsparseCooMatrix* cooMatx, const char* filePath, clsparseControl control,
                                          cl_bool read_explicit_zeroes) {
    return coo_from_file<double>(cooMatx, filePath, control, read_explicit_zeroes);
}

clsparseStatus clsparseSCsrMatrixfromFile(clsparseCsrMatrix* csrMatx, const char* filePath, clsparseControl control,
                                          cl_bool read_explicit_zeroes) {
    return csr_from_file<float>(csrMatx, filePath, control, read_explicit_zeroes);
}

clsparseStatus clsparseDCsrMatrixfromFile(clsparseCsrMatrix* csrMatx, const char* filePath, clsparseControl control,
                                          cl_bool read_explicit_zeroes) {
    return csr_from_file<double>(csrMatx, filePath, control, read_explicit_zeroes);
}

clsparseStatus clsparseB200ReadMatrixMarketHost(const char* filePath, cl_bool read_explicit_zeroes,
                                                clsparseIdx_t* numRows, clsparseIdx_t* numCols,
                                                clsparseIdx_t* numNonzeros, clsparseIdx_t* rowPointer,
                                                clsparseIdx_t* colIndices, cl_double* values, size_t capacity) {
    if (!numRows || !numCols || !numNonzeros) return clsparseInvalidValue;
    MMHeader h;
    std::vector<Entry<double>> en;
    const clsparseStatus st = read_entries<double>(filePath, read_explicit_zeroes != 0, h, en);
    if (st != clsparseSuccess) return st;
    *numRows = static_cast<clsparseIdx_t>(h.rows);
    *numCols = static_cast<clsparseIdx_t>(h.cols);
    *numNonzeros = static_cast<clsparseIdx_t>(en.size());
    if (!rowPointer || !colIndices || !values) return clsparseSuccess;  // sizes only
    if (capacity < en.size()) return clsparseInsufficientMemory;
    std::vector<uint32_t> rp, col;
    std::vector<double> val;
    to_csr(en, static_cast<uint32_t>(h.rows), rp, col, val);
    std::copy(rp.begin(), rp.end(), rowPointer);
    std::copy(col.begin(), col.end(), colIndices);
    std::copy(val.begin(), val.end(), values);
    return clsparseSuccess;
}

}  // extern "C"
