// mtx.cu -- Matrix Market ingestion and COO -> CRS (smax_utils_read_mtx,
// smax_utils_convert_coo_to_crs, include/smax_b200.h).
//
// Reference: the examples' matrix reader, COOMatrix::read_from_mtx without
// fast_matrix_market (examples/matrix_structs.hpp:52-180, examples/mmio.cpp)
// and CRSMatrix::convert_coo_to_crs (matrix_structs.hpp:338-387):
//   * banner "%%MatrixMarket matrix coordinate <data> <storage>" (tokens after
//     the first compared in lower case, mmio.cpp:56-136); accepted: data real,
//     integer or pattern, storage general or symmetric (matrix_structs.hpp:
//     101-107); comment lines start with '%'; the size line holds M N nz;
//   * entries "i j v" (1-based; pattern entries "i j" get the value 0.01,
//     mmio.hpp:183-189), read in file order;
//   * symmetric files: every off-diagonal (i, j, v) is followed by (j, i, v)
//     (matrix_structs.hpp:127-138);
//   * a stable sort of the entries by row only -- within a row the file order
//     is kept (sort_perm, examples/permutation_helpers.hpp:1-11) -- then the
//     row pointer by counting.
// The text is parsed on the host by one thread per slice of the file (each
// slice starts at a line boundary; the slices' entries are concatenated in
// file order); integers are read as %d reads them, values with strtod (%lg).
// The sort, the gathers and the row pointer run on the GPU: a stable device
// radix sort of (row, position) pairs.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace smax {

namespace {

__global__ void iota_kernel(int *__restrict__ a, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] = (int)i;
}

// col/val in sorted order, row counts, and a range check of every index
template <typename VT>
__global__ void coo_gather_kernel(const int *__restrict__ perm, const int *__restrict__ I, const int *__restrict__ J,
                                  const double *__restrict__ V, int64_t nnz, int64_t n_rows, int64_t n_cols,
                                  int *__restrict__ col, VT *__restrict__ val, int *__restrict__ count,
                                  DevStatus *status) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
        const int k = perm[e];
        const int r = I[k], c = J[k];
        if (r < 0 || r >= n_rows) {
            report(status, SMAX_ERR_BAD_ARG, k);
            continue;
        }
        if (c < 0 || c >= n_cols) report(status, SMAX_ERR_COL_OOB, k);
        col[e] = c;
        val[e] = (VT)V[k];
        atomicAdd(count + r, 1);
    }
}

unsigned grid_of(int64_t n) {
    const int64_t cap = (int64_t)sm_count() * 8;
    int64_t g = (n + 255) / 256;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
}

void *host_new(size_t bytes) { return ::operator new[](bytes ? bytes : 1); }

// COO (host or device arrays, values as double) -> CRS host arrays (new[])
void coo_to_crs(int vbytes, int64_t n_rows, int64_t n_cols, int64_t nnz, const int *I, const int *J,
                const double *V, void **row_ptr, void **col, void **val) {
    if (nnz >= (int64_t(1) << 31) || n_rows >= (int64_t(1) << 31) || n_cols >= (int64_t(1) << 31))
        fail(SMAX_ERR_UNSUPPORTED, "int32 indices cannot address this matrix");
    cudaStream_t st = nullptr;
    SMAX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Close {
        cudaStream_t s;
        ~Close() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } close{st};
    const size_t nb = (size_t)(nnz > 0 ? nnz : 1);
    DevBuf dI(sizeof(int) * nb), dJ(sizeof(int) * nb), dV(sizeof(double) * nb), keys(sizeof(int) * nb),
        idx(sizeof(int) * nb), perm(sizeof(int) * nb), dcol(sizeof(int) * nb), dval((size_t)vbytes * nb),
        cnt(sizeof(int) * (n_rows + 1)), drp(sizeof(int) * (n_rows + 1)), status(sizeof(DevStatus));
    SMAX_CUDA(cudaMemsetAsync(status.p, 0, sizeof(DevStatus), st));
    SMAX_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (n_rows + 1), st));
    if (nnz > 0) {
        SMAX_CUDA(cudaMemcpyAsync(dI.p, I, sizeof(int) * nnz, cudaMemcpyDefault, st));
        SMAX_CUDA(cudaMemcpyAsync(dJ.p, J, sizeof(int) * nnz, cudaMemcpyDefault, st));
        SMAX_CUDA(cudaMemcpyAsync(dV.p, V, sizeof(double) * nnz, cudaMemcpyDefault, st));
        iota_kernel<<<grid_of(nnz), 256, 0, st>>>(idx.as<int>(), nnz);
        SMAX_CUDA(cudaGetLastError());
        // rows as unsigned keys: a negative row sorts last and is reported below
        size_t tb = 0;
        SMAX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, reinterpret_cast<unsigned *>(dI.p),
                                                  reinterpret_cast<unsigned *>(keys.p), idx.as<int>(),
                                                  perm.as<int>(), (int)nnz, 0, 32, st));
        DevBuf tmp(tb);
        SMAX_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, reinterpret_cast<unsigned *>(dI.p),
                                                  reinterpret_cast<unsigned *>(keys.p), idx.as<int>(),
                                                  perm.as<int>(), (int)nnz, 0, 32, st));
        if (vbytes == 8)
            coo_gather_kernel<double><<<grid_of(nnz), 256, 0, st>>>(perm.as<int>(), dI.as<int>(), dJ.as<int>(),
                                                                    dV.as<double>(), nnz, n_rows, n_cols,
                                                                    dcol.as<int>(), dval.as<double>(), cnt.as<int>(),
                                                                    status.as<DevStatus>());
        else
            coo_gather_kernel<float><<<grid_of(nnz), 256, 0, st>>>(perm.as<int>(), dI.as<int>(), dJ.as<int>(),
                                                                   dV.as<double>(), nnz, n_rows, n_cols,
                                                                   dcol.as<int>(), dval.as<float>(), cnt.as<int>(),
                                                                   status.as<DevStatus>());
        SMAX_CUDA(cudaGetLastError());
    }
    DevStatus hs{};
    SMAX_CUDA(cudaMemcpyAsync(&hs, status.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SMAX_CUDA(cudaStreamSynchronize(st));
    if (hs.code)
        fail(hs.code, std::string(hs.code == SMAX_ERR_COL_OOB ? "column" : "row") + " index out of range at entry " +
                          std::to_string(hs.index));
    SMAX_CUDA(cudaMemsetAsync(drp.p, 0, sizeof(int), st));
    if (n_rows > 0) {
        size_t tb = 0;
        SMAX_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, cnt.as<int>(), drp.as<int>() + 1, (int)n_rows, st));
        DevBuf tmp(tb);
        SMAX_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, cnt.as<int>(), drp.as<int>() + 1, (int)n_rows, st));
        SMAX_CUDA(cudaStreamSynchronize(st));
    }
    int *hrp = static_cast<int *>(host_new(sizeof(int) * (n_rows + 1)));
    int *hcol = static_cast<int *>(host_new(sizeof(int) * nnz));
    void *hval = host_new((size_t)vbytes * nnz);
    SMAX_CUDA(cudaMemcpyAsync(hrp, drp.p, sizeof(int) * (n_rows + 1), cudaMemcpyDeviceToHost, st));
    if (nnz > 0) {
        SMAX_CUDA(cudaMemcpyAsync(hcol, dcol.p, sizeof(int) * nnz, cudaMemcpyDeviceToHost, st));
        SMAX_CUDA(cudaMemcpyAsync(hval, dval.p, (size_t)vbytes * nnz, cudaMemcpyDeviceToHost, st));
    }
    SMAX_CUDA(cudaStreamSynchronize(st));
    *row_ptr = hrp;
    *col = hcol;
    *val = hval;
}

// ------------------------------------------------------------ text parsing --
struct Header {
    bool pattern = false, symmetric = false;
    long long M = 0, N = 0, nz = 0;
    size_t data_begin = 0;  // offset of the first entry
};

bool next_line(const std::string &s, size_t &pos, size_t &b, size_t &e) {
    if (pos >= s.size()) return false;
    b = pos;
    size_t nl = s.find('\n', pos);
    e = nl == std::string::npos ? s.size() : nl;
    pos = nl == std::string::npos ? s.size() : nl + 1;
    return true;
}

std::string lower(std::string t) {
    for (auto &c : t) c = (char)std::tolower((unsigned char)c);
    return t;
}

Header parse_header(const std::string &s) {
    Header h;
    size_t pos = 0, b = 0, e = 0;
    if (!next_line(s, pos, b, e)) fail(SMAX_ERR_BAD_ARG, "empty Matrix Market file");
    char tok[5][128] = {};
    const std::string first = s.substr(b, std::min<size_t>(e - b, 1023));
    if (std::sscanf(first.c_str(), "%127s %127s %127s %127s %127s", tok[0], tok[1], tok[2], tok[3], tok[4]) != 5)
        fail(SMAX_ERR_BAD_ARG, "could not process the Matrix Market banner");
    if (std::strncmp(tok[0], "%%MatrixMarket", 14) != 0) fail(SMAX_ERR_BAD_ARG, "no Matrix Market banner");
    const std::string obj = lower(tok[1]), fmt = lower(tok[2]), data = lower(tok[3]), sym = lower(tok[4]);
    if (obj != "matrix" || fmt != "coordinate") fail(SMAX_ERR_UNSUPPORTED, "only sparse (coordinate) matrices are read");
    if (data != "real" && data != "integer" && data != "pattern")
        fail(SMAX_ERR_UNSUPPORTED, "unsupported Matrix Market data type: " + data);
    if (sym != "general" && sym != "symmetric")
        fail(SMAX_ERR_UNSUPPORTED, "unsupported Matrix Market storage: " + sym);
    h.pattern = data == "pattern";
    h.symmetric = sym == "symmetric";
    // the size line: the first line not starting with '%' (mmio.cpp:138-163)
    while (true) {
        if (!next_line(s, pos, b, e)) fail(SMAX_ERR_BAD_ARG, "premature end of file before the size line");
        if (e > b && s[b] == '%') continue;
        const std::string line = s.substr(b, e - b);
        if (std::sscanf(line.c_str(), "%lld %lld %lld", &h.M, &h.N, &h.nz) == 3) break;
        bool blank = true;
        for (char c : line) blank &= (std::isspace((unsigned char)c) != 0);
        if (!blank) fail(SMAX_ERR_BAD_ARG, "could not parse the matrix size");
    }
    if (h.M < 0 || h.N < 0 || h.nz < 0) fail(SMAX_ERR_BAD_ARG, "negative matrix size");
    h.data_begin = pos;
    return h;
}

// Parses whitespace-separated entries of [p, end) (p at a line start, the
// text NUL-terminated after its last byte); appends per entry i-1, j-1 and
// the value.  Integers are read by hand (optional sign, decimal digits, as
// %d); values by strtod in place (what %lg does).  Returns false on a
// malformed token.
bool parse_slice(const char *p, const char *end, bool pattern, std::vector<int> &I, std::vector<int> &J,
                 std::vector<double> &V) {
    auto space = [](char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; };
    auto skip = [&] {
        while (p < end && space(*p)) ++p;
    };
    auto integer = [&](long long &out) {
        skip();
        if (p >= end) return false;
        bool neg = false;
        if (*p == '+' || *p == '-') neg = *p++ == '-';
        const char *d0 = p;
        long long v = 0;
        while (p < end && *p >= '0' && *p <= '9') {
            v = v * 10 + (*p - '0');
            if (v > (1ll << 40)) return false;
            ++p;
        }
        if (p == d0 || (p < end && !space(*p))) return false;
        out = neg ? -v : v;
        return true;
    };
    while (true) {
        skip();
        if (p >= end) return true;
        long long r = 0, c = 0;
        if (!integer(r) || !integer(c)) return false;
        double v = 0.01;
        if (!pattern) {
            skip();
            if (p >= end) return false;
            char *q = nullptr;
            v = std::strtod(p, &q);
            if (q == p || (q < end && !space(*q)) || q > end) return false;
            p = q;
        }
        if (r < -(1ll << 31) + 2 || r > (1ll << 31) || c < -(1ll << 31) + 2 || c > (1ll << 31)) return false;
        I.push_back((int)(r - 1));
        J.push_back((int)(c - 1));
        V.push_back(v);
    }
}

std::string read_file(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) fail(SMAX_ERR_BAD_ARG, std::string("unable to open file: ") + path);
    std::string s;
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (len > 0) {
        s.resize((size_t)len);
        if (std::fread(&s[0], 1, (size_t)len, f) != (size_t)len) {
            std::fclose(f);
            fail(SMAX_ERR_BAD_ARG, std::string("could not read file: ") + path);
        }
    }
    std::fclose(f);
    return s;
}

}  // namespace

}  // namespace smax

using namespace smax;

extern "C" {

smax_status smax_utils_convert_coo_to_crs(int float_type, uint64_t n_rows, uint64_t n_cols, uint64_t nnz,
                                          const int *I, const int *J, const double *val, void **row_ptr,
                                          void **col, void **val_out) {
    return guarded([&] {
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        if (!row_ptr || !col || !val_out) fail(SMAX_ERR_BAD_ARG, "null output pointer");
        if (nnz && (!I || !J || !val)) fail(SMAX_ERR_BAD_ARG, "null COO array");
        coo_to_crs(float_type == SMAX_FLOAT64 ? 8 : 4, (int64_t)n_rows, (int64_t)n_cols, (int64_t)nnz, I, J, val,
                   row_ptr, col, val_out);
    });
}

smax_status smax_utils_read_mtx(const char *path, int float_type, uint64_t *n_rows, uint64_t *n_cols, uint64_t *nnz,
                                void **row_ptr, void **col, void **val) {
    return guarded([&] {
        if (!path || !n_rows || !n_cols || !nnz || !row_ptr || !col || !val) fail(SMAX_ERR_BAD_ARG, "null argument");
        if (float_type != SMAX_FLOAT32 && float_type != SMAX_FLOAT64)
            fail(SMAX_ERR_UNSUPPORTED_TYPE, "value type must be float32 or float64");
        const std::string s = read_file(path);
        const Header h = parse_header(s);
        if (h.M >= (1ll << 31) || h.N >= (1ll << 31) || h.nz >= (1ll << 31))
            fail(SMAX_ERR_UNSUPPORTED, "int32 indices cannot address this matrix");
        // slices of the entry text, each starting at a line boundary
        const size_t beg = h.data_begin, len = s.size() - beg;
        unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
        if (len < (size_t)(1 << 20)) nt = 1;
        std::vector<size_t> cut(nt + 1, s.size());
        cut[0] = beg;
        for (unsigned t = 1; t < nt; ++t) {
            size_t c = beg + len * t / nt;
            c = std::max(c, cut[t - 1]);
            const size_t nl = s.find('\n', c);
            cut[t] = nl == std::string::npos ? s.size() : nl + 1;
        }
        std::vector<std::vector<int>> Is(nt), Js(nt);
        std::vector<std::vector<double>> Vs(nt);
        std::vector<char> ok(nt, 1);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                ok[t] = parse_slice(s.data() + cut[t], s.data() + cut[t + 1], h.pattern, Is[t], Js[t], Vs[t]);
            });
        for (auto &x : th) x.join();
        if (std::find(ok.begin(), ok.end(), 0) != ok.end() && nt > 1) {
            // an entry split over lines can straddle a cut: read the whole text as one slice
            nt = 1;
            Is.assign(1, {});
            Js.assign(1, {});
            Vs.assign(1, {});
            ok.assign(1, parse_slice(s.data() + beg, s.data() + s.size(), h.pattern, Is[0], Js[0], Vs[0]));
        }
        size_t total = 0;
        for (unsigned t = 0; t < nt; ++t) {
            if (!ok[t]) fail(SMAX_ERR_BAD_ARG, "malformed entry in the Matrix Market file");
            total += Is[t].size();
        }
        if (total < (size_t)h.nz) fail(SMAX_ERR_BAD_ARG, "premature end of file: fewer entries than announced");
        // the announced count is read (trailing tokens are ignored, as fscanf does)
        std::vector<int> I, J;
        std::vector<double> V;
        const size_t want = (size_t)h.nz;
        const size_t out = h.symmetric ? 2 * want : want;
        I.reserve(out);
        J.reserve(out);
        V.reserve(out);
        size_t taken = 0;
        for (unsigned t = 0; t < nt && taken < want; ++t)
            for (size_t k = 0; k < Is[t].size() && taken < want; ++k, ++taken) {
                I.push_back(Is[t][k]);
                J.push_back(Js[t][k]);
                V.push_back(Vs[t][k]);
                if (h.symmetric && Is[t][k] != Js[t][k]) {
                    I.push_back(Js[t][k]);
                    J.push_back(Is[t][k]);
                    V.push_back(Vs[t][k]);
                }
            }
        if (I.size() >= (size_t)1 << 31) fail(SMAX_ERR_UNSUPPORTED, "int32 indices cannot address this matrix");
        coo_to_crs(float_type == SMAX_FLOAT64 ? 8 : 4, h.M, h.N, (int64_t)I.size(), I.data(), J.data(), V.data(),
                   row_ptr, col, val);
        *n_rows = (uint64_t)h.M;
        *n_cols = (uint64_t)h.N;
        *nnz = (uint64_t)I.size();
    });
}

}  // extern "C"
