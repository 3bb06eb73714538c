// kernelset.cpp -- kernel-file loader, run-length packer, variances and the device kernel-set blob.
//
// Host code; built with -ffp-contract=off so every float multiply and add rounds separately, as in
// the reference's x86-64 build (no FMA without -march).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

#include "internal.h"

namespace lpaici {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_error(cudaError_t e, const char *what) {
    return set_error(e == cudaErrorMemoryAllocation ? LPAICI_ERR_NO_MEMORY : LPAICI_ERR_CUDA, "%s: %s (%s)", what,
                     cudaGetErrorString(e), cudaGetErrorName(e));
}

// ---------------------------------------------------------------------------------------------
// The adjoint's kernels.  The gather correlates fields with the kernels mirrored through their centre
// (taps (-dy, -dx)).  Scale s is stored as the mirrored difference D_s = h_s - h_{s-1} (D_0 = h_0): with
// c the adjoint field and [.] the selection mask,
//     sum_s h_s * (c [s* = s]) = sum_s D_s * (c [s* >= s]),
// so the gather masks one field in place, scale after scale, instead of building a field per scale.
// The difference is formed in double over the union of the two kernels' boxes (centres aligned) and
// rounded once.  Same device layout as the forward blob (BlobLayout): run ranges, runs
// {dy, dx0, len, wofs}, weights as {w, w} pairs with every run padded to an even length, 16 spare taps.
// ---------------------------------------------------------------------------------------------
static int build_adjoint_blob(lpaici_kernelset *ks) {
    const int D = ks->D, S = ks->S, nk = D * S;
    std::vector<int> begin(nk + 1), rdy, rdx, rlen;
    std::vector<float> w;
    for (int d = 0; d < D; d++)
        for (int s = 0; s < S; s++) {
            const int k = d * S + s;
            begin[k] = static_cast<int>(rdy.size());
            const int kp = s > 0 ? k - 1 : -1;  // the kernel subtracted: h_{s-1}
            const int hy = std::max(ks->rows[k] / 2, kp >= 0 ? ks->rows[kp] / 2 : 0);
            const int hx = std::max(ks->cols[k] / 2, kp >= 0 ? ks->cols[kp] / 2 : 0);
            const int bw = 2 * hx + 1;
            std::vector<double> box(static_cast<size_t>(2 * hy + 1) * bw, 0.0);  // offset (dy, dx) at (dy+hy, dx+hx)
            auto add = [&](int kk, double sign) {
                const float *h = ks->dense_w.data() + ks->off[kk];
                const int R = ks->rows[kk], Cc = ks->cols[kk];
                for (int r = 0; r < R; r++)
                    for (int c = 0; c < Cc; c++)
                        box[static_cast<size_t>(r - R / 2 + hy) * bw + (c - Cc / 2 + hx)] += sign * h[r * Cc + c];
            };
            add(k, 1.0);
            if (kp >= 0) add(kp, -1.0);
            // mirrored: tap (my, mx) of the gather kernel is box(-my, -mx)
            for (int my = -hy; my <= hy; my++) {
                const double *row = box.data() + static_cast<size_t>(-my + hy) * bw;
                int first = 1 << 30, last = -(1 << 30);
                for (int mx = -hx; mx <= hx; mx++)
                    if (static_cast<float>(row[-mx + hx]) != 0.0f) {
                        first = std::min(first, mx);
                        last = std::max(last, mx);
                    }
                if (first > last) continue;
                rdy.push_back(my);
                rdx.push_back(first);
                rlen.push_back(last - first + 1);
                for (int mx = first; mx <= last; mx++) w.push_back(static_cast<float>(row[-mx + hx]));
            }
        }
    begin[nk] = static_cast<int>(rdy.size());
    const int n_runs = begin[nk];
    BlobLayout L;
    L.nk = nk;
    L.n_runs = n_runs;
    L.run_word = (nk + 1 + 3) & ~3;
    L.weight_word = L.run_word + 4 * n_runs;
    std::vector<int> wofs(n_runs);
    int n2 = 0;
    for (int r = 0; r < n_runs; r++) {
        wofs[r] = n2;
        n2 += (rlen[r] + 1) & ~1;
    }
    L.n_wdup = n2;
    L.total_words = (L.weight_word + 2 * (n2 + 16) + 3) & ~3;
    ks->adj_layout = L;
    ks->adj_blob.assign(L.total_words, 0);
    for (int k = 0; k <= nk; k++) ks->adj_blob[k] = begin[k];
    float *wd = reinterpret_cast<float *>(ks->adj_blob.data() + L.weight_word);
    int wi = 0;
    for (int r = 0; r < n_runs; r++) {
        ks->adj_blob[L.run_word + 4 * r + 0] = rdy[r];
        ks->adj_blob[L.run_word + 4 * r + 1] = rdx[r];
        ks->adj_blob[L.run_word + 4 * r + 2] = rlen[r];
        ks->adj_blob[L.run_word + 4 * r + 3] = wofs[r];
        for (int j = 0; j < rlen[r]; j++, wi++) {
            wd[2 * (wofs[r] + j)] = w[wi];
            wd[2 * (wofs[r] + j) + 1] = w[wi];
        }
    }
    return LPAICI_OK;
}

// ---------------------------------------------------------------------------------------------
// Packing: one run per kernel row, from its first to its last nonzero (interior zeros kept), with
// centre-relative coordinates (row - rows/2, first - cols/2): the layout of build_sparse_kernels
// (src/v4_1_lpa_ici_2D_sparse_shared.cu:826-877), here without any capacity limit.
// ---------------------------------------------------------------------------------------------
static int finish_kernelset(lpaici_kernelset *ks) {
    const int nk = ks->D * ks->S;
    if (nk > kMaxKernels)
        return set_error(LPAICI_ERR_UNSUPPORTED, "kernel set has %d kernels (%d directions x %d scales); at most %d",
                         nk, ks->D, ks->S, kMaxKernels);
    ks->norm2.assign(nk, 0.0f);
    ks->nnz.assign(nk, 0);
    ks->radius = 0;
    for (int k = 0; k < nk; k++) {
        const float *h = ks->dense_w.data() + ks->off[k];
        const int R = ks->rows[k], Cc = ks->cols[k];
        float nsq = 0.0f;
        for (int i = 0; i < R * Cc; i++) nsq += h[i] * h[i];  // compute_kernel_variances order
        ks->norm2[k] = nsq;
        ks->k_first_run.push_back(static_cast<int>(ks->run_row.size()));
        ks->k_first_weight.push_back(static_cast<int>(ks->run_w.size()));
        for (int r = 0; r < R; r++) {
            int first = -1, last = -1;
            for (int c = 0; c < Cc; c++)
                if (h[r * Cc + c] != 0.0f) {
                    if (first < 0) first = c;
                    last = c;
                    ks->nnz[k]++;
                }
            if (first < 0) continue;
            const int dy = r - R / 2, dx0 = first - Cc / 2, len = last - first + 1;
            ks->run_row.push_back(dy);
            ks->run_col.push_back(dx0);
            ks->run_len.push_back(len);
            for (int c = first; c <= last; c++) ks->run_w.push_back(h[r * Cc + c]);
            int reach = std::abs(dy);
            if (std::abs(dx0) > reach) reach = std::abs(dx0);
            if (std::abs(dx0 + len - 1) > reach) reach = std::abs(dx0 + len - 1);
            if (reach > ks->radius) ks->radius = reach;
        }
        ks->k_num_runs.push_back(static_cast<int>(ks->run_row.size()) - ks->k_first_run[k]);
    }
    if (ks->radius > kMaxRadius)
        return set_error(LPAICI_ERR_UNSUPPORTED, "kernel radius %d exceeds the supported %d", ks->radius, kMaxRadius);

    // device blob: [run begin per kernel (nk+1)] [Run records] [{w, w} per tap, runs padded to even]
    BlobLayout &L = ks->layout;
    L.nk = nk;
    L.n_runs = static_cast<int>(ks->run_row.size());
    L.run_word = (nk + 1 + 3) & ~3;
    L.weight_word = L.run_word + 4 * L.n_runs;
    std::vector<int> wofs(L.n_runs);
    int n2 = 0;
    for (int r = 0; r < L.n_runs; r++) {
        wofs[r] = n2;
        n2 += (ks->run_len[r] + 1) & ~1;
    }
    L.n_wdup = n2;
    // 16 spare {0, 0} taps after the last run, a margin: the kernels' weight loads stay within each
    // run's taps and its even-length padding
    L.total_words = (L.weight_word + 2 * (n2 + 16) + 3) & ~3;
    ks->blob.assign(L.total_words, 0);
    for (int k = 0; k < nk; k++) ks->blob[k] = ks->k_first_run[k];
    ks->blob[nk] = L.n_runs;
    float *wd = reinterpret_cast<float *>(ks->blob.data() + L.weight_word);
    for (int k = 0; k < nk; k++) {
        int w = ks->k_first_weight[k];
        for (int r = ks->k_first_run[k]; r < ks->k_first_run[k] + ks->k_num_runs[k]; r++) {
            ks->blob[L.run_word + 4 * r + 0] = ks->run_row[r];
            ks->blob[L.run_word + 4 * r + 1] = ks->run_col[r];
            ks->blob[L.run_word + 4 * r + 2] = ks->run_len[r];
            ks->blob[L.run_word + 4 * r + 3] = wofs[r];
            for (int j = 0; j < ks->run_len[r]; j++) {
                wd[2 * (wofs[r] + j)] = ks->run_w[w + j];
                wd[2 * (wofs[r] + j) + 1] = ks->run_w[w + j];
            }
            w += ks->run_len[r];
        }
    }

    return build_adjoint_blob(ks);
}

int device_blob(const lpaici_kernelset *ks, const int **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lock(ks->mu);
    if (static_cast<int>(ks->dev_blob.size()) <= dev) {
        ks->dev_blob.resize(dev + 1, nullptr);
        ks->tuned_config.resize(dev + 1, -1);
    }
    if (!ks->dev_blob[dev]) {
        int *p = nullptr;
        e = cudaMalloc(&p, sizeof(int32_t) * ks->blob.size());
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc(kernel set)");
        e = cudaMemcpy(p, ks->blob.data(), sizeof(int32_t) * ks->blob.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(p);
            return cuda_error(e, "cudaMemcpy(kernel set)");
        }
        ks->dev_blob[dev] = p;
    }
    *out = ks->dev_blob[dev];
    return LPAICI_OK;
}

int device_adj_blob(const lpaici_kernelset *ks, const int **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lock(ks->mu);
    if (static_cast<int>(ks->dev_adj_blob.size()) <= dev) ks->dev_adj_blob.resize(dev + 1, nullptr);
    if (!ks->dev_adj_blob[dev]) {
        int *p = nullptr;
        e = cudaMalloc(&p, sizeof(int32_t) * ks->adj_blob.size());
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc(adjoint kernel set)");
        e = cudaMemcpy(p, ks->adj_blob.data(), sizeof(int32_t) * ks->adj_blob.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(p);
            return cuda_error(e, "cudaMemcpy(adjoint kernel set)");
        }
        ks->dev_adj_blob[dev] = p;
    }
    *out = ks->dev_adj_blob[dev];
    return LPAICI_OK;
}

void fill_tables(const lpaici_kernelset *ks, const float *var_or_null, float sigma, float gamma, KernelTables *t) {
    const int nk = ks->D * ks->S;
    t->D = ks->D;
    t->S = ks->S;
    t->neg_zero = -0.0f;
    t->R = ks->radius;
    t->blob_words = ks->layout.total_words;
    t->run_word = ks->layout.run_word;
    t->weight_word = ks->layout.weight_word;
    const float s2 = sigma * sigma;
    for (int k = 0; k < nk; k++) {
        const float v = var_or_null ? var_or_null[k] : s2 * ks->norm2[k];
        t->var[k] = v;
        t->thr[k] = gamma * std::sqrt(v);  // src/v1_0_lpa_ici_2D_fused.cpp:905
    }
}

// ---------------------------------------------------------------------------------------------
// Text loader with the semantics of load_LPA_kernels_standardized
// (src/v1_0_lpa_ici_2D_fused.cpp:466-551): header "D S" (> 0), then per kernel "rows cols" (> 0)
// and rows*cols weights; direction 0 fixes each scale's size; every other direction is
// centre-cropped to it with offset (file - target) / 2.
// ---------------------------------------------------------------------------------------------
namespace {
// Numbers are read like std::istream's operator>> in the "C" locale: skip whitespace, take the
// longest prefix that looks like a number and leave the rest of the text for the next read.
//   int:   [+-]?[0-9]+                                    (fails on overflow)
//   float: [+-]?[0-9]*(\.[0-9]*)?([eE][+-]?[0-9]*)?  with at least one mantissa digit, converted
//          with correct rounding (strtof); fails if the exponent has no digits or the value
//          overflows; underflow gives 0 or a subnormal.  "inf", "nan" and hex text fail or stop at
//          the first letter, as they do for operator>>.
struct Stream {
    const char *p, *end;
    static bool space(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }
    static bool digit(char c) { return c >= '0' && c <= '9'; }
    void skip() {
        while (p < end && space(*p)) p++;
    }
    bool next_int(int &v) {
        skip();
        const char *b = p;
        if (p < end && (*p == '+' || *p == '-')) p++;
        const char *d = p;
        while (p < end && digit(*p)) p++;
        if (p == d) return false;
        const std::string t(b, p);
        errno = 0;
        const long x = std::strtol(t.c_str(), nullptr, 10);
        if (errno != 0 || x > 2147483647L || x < -2147483647L - 1) return false;
        v = static_cast<int>(x);
        return true;
    }
    bool next_float(float &v) {
        skip();
        const char *b = p;
        if (p < end && (*p == '+' || *p == '-')) p++;
        int mant = 0;
        while (p < end && digit(*p)) p++, mant++;
        if (p < end && *p == '.') {
            p++;
            while (p < end && digit(*p)) p++, mant++;
        }
        if (mant == 0) return false;
        if (p < end && (*p == 'e' || *p == 'E')) {
            p++;
            if (p < end && (*p == '+' || *p == '-')) p++;
            int ed = 0;
            while (p < end && digit(*p)) p++, ed++;
            if (ed == 0) return false;
        }
        const std::string t(b, p);
        char *e = nullptr;
        v = std::strtof(t.c_str(), &e);
        return *e == '\0' && !std::isinf(v);
    }
};
}  // namespace

}  // namespace lpaici

using namespace lpaici;

// ---------------------------------------------------------------------------------------------
// Binary tap-list file (lpaici_kernelset_save): the run-length packing of every kernel, which
// together with the kernel sizes restores the loader's cropped dense output (zero outside the runs).
//   "LPAICIT1"  int32 D, S  int32 rows[nk], cols[nk]  int32 n_runs, n_taps  int32 first_run[nk+1]
//   int32 dy[n_runs], dx0[n_runs], len[n_runs]  float w[n_taps]  uint64 FNV-1a of all bytes before
// Little-endian; offsets dy, dx0 are centre-relative as in build_sparse_kernels.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr char kTapMagic[8] = {'L', 'P', 'A', 'I', 'C', 'I', 'T', '1'};

uint64_t fnv1a(const char *p, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; i++) {
        h ^= static_cast<unsigned char>(p[i]);
        h *= 1099511628211ull;
    }
    return h;
}

struct Reader {
    const char *p, *end;
    template <typename T>
    bool get(T *dst, size_t n) {
        const size_t bytes = sizeof(T) * n;
        if (static_cast<size_t>(end - p) < bytes) return false;
        std::memcpy(dst, p, bytes);
        p += bytes;
        return true;
    }
};

// Fills ks (D, S, dense arrays) from a tap-list file image; LPAICI_OK or LPAICI_ERR_KERNEL_FORMAT.
int parse_tap_file(const std::string &bytes, const char *path, lpaici_kernelset *ks) {
    const size_t body = bytes.size() >= sizeof(uint64_t) ? bytes.size() - sizeof(uint64_t) : 0;
    uint64_t stored = 0;
    if (body < sizeof(kTapMagic)) return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: truncated tap-list file", path);
    std::memcpy(&stored, bytes.data() + body, sizeof(stored));
    if (stored != fnv1a(bytes.data(), body))
        return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: tap-list checksum mismatch", path);
    Reader rd{bytes.data() + sizeof(kTapMagic), bytes.data() + body};
    int D = 0, S = 0;
    if (!rd.get(&D, 1) || !rd.get(&S, 1) || D <= 0 || S <= 0)
        return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: bad tap-list header", path);
    if (static_cast<long>(D) * S > kMaxKernels)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%s has %d x %d kernels; at most %d", path, D, S, kMaxKernels);
    const int nk = D * S;
    std::vector<int> rows(nk), cols(nk), first(nk + 1);
    int n_runs = 0, n_taps = 0;
    if (!rd.get(rows.data(), nk) || !rd.get(cols.data(), nk) || !rd.get(&n_runs, 1) || !rd.get(&n_taps, 1) ||
        n_runs < 0 || n_taps < 0 || n_runs > (1 << 26) || n_taps > (1 << 28) || !rd.get(first.data(), nk + 1))
        return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: truncated tap-list file", path);
    std::vector<int> dy(n_runs), dx0(n_runs), len(n_runs);
    std::vector<float> w(n_taps);
    if (!rd.get(dy.data(), n_runs) || !rd.get(dx0.data(), n_runs) || !rd.get(len.data(), n_runs) ||
        !rd.get(w.data(), n_taps) || rd.p != rd.end)
        return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: tap-list sizes do not match the file", path);
    if (first[0] != 0 || first[nk] != n_runs)
        return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: bad run ranges", path);
    ks->D = D;
    ks->S = S;
    long taps = 0;
    for (int k = 0; k < nk; k++) {
        if (rows[k] <= 0 || cols[k] <= 0 || static_cast<long>(rows[k]) * cols[k] > (1L << 26) || first[k + 1] < first[k])
            return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: bad size or run range of kernel %d", path, k);
        ks->off.push_back(static_cast<int>(ks->dense_w.size()));
        ks->rows.push_back(rows[k]);
        ks->cols.push_back(cols[k]);
        const size_t base = ks->dense_w.size();
        ks->dense_w.resize(base + static_cast<size_t>(rows[k]) * cols[k], 0.0f);
        for (int r = first[k]; r < first[k + 1]; r++) {
            const int row = dy[r] + rows[k] / 2, col = dx0[r] + cols[k] / 2;
            if (row < 0 || row >= rows[k] || col < 0 || len[r] <= 0 || col + len[r] > cols[k] || taps + len[r] > n_taps)
                return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: run %d lies outside kernel %d", path, r, k);
            std::memcpy(&ks->dense_w[base + static_cast<size_t>(row) * cols[k] + col], &w[taps], sizeof(float) * len[r]);
            taps += len[r];
        }
    }
    if (taps != n_taps) return set_error(LPAICI_ERR_KERNEL_FORMAT, "%s: %ld taps in runs, %d stored", path, taps, n_taps);
    return LPAICI_OK;
}

}  // namespace

extern "C" {

const char *lpaici_last_error(void) { return g_last_error.c_str(); }

const char *lpaici_status_string(int status) {
    switch (status) {
        case LPAICI_OK: return "LPAICI_OK";
        case LPAICI_ERR_INVALID_ARG: return "LPAICI_ERR_INVALID_ARG";
        case LPAICI_ERR_FILE: return "LPAICI_ERR_FILE";
        case LPAICI_ERR_KERNEL_FORMAT: return "LPAICI_ERR_KERNEL_FORMAT";
        case LPAICI_ERR_UNSUPPORTED: return "LPAICI_ERR_UNSUPPORTED";
        case LPAICI_ERR_CUDA: return "LPAICI_ERR_CUDA";
        case LPAICI_ERR_NO_MEMORY: return "LPAICI_ERR_NO_MEMORY";
        default: return "LPAICI_ERR_UNKNOWN";
    }
}

int lpaici_kernelset_load(const char *path, lpaici_kernelset **out) {
    if (!path || !out) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_load: null argument");
    *out = nullptr;
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return set_error(LPAICI_ERR_FILE, "Failed to open %s", path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    if (text.size() >= sizeof(kTapMagic) && std::memcmp(text.data(), kTapMagic, sizeof(kTapMagic)) == 0) {
        auto *ks = new lpaici_kernelset();
        int rc = parse_tap_file(text, path, ks);
        if (rc == LPAICI_OK) rc = finish_kernelset(ks);
        if (rc == LPAICI_OK) {
            int ndev = 0;
            if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
                const int *p = nullptr;
                rc = device_blob(ks, &p);
            } else {
                cudaGetLastError();
            }
        }
        if (rc != LPAICI_OK) {
            delete ks;
            return rc;
        }
        *out = ks;
        return LPAICI_OK;
    }
    Stream tk{text.data(), text.data() + text.size()};

    int D = 0, S = 0;
    if (!tk.next_int(D) || !tk.next_int(S) || D <= 0 || S <= 0)
        return set_error(LPAICI_ERR_KERNEL_FORMAT, "invalid header in %s", path);
    if (static_cast<long>(D) * S > kMaxKernels)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%s has %d x %d kernels; at most %d", path, D, S, kMaxKernels);

    auto *ks = new lpaici_kernelset();
    ks->D = D;
    ks->S = S;
    std::vector<int> trow(S), tcol(S);
    std::vector<float> tmp;
    for (int d = 0; d < D; d++) {
        for (int s = 0; s < S; s++) {
            int fr = 0, fc = 0;
            if (!tk.next_int(fr) || !tk.next_int(fc) || fr <= 0 || fc <= 0 || static_cast<long>(fr) * fc > (1L << 26)) {
                delete ks;
                return set_error(LPAICI_ERR_KERNEL_FORMAT, "invalid size of kernel %d, %d in %s", d, s, path);
            }
            tmp.resize(static_cast<size_t>(fr) * fc);
            for (auto &v : tmp)
                if (!tk.next_float(v)) {
                    delete ks;
                    return set_error(LPAICI_ERR_KERNEL_FORMAT, "missing weights of kernel %d, %d in %s", d, s, path);
                }
            if (d == 0) {
                trow[s] = fr;
                tcol[s] = fc;
            }
            const int tr = trow[s], tc = tcol[s];
            if (fr < tr || fc < tc) {
                delete ks;
                return set_error(LPAICI_ERR_KERNEL_FORMAT,
                                 "Matrix at direction %d, scale %d is too small to crop to the target size", d, s);
            }
            const int ro = (fr - tr) / 2, co = (fc - tc) / 2;
            ks->off.push_back(static_cast<int>(ks->dense_w.size()));
            ks->rows.push_back(tr);
            ks->cols.push_back(tc);
            for (int r = 0; r < tr; r++)
                for (int c = 0; c < tc; c++) ks->dense_w.push_back(tmp[static_cast<size_t>(r + ro) * fc + (c + co)]);
        }
    }
    int rc = finish_kernelset(ks);
    if (rc != LPAICI_OK) {
        delete ks;
        return rc;
    }
    // best effort: upload to the current device now, outside any stream capture
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
        const int *p = nullptr;
        rc = device_blob(ks, &p);
        if (rc != LPAICI_OK) {
            delete ks;
            return rc;
        }
    } else {
        cudaGetLastError();
    }
    *out = ks;
    return LPAICI_OK;
}

int lpaici_kernelset_generate(int num_dirs, int num_scales, const int *scales, int order, int shape,
                              lpaici_kernelset **out) {
    if (!scales || !out || num_dirs <= 0 || num_scales <= 0 || order < 0 || order > 4 ||
        (shape != LPAICI_SHAPE_SECTOR && shape != LPAICI_SHAPE_QUADRANT))
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_generate: bad directions, scales, order or shape");
    *out = nullptr;
    if (static_cast<long>(num_dirs) * num_scales > kMaxKernels)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%d x %d kernels; at most %d", num_dirs, num_scales, kMaxKernels);
    for (int s = 0; s < num_scales; s++)
        if (scales[s] < 1 || scales[s] > kMaxRadius + 1)
            return set_error(LPAICI_ERR_INVALID_ARG, "scale %d is %d; 1 .. %d", s, scales[s], kMaxRadius + 1);
    const double kPi = 3.14159265358979323846;
    std::vector<float> w;
    std::vector<int> off, rows, cols;
    for (int d = 0; d < num_dirs; d++) {
        const double th = 2.0 * kPi * d / num_dirs, c = std::cos(th), sn = std::sin(th);
        for (int si = 0; si < num_scales; si++) {
            const int h = scales[si], R = h - 1, n = 2 * R + 1;
            // support: pixel (x, y) (y down) has u = x cos + (-y) sin along the direction, v across it
            std::vector<int> idx;
            std::vector<double> us;
            for (int y = -R; y <= R; y++)
                for (int x = -R; x <= R; x++) {
                    const double X = x, Y = -y;
                    const double u = X * c + Y * sn, v = -X * sn + Y * c;
                    bool in;
                    if (shape == LPAICI_SHAPE_SECTOR)
                        in = (x == 0 && y == 0) || (u < h - 0.5 && std::fabs(std::atan2(v, u)) <= kPi / num_dirs + 1e-9);
                    else
                        in = u > -0.5 && u < h - 0.5 && v < 0.5 && v > -(h - 0.5);
                    if (in) {
                        idx.push_back((y + R) * n + (x + R));
                        us.push_back(u);
                    }
                }
            // least-squares polynomial in u of order p (at most the distinct u values less one), equal
            // weights, evaluated at the origin: g_i = sum_q beta_q u_i^q, (sum_i u_i^(j+q)) beta = e_0
            std::vector<double> distinct = us;
            std::sort(distinct.begin(), distinct.end());
            int nu = 0;
            for (size_t i = 0; i < distinct.size(); i++)
                if (i == 0 || distinct[i] - distinct[i - 1] > 1e-9) nu++;
            const int p = std::min(order, nu - 1), m = p + 1;
            double A[5][6] = {};
            for (int j = 0; j < m; j++) {
                for (int q = 0; q < m; q++)
                    for (const double u : us) A[j][q] += std::pow(u, j + q);
                A[j][m] = j == 0 ? 1.0 : 0.0;
            }
            for (int col = 0; col < m; col++) {  // Gauss-Jordan with partial pivoting
                int piv = col;
                for (int r = col + 1; r < m; r++)
                    if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
                for (int q = 0; q <= m; q++) std::swap(A[col][q], A[piv][q]);
                for (int r = 0; r < m; r++) {
                    if (r == col) continue;
                    const double f = A[r][col] / A[col][col];
                    for (int q = col; q <= m; q++) A[r][q] -= f * A[col][q];
                }
            }
            off.push_back(static_cast<int>(w.size()));
            rows.push_back(n);
            cols.push_back(n);
            const size_t base = w.size();
            w.resize(base + static_cast<size_t>(n) * n, 0.0f);
            for (size_t i = 0; i < idx.size(); i++) {
                double g = 0.0;
                for (int q = 0; q < m; q++) g += A[q][m] / A[q][q] * std::pow(us[i], q);
                w[base + idx[i]] = static_cast<float>(g);
            }
        }
    }
    return lpaici_kernelset_create(w.data(), off.data(), rows.data(), cols.data(), num_dirs, num_scales, out);
}

int lpaici_kernelset_write_text(const lpaici_kernelset *ks, const char *path) {
    if (!ks || !path) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_write_text: null argument");
    FILE *f = std::fopen(path, "w");
    if (!f) return set_error(LPAICI_ERR_FILE, "cannot write %s", path);
    std::fprintf(f, "%d %d\n", ks->D, ks->S);
    for (int k = 0; k < ks->D * ks->S; k++) {
        std::fprintf(f, "%d %d\n", ks->rows[k], ks->cols[k]);
        const float *h = ks->dense_w.data() + ks->off[k];
        for (int i = 0; i < ks->rows[k] * ks->cols[k]; i++) std::fprintf(f, "%f ", static_cast<double>(h[i]));
        std::fprintf(f, "\n");
    }
    const bool ok = std::fflush(f) == 0 && !std::ferror(f);
    std::fclose(f);
    return ok ? LPAICI_OK : set_error(LPAICI_ERR_FILE, "writing %s failed", path);
}

int lpaici_kernelset_create(const float *weights, const int *offsets, const int *rows, const int *cols, int num_dirs,
                            int num_scales, lpaici_kernelset **out) {
    if (!weights || !offsets || !rows || !cols || !out || num_dirs <= 0 || num_scales <= 0)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_create: null array or non-positive D/S");
    *out = nullptr;
    const long nk = static_cast<long>(num_dirs) * num_scales;
    if (nk > kMaxKernels)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%d x %d kernels; at most %d", num_dirs, num_scales, kMaxKernels);
    auto *ks = new lpaici_kernelset();
    ks->D = num_dirs;
    ks->S = num_scales;
    for (long k = 0; k < nk; k++) {
        if (rows[k] <= 0 || cols[k] <= 0 || offsets[k] < 0 || static_cast<long>(rows[k]) * cols[k] > (1L << 26)) {
            delete ks;
            return set_error(LPAICI_ERR_KERNEL_FORMAT, "kernel %ld has size %d x %d at offset %d", k, rows[k], cols[k],
                             offsets[k]);
        }
        ks->off.push_back(static_cast<int>(ks->dense_w.size()));
        ks->rows.push_back(rows[k]);
        ks->cols.push_back(cols[k]);
        ks->dense_w.insert(ks->dense_w.end(), weights + offsets[k], weights + offsets[k] + rows[k] * cols[k]);
    }
    int rc = finish_kernelset(ks);
    if (rc != LPAICI_OK) {
        delete ks;
        return rc;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
        const int *p = nullptr;
        rc = device_blob(ks, &p);
        if (rc != LPAICI_OK) {
            delete ks;
            return rc;
        }
    } else {
        cudaGetLastError();
    }
    *out = ks;
    return LPAICI_OK;
}

int lpaici_kernelset_save(const lpaici_kernelset *ks, const char *path) {
    if (!ks || !path) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_save: null argument");
    const int nk = ks->D * ks->S;
    std::string b(kTapMagic, sizeof(kTapMagic));
    auto put = [&b](const void *p, size_t n) { b.append(static_cast<const char *>(p), n); };
    const int n_runs = static_cast<int>(ks->run_row.size()), n_taps = static_cast<int>(ks->run_w.size());
    std::vector<int> first(ks->k_first_run);
    first.push_back(n_runs);
    put(&ks->D, sizeof(int));
    put(&ks->S, sizeof(int));
    put(ks->rows.data(), sizeof(int) * nk);
    put(ks->cols.data(), sizeof(int) * nk);
    put(&n_runs, sizeof(int));
    put(&n_taps, sizeof(int));
    put(first.data(), sizeof(int) * (nk + 1));
    put(ks->run_row.data(), sizeof(int) * n_runs);
    put(ks->run_col.data(), sizeof(int) * n_runs);
    put(ks->run_len.data(), sizeof(int) * n_runs);
    put(ks->run_w.data(), sizeof(float) * n_taps);
    const uint64_t h = fnv1a(b.data(), b.size());
    put(&h, sizeof(h));
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.is_open()) return set_error(LPAICI_ERR_FILE, "cannot create %s", path);
    f.write(b.data(), static_cast<std::streamsize>(b.size()));
    f.close();
    if (!f) return set_error(LPAICI_ERR_FILE, "cannot write %s", path);
    return LPAICI_OK;
}

int lpaici_kernelset_destroy(lpaici_kernelset *ks) {
    if (!ks) return LPAICI_OK;
    int cur = -1;
    cudaGetDevice(&cur);
    for (size_t d = 0; d < ks->dev_blob.size(); d++)
        if (ks->dev_blob[d]) {
            cudaSetDevice(static_cast<int>(d));
            cudaFree(ks->dev_blob[d]);
        }
    for (size_t d = 0; d < ks->dev_adj_blob.size(); d++)
        if (ks->dev_adj_blob[d]) {
            cudaSetDevice(static_cast<int>(d));
            cudaFree(ks->dev_adj_blob[d]);
        }
    if (cur >= 0) cudaSetDevice(cur);
    cudaGetLastError();
    delete ks;
    return LPAICI_OK;
}

int lpaici_kernelset_get_info(const lpaici_kernelset *ks, lpaici_kernelset_info_t *info) {
    if (!ks || !info) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_get_info: null argument");
    info->num_dirs = ks->D;
    info->num_scales = ks->S;
    info->dense_size = static_cast<int>(ks->dense_w.size());
    info->n_taps = static_cast<int>(ks->run_w.size());
    info->n_runs = static_cast<int>(ks->run_row.size());
    info->radius = ks->radius;
    info->blob_bytes = static_cast<int>(sizeof(int32_t) * ks->blob.size());
    info->adjoint_blob_bytes = static_cast<int>(sizeof(int32_t) * ks->adj_blob.size());
    return LPAICI_OK;
}

int lpaici_kernelset_get_dense(const lpaici_kernelset *ks, float *weights, int *offsets, int *rows, int *cols) {
    if (!ks || !weights || !offsets || !rows || !cols)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_get_dense: null argument");
    std::memcpy(weights, ks->dense_w.data(), sizeof(float) * ks->dense_w.size());
    std::memcpy(offsets, ks->off.data(), sizeof(int) * ks->off.size());
    std::memcpy(rows, ks->rows.data(), sizeof(int) * ks->rows.size());
    std::memcpy(cols, ks->cols.data(), sizeof(int) * ks->cols.size());
    return LPAICI_OK;
}

int lpaici_kernelset_get_runs(const lpaici_kernelset *ks, float *weights, int *run_row, int *run_col, int *run_len,
                              int *kernel_first_run, int *kernel_num_runs, int *kernel_first_weight) {
    if (!ks || !weights || !run_row || !run_col || !run_len || !kernel_first_run || !kernel_num_runs ||
        !kernel_first_weight)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernelset_get_runs: null argument");
    std::memcpy(weights, ks->run_w.data(), sizeof(float) * ks->run_w.size());
    std::memcpy(run_row, ks->run_row.data(), sizeof(int) * ks->run_row.size());
    std::memcpy(run_col, ks->run_col.data(), sizeof(int) * ks->run_col.size());
    std::memcpy(run_len, ks->run_len.data(), sizeof(int) * ks->run_len.size());
    std::memcpy(kernel_first_run, ks->k_first_run.data(), sizeof(int) * ks->k_first_run.size());
    std::memcpy(kernel_num_runs, ks->k_num_runs.data(), sizeof(int) * ks->k_num_runs.size());
    std::memcpy(kernel_first_weight, ks->k_first_weight.data(), sizeof(int) * ks->k_first_weight.size());
    return LPAICI_OK;
}

int lpaici_kernel_variances(const lpaici_kernelset *ks, float sigma, float *var) {
    if (!ks || !var) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_kernel_variances: null argument");
    const float s2 = sigma * sigma;
    for (int k = 0; k < ks->D * ks->S; k++) var[k] = s2 * ks->norm2[k];
    return LPAICI_OK;
}

int lpaici_add_noise(const float *clean, float *noisy, long n, float sigma, unsigned int seed) {
    if (!clean || !noisy || n < 0) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_add_noise: bad argument");
    std::mt19937 gen{seed};
    std::normal_distribution<float> dist{0.0, sigma};
    for (long i = 0; i < n; i++) {
        const float sample = dist(gen);
        noisy[i] = clean[i] + sample;
    }
    return LPAICI_OK;
}

double lpaici_psnr(const float *a, const float *b, long n) {
    if (!a || !b || n <= 0) return NAN;
    double sum = 0.0;
    for (long i = 0; i < n; i++) {
        const float diff = a[i] - b[i];
        const float sq = diff * diff;
        sum += sq;
    }
    const double mse = sum / n;
    return 10.0 * std::log10(1.0f / mse);
}

}  // extern "C"
