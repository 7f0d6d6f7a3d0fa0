// Post-processing of a count's outputs, the reference's PostProcess::merge_all
// (tool/PostProcess.h:63-139) on the device:
//
//   final_root.bin  every root file's records, root 0..255 in order, as they
//                   are (merge_buckets, :176-210)
//   final_low.bin   the low.bin keys that are no root file's key, sorted and
//                   without repeats, each as its N raw 64-bit words
//                   (process_low_bin + merge_sorted_chunks, :83-139, :244-323)
//   freq_hist.txt   "count\tnum_kmers", then one line per count in ascending
//                   order: every root record adds one key at its count + 1,
//                   every final_low.bin key one at count 1 (load_root_files,
//                   :142-174; write_hist, :71-81); not written when both are
//                   empty
//
// The reference reads low.bin as raw kmer<N> records, which is its packed
// layout only when the packed size is 8N bytes (k = 29..32, 61..64, ...);
// here low.bin is unpacked with k, so every k gets the keys its low.bin
// holds.  Like the reference, the count + 1 rule assumes every root key also
// sits in low.bin (true except for the filter's false positives).
//
// Device side: unpack the low keys, copy and sort the root keys, drop every
// low key found in them (binary search), sort the rest (the radix sort of
// kc_sort.cu) and keep the first of each run of equal keys.  The histogram is
// taken on the host from the root records it writes anyway.

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cuda_runtime.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"
#include "kc_kernels.cuh"
#include "kc_scan.cuh"

namespace {

int pfail(int code, const std::string& m) { return kc_internal_set_error(code, m.c_str()); }

#define PCK(x)                                                                                  \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) return pfail(KC_ERR_DEVICE, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline uint64_t cdiv(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Device buffers of one post-processing call (released on every exit).
struct Scratch {
    std::vector<void*> bufs;
    ~Scratch() {
        for (void* p : bufs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T** out, uint64_t count) {
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<uint64_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) bufs.push_back(p);
        *out = static_cast<T*>(p);
        return e;
    }
};

template <int NW>
__global__ void post_unpack(const uint8_t* __restrict__ low, uint64_t n, uint32_t k, uint64_t* __restrict__ out) {
    const uint32_t full = k / 32, tail_bytes = (2 * (k % 32) + 7) / 8, P = full * 8 + tail_bytes;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        const auto key = kc::unpack_low<NW>(low, r, P, full, tail_bytes);
        if constexpr (NW == 1) out[r] = key;
        else if constexpr (NW == 2) {
            out[2 * r] = key.w0;
            out[2 * r + 1] = key.w1;
        } else {
            out[4 * r] = key.w0;
            out[4 * r + 1] = key.w1;
            out[4 * r + 2] = key.w2;
            out[4 * r + 3] = key.w3;
        }
    }
}

template <int NW>
__global__ void post_root_keys(const uint64_t* __restrict__ rec, uint64_t n, uint64_t* __restrict__ out) {
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x)
        for (int w = 0; w < NW; ++w) out[(uint64_t)NW * r + w] = rec[(uint64_t)(NW + 1) * r + w];
}

template <int NW>
__device__ __forceinline__ int key_cmp(const uint64_t* a, const uint64_t* b) {
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if (a[w] < b[w]) return -1;
        if (a[w] > b[w]) return 1;
    }
    return 0;
}

// keep[i] = 1 when low key i is no root key (sorted root keys, binary search).
template <int NW>
__global__ void post_mark(const uint64_t* __restrict__ lk, uint64_t n, const uint64_t* __restrict__ rk, uint64_t nr,
                          uint32_t* __restrict__ keep) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t* key = lk + (uint64_t)NW * i;
        uint64_t lo = 0, hi = nr;
        bool found = false;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            const int c = key_cmp<NW>(rk + (uint64_t)NW * mid, key);
            if (c == 0) {
                found = true;
                break;
            }
            if (c < 0) lo = mid + 1;
            else hi = mid;
        }
        keep[i] = found ? 0u : 1u;
    }
}

// flag[i] = 1 for the first key of each run of equal keys (sorted input).
template <int NW>
__global__ void post_first_of_run(const uint64_t* __restrict__ k, uint64_t n, uint32_t* __restrict__ flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || key_cmp<NW>(k + (uint64_t)NW * (i - 1), k + (uint64_t)NW * i) != 0) ? 1u : 0u;
}

template <int NW>
__global__ void post_compact(const uint64_t* __restrict__ in, const uint32_t* __restrict__ flag,
                             const uint64_t* __restrict__ pos, uint64_t n, uint64_t* __restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i])
            for (int w = 0; w < NW; ++w) out[(uint64_t)NW * pos[i] + w] = in[(uint64_t)NW * i + w];
}

// Exclusive scan of n flags into pos; returns the total (synchronises).
int scan_flags(Scratch& sc, const uint32_t* flags, uint64_t n, uint64_t* pos, uint64_t* total, cudaStream_t st) {
    const uint64_t nb = std::max<uint64_t>(1, cdiv(n, kc::SCAN_TILE));
    uint64_t* sums = nullptr;
    uint64_t* d_total = nullptr;
    PCK(sc.get(&sums, nb + 1));
    PCK(sc.get(&d_total, 1));
    if (n) kc::scan_reduce<uint32_t><<<nb, kc::SCAN_BLOCK, 0, st>>>(flags, n, sums);
    else PCK(cudaMemsetAsync(sums, 0, sizeof(uint64_t), st));
    kc::scan_sums<<<1, kc::SCAN_BLOCK, 0, st>>>(sums, n ? nb : 1, 0, d_total);
    if (n) kc::scan_apply<uint32_t, uint64_t><<<nb, kc::SCAN_BLOCK, 0, st>>>(flags, n, sums, pos);
    PCK(cudaGetLastError());
    PCK(cudaMemcpyAsync(total, d_total, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    PCK(cudaStreamSynchronize(st));
    return KC_OK;
}

int sort_keys(Scratch& sc, uint64_t* keys, uint64_t n, uint32_t nw, uint32_t k, cudaStream_t st) {
    if (n < 2) return KC_OK;
    uint64_t bt, bh, bo, bs;
    kc_sort_scratch_bytes(n, 8ull * nw, &bt, &bh, &bo, &bs);
    uint8_t *t = nullptr, *h = nullptr, *o = nullptr, *s = nullptr;
    PCK(sc.get(&t, bt));
    PCK(sc.get(&h, bh));
    PCK(sc.get(&o, bo));
    PCK(sc.get(&s, bs));
    const int rc = kc_sort_keys(keys, n, nw, k, KcSortScratch{t, h, o, s}, st);
    if (rc) return pfail(rc, std::string("post-processing sort failed: ") + kc_sort_error());
    return KC_OK;
}

// final_low keys (sorted, unique, not among the root keys) of L packed low
// keys at d_low and R root records at d_roots (both device memory); host
// result in `out` (NW words per key).
template <int NW>
int final_low_keys(const uint8_t* d_low, uint64_t L, const void* d_roots, uint64_t R, uint32_t k, cudaStream_t st,
                   std::vector<uint64_t>& out, uint64_t* dropped) {
    Scratch sc;
    const int grid = 148 * 8;
    uint64_t *lk = nullptr, *rk = nullptr, *pos = nullptr, *kept = nullptr;
    uint32_t* flag = nullptr;
    PCK(sc.get(&lk, (uint64_t)NW * L));
    PCK(sc.get(&rk, (uint64_t)NW * R));
    PCK(sc.get(&flag, L));
    PCK(sc.get(&pos, L));
    PCK(sc.get(&kept, (uint64_t)NW * L));
    if (L) post_unpack<NW><<<grid, 256, 0, st>>>(d_low, L, k, lk);
    if (R) post_root_keys<NW><<<grid, 256, 0, st>>>(static_cast<const uint64_t*>(d_roots), R, rk);
    PCK(cudaGetLastError());
    int rc;
    if ((rc = sort_keys(sc, rk, R, NW, k, st))) return rc;
    if (L) post_mark<NW><<<grid, 256, 0, st>>>(lk, L, rk, R, flag);
    PCK(cudaGetLastError());
    uint64_t M = 0;
    if ((rc = scan_flags(sc, flag, L, pos, &M, st))) return rc;
    *dropped = L - M;
    if (L) post_compact<NW><<<grid, 256, 0, st>>>(lk, flag, pos, L, kept);
    PCK(cudaGetLastError());
    if ((rc = sort_keys(sc, kept, M, NW, k, st))) return rc;
    if (M) post_first_of_run<NW><<<grid, 256, 0, st>>>(kept, M, flag);
    PCK(cudaGetLastError());
    uint64_t U = 0;
    if ((rc = scan_flags(sc, flag, M, pos, &U, st))) return rc;
    if (M) post_compact<NW><<<grid, 256, 0, st>>>(kept, flag, pos, M, lk);  // lk is free again
    PCK(cudaGetLastError());
    out.resize((uint64_t)NW * U);
    if (U) PCK(cudaMemcpyAsync(out.data(), lk, U * NW * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    PCK(cudaStreamSynchronize(st));
    return KC_OK;
}

bool write_all(int fd, const void* data, uint64_t n) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    while (n) {
        const ssize_t w = ::write(fd, p, n > (1ull << 30) ? (1ull << 30) : n);
        if (w > 0) {
            p += w;
            n -= (uint64_t)w;
        } else if (w < 0 && errno == EINTR) {
            continue;
        } else {
            return false;
        }
    }
    return true;
}

int write_file(const std::string& path, const void* data, uint64_t n) {
    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return pfail(KC_ERR_IO, "cannot open " + path + ": " + std::strerror(errno));
    const bool ok = write_all(fd, data, n);
    if (::close(fd) != 0 || !ok) return pfail(KC_ERR_IO, "short write to " + path);
    return KC_OK;
}

std::string with_slash(const char* d) {
    std::string s = d && *d ? d : ".";
    if (s.back() != '/') s.push_back('/');
    return s;
}

// Common part: device low bytes + device root records (and the same records
// in host memory) -> the three files.
int post_process(uint32_t k, const uint8_t* d_low, uint64_t L, const void* d_roots, const uint8_t* h_roots,
                 uint64_t R, cudaStream_t st, const std::string& dir, kc_post_stats* stats) {
    const uint32_t nw = k <= 32 ? 1 : (k <= 64 ? 2 : 4);
    const uint64_t rec = 8ull * nw + 8;
    if (::mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST)
        return pfail(KC_ERR_IO, "cannot create " + dir + ": " + std::strerror(errno));
    int rc;
    if ((rc = write_file(dir + "final_root.bin", h_roots, R * rec))) return rc;
    std::vector<uint64_t> fl;
    uint64_t dropped = 0;
    rc = nw == 1 ? final_low_keys<1>(d_low, L, d_roots, R, k, st, fl, &dropped)
                 : (nw == 2 ? final_low_keys<2>(d_low, L, d_roots, R, k, st, fl, &dropped)
                            : final_low_keys<4>(d_low, L, d_roots, R, k, st, fl, &dropped));
    if (rc) return rc;
    if ((rc = write_file(dir + "final_low.bin", fl.data(), fl.size() * sizeof(uint64_t)))) return rc;
    // histogram: count + 1 per root record (32-bit arithmetic, as the
    // reference's uint32_t), 1 per final_low key
    const uint64_t U = fl.size() / nw;
    std::vector<uint64_t> small(1u << 20, 0);
    std::map<uint32_t, uint64_t> large;
    for (uint64_t r = 0; r < R; ++r) {
        uint32_t c;
        std::memcpy(&c, h_roots + r * rec + 8ull * nw, sizeof c);
        const uint32_t v = c + 1u;
        if (v < small.size()) ++small[v];
        else ++large[v];
    }
    if (U) small[1] += U;
    std::string text;
    uint64_t lines = 0;
    for (uint32_t v = 0; v < small.size(); ++v)
        if (small[v]) {
            text += std::to_string(v) + "\t" + std::to_string(small[v]) + "\n";
            ++lines;
        }
    for (const auto& [v, n] : large) {
        text += std::to_string(v) + "\t" + std::to_string(n) + "\n";
        ++lines;
    }
    if (lines) {
        text = "count\tnum_kmers\n" + text;
        if ((rc = write_file(dir + "freq_hist.txt", text.data(), text.size()))) return rc;
    }
    if (stats) {
        stats->root_records = R;
        stats->low_in = L;
        stats->low_in_roots = dropped;
        stats->final_low = U;
        stats->hist_lines = lines;
    }
    return KC_OK;
}

bool read_file(const std::string& path, std::vector<uint8_t>& out, bool* exists) {
    out.clear();
    *exists = false;
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) return errno == ENOENT;
    *exists = true;
    struct stat st;
    if (fstat(fd, &st) != 0) {
        ::close(fd);
        return false;
    }
    out.resize((size_t)st.st_size);
    uint64_t got = 0;
    while (got < out.size()) {
        const ssize_t r = ::read(fd, out.data() + got, out.size() - got);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        got += (uint64_t)r;
    }
    ::close(fd);
    return got == out.size();
}

}  // namespace

extern "C" {

int kc_post_process(kc_context* ctx, const char* out_dir, kc_post_stats* stats) {
    if (!ctx || !out_dir) return pfail(KC_ERR_INVALID, "null argument");
    const void *d_low = nullptr, *d_roots = nullptr;
    uint64_t low_bytes = 0, R = 0;
    int rc = kc_device_results(ctx, &d_low, &low_bytes, &d_roots, &R);
    if (rc) return rc;
    const uint32_t k = kc_internal_k(ctx);
    const uint64_t P = kc_packed_bytes(k), rec = kc_record_bytes(k);
    cudaStream_t st = static_cast<cudaStream_t>(kc_stream(ctx));
    std::vector<uint8_t> h_roots(R * rec);
    if (R) PCK(cudaMemcpyAsync(h_roots.data(), d_roots, R * rec, cudaMemcpyDeviceToHost, st));
    PCK(cudaStreamSynchronize(st));
    return post_process(k, static_cast<const uint8_t*>(d_low), low_bytes / P, d_roots, h_roots.data(), R, st,
                        with_slash(out_dir), stats);
}

int kc_post_process_dir(const kc_config* cfg, const char* temp_dir, const char* out_dir, kc_post_stats* stats) {
    if (!cfg || !temp_dir || !out_dir) return pfail(KC_ERR_INVALID, "null argument");
    const uint32_t k = cfg->k;
    if (k < 1 || k > 128) return pfail(KC_ERR_INVALID, "k out of range: 1..128");
    const uint64_t P = kc_packed_bytes(k), rec = kc_record_bytes(k);
    const std::string in = with_slash(temp_dir);
    std::vector<uint8_t> low, roots, part;
    bool exists = false;
    if (!read_file(in + "low.bin", low, &exists)) return pfail(KC_ERR_IO, "cannot read " + in + "low.bin");
    if (low.size() % P)
        return pfail(KC_ERR_IO, "Invalid low.bin size: " + std::to_string(low.size()) +
                                    " is not divisible by packed k-mer size " + std::to_string(P));
    for (int r = 0; r < 256; ++r) {
        const std::string f = in + "root_" + std::to_string(r) + ".bin";
        if (!read_file(f, part, &exists)) return pfail(KC_ERR_IO, "cannot read " + f);
        const uint64_t whole = part.size() / rec * rec;  // as the reference: whole records only
        roots.insert(roots.end(), part.begin(), part.begin() + whole);
    }
    const uint64_t L = low.size() / P, R = roots.size() / rec;
    int rc = cudaSetDevice(cfg->device) == cudaSuccess ? KC_OK : pfail(KC_ERR_DEVICE, "cudaSetDevice failed");
    if (rc) return rc;
    cudaStream_t st = nullptr;
    PCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    {
        Scratch sc;
        uint8_t *d_low = nullptr, *d_roots = nullptr;
        if ((rc = sc.get(&d_low, low.size() + 8) == cudaSuccess ? KC_OK : KC_ERR_NOMEM) ||
            (rc = sc.get(&d_roots, roots.size() + 8) == cudaSuccess ? KC_OK : KC_ERR_NOMEM)) {
            cudaStreamDestroy(st);
            return pfail(rc, "device allocation failed");
        }
        if (!low.empty()) cudaMemcpyAsync(d_low, low.data(), low.size(), cudaMemcpyHostToDevice, st);
        if (!roots.empty()) cudaMemcpyAsync(d_roots, roots.data(), roots.size(), cudaMemcpyHostToDevice, st);
        rc = post_process(k, d_low, L, d_roots, roots.data(), R, st, with_slash(out_dir), stats);
        cudaStreamSynchronize(st);
    }
    cudaStreamDestroy(st);
    return rc;
}

}  // extern "C"
