// File side of the C ABI: FASTQ input (plain or gzip) and the reference's
// output files.
//
//   input   gzip is detected by the magic bytes 1F 8B and inflated with zlib,
//           as src/FastqReader.h:93-104 does; plain files are read as bytes.
//   output  <dir>/low.bin       packed keys     (src/ExportWriter.h:339-344)
//           <dir>/root_{id}.bin ExportRecord<N> (src/FinalDrainWriter.h:31-90),
//           all 256 created, empty ones included.

#include <algorithm>
#include <cerrno>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include "../../include/kmer_count.h"
#include "kc_internal.h"

namespace {

int io_fail(const std::string& m) { return kc_internal_set_error(KC_ERR_IO, m.c_str()); }

bool write_all(int fd, const uint8_t* p, uint64_t n) {
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

bool pwrite_all(int fd, const uint8_t* p, uint64_t n, uint64_t off) {
    while (n) {
        const ssize_t w = ::pwrite(fd, p, n > (1ull << 30) ? (1ull << 30) : n, (off_t)off);
        if (w > 0) {
            p += w;
            n -= (uint64_t)w;
            off += (uint64_t)w;
        } else if (w < 0 && errno == EINTR) {
            continue;
        } else {
            return false;
        }
    }
    return true;
}

// Writes one large piece as slices from several threads (pwrite at each
// slice's offset): one thread copying into the page cache (~3.5 GB/s) is
// otherwise the limit of a file-to-file count.  write() returns when every
// slice is written.
class WritePool {
public:
    explicit WritePool(unsigned n) {
        for (unsigned i = 0; i < n; ++i) th_.emplace_back([this, i] { run(i); });
    }
    ~WritePool() {
        {
            std::lock_guard<std::mutex> l(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    bool write(int fd, const uint8_t* p, uint64_t n, uint64_t off) {
        if (th_.empty() || n < (8ull << 20)) return pwrite_all(fd, p, n, off);
        std::unique_lock<std::mutex> l(m_);
        fd_ = fd;
        p_ = p;
        n_ = n;
        off_ = off;
        ok_ = true;
        pending_ = (unsigned)th_.size();
        ++gen_;
        cv_.notify_all();
        done_.wait(l, [this] { return pending_ == 0; });
        return ok_;
    }

private:
    void run(unsigned i) {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> l(m_);
        for (;;) {
            cv_.wait(l, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            const uint64_t per = ((n_ + th_.size() - 1) / th_.size() + (1ull << 20) - 1) & ~((1ull << 20) - 1);
            const uint64_t lo = std::min<uint64_t>(n_, per * i), hi = std::min<uint64_t>(n_, lo + per);
            const int fd = fd_;
            const uint8_t* p = p_;
            const uint64_t off = off_;
            l.unlock();
            const bool r = lo >= hi || pwrite_all(fd, p + lo, hi - lo, off + lo);
            l.lock();
            if (!r) ok_ = false;
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    int fd_ = -1;
    const uint8_t* p_ = nullptr;
    uint64_t n_ = 0, off_ = 0, gen_ = 0;
    unsigned pending_ = 0;
    bool ok_ = true, stop_ = false;
};

unsigned write_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    return std::max(1u, std::min(8u, hw ? hw / 2 : 1u));
}

int write_file(const std::string& path, const uint8_t* p, uint64_t n) {
    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return io_fail("cannot open " + path + ": " + std::strerror(errno));
    const bool ok = write_all(fd, p, n);
    const int e = errno;
    if (::close(fd) != 0 || !ok) return io_fail("short write to " + path + ": " + std::strerror(ok ? errno : e));
    return KC_OK;
}

std::string with_slash(const char* d) {
    std::string s = d && *d ? d : ".";
    if (s.back() != '/') s.push_back('/');
    return s;
}

// Reads the whole input into page-locked memory (inflating gzip).
int read_fastq(const char* path, uint8_t** out, uint64_t* n) {
    *out = nullptr;
    *n = 0;
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return io_fail(std::string("Failed to open file ") + path + ": " + std::strerror(errno));
    struct stat st;
    if (fstat(fd, &st) != 0) {
        ::close(fd);
        return io_fail(std::string("Failed to get file size of ") + path);
    }
    unsigned char magic[2] = {0, 0};
    const ssize_t m = ::read(fd, magic, 2);
    const bool gz = m == 2 && magic[0] == 0x1F && magic[1] == 0x8B;
    if (!gz) {
        const uint64_t size = (uint64_t)st.st_size;
        uint8_t* buf = (uint8_t*)kc_host_alloc(size + 1);
        if (!buf) {
            ::close(fd);
            return KC_ERR_NOMEM;
        }
        uint64_t got = 0;
        if (lseek(fd, 0, SEEK_SET) != 0) {
            ::close(fd);
            kc_host_free(buf);
            return io_fail("seek failed");
        }
        while (got < size) {
            const ssize_t r = ::read(fd, buf + got, std::min<uint64_t>(size - got, 1ull << 30));
            if (r < 0 && errno == EINTR) continue;
            if (r <= 0) {
                ::close(fd);
                kc_host_free(buf);
                return io_fail(std::string("Failed to read fastq data from ") + path);
            }
            got += (uint64_t)r;
        }
        ::close(fd);
        *out = buf;
        *n = size;
        return KC_OK;
    }
    ::close(fd);
    gzFile gzf = gzopen(path, "rb");
    if (!gzf) return io_fail(std::string("Failed to open gzip file: ") + path);
    gzbuffer(gzf, 1u << 20);
    std::vector<uint8_t> tmp;
    tmp.reserve((size_t)st.st_size * 4 + 1);  // the reference also assumes ~4x (src/FastqPreReader.h:316-326)
    std::vector<uint8_t> chunk(1u << 24);
    for (;;) {
        const int r = gzread(gzf, chunk.data(), (unsigned)chunk.size());
        if (r < 0) {
            int errnum = 0;
            const char* msg = gzerror(gzf, &errnum);
            gzclose(gzf);
            return io_fail(std::string("Failed to read fastq data: ") + (msg ? msg : "gzip error"));
        }
        if (r == 0) break;
        tmp.insert(tmp.end(), chunk.begin(), chunk.begin() + r);
    }
    gzclose(gzf);
    uint8_t* buf = (uint8_t*)kc_host_alloc(tmp.size() + 1);
    if (!buf) return KC_ERR_NOMEM;
    if (!tmp.empty()) std::memcpy(buf, tmp.data(), tmp.size());
    *out = buf;
    *n = tmp.size();
    return KC_OK;
}

}  // namespace

extern "C" {

int kc_write_outputs(kc_context* ctx, const char* out_dir) {
    if (!ctx) return kc_internal_set_error(KC_ERR_INVALID, "null context");
    uint64_t low_bytes = 0, n_root = 0, counts[256];
    int rc = kc_result_sizes(ctx, &low_bytes, &n_root, counts);
    if (rc) return rc;
    const std::string dir = with_slash(out_dir);
    if (::mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST)
        return io_fail("cannot create " + dir + ": " + std::strerror(errno));
    const uint64_t rec = kc_internal_record_bytes(ctx);
    const uint64_t root_bytes = n_root * rec;
    uint8_t* host = (uint8_t*)kc_host_alloc(std::max(low_bytes, root_bytes) + 1);
    if (!host) return KC_ERR_NOMEM;
    if ((rc = kc_copy_low(ctx, host, low_bytes)) == KC_OK) rc = write_file(dir + "low.bin", host, low_bytes);
    if (rc == KC_OK && (rc = kc_copy_roots(ctx, host, root_bytes)) == KC_OK) {
        uint64_t off = 0;
        for (int r = 0; r < 256 && rc == KC_OK; ++r) {
            rc = write_file(dir + "root_" + std::to_string(r) + ".bin", host + off * rec, counts[r] * rec);
            off += counts[r];
        }
    }
    kc_host_free(host);
    return rc;
}

// Sink that writes low.bin sequentially and root_{id}.bin one after another,
// each piece in slices from a small pool of threads.
struct FileSink {
    std::string dir;
    int low_fd = -1;
    int root_fd = -1;
    int cur_root = -1;
    uint64_t low_off = 0, root_off = 0;
    WritePool pool{write_threads()};
    std::string err;
    static int call(void* u, int kind, uint32_t root, const uint8_t* data, uint64_t bytes) {
        FileSink* f = static_cast<FileSink*>(u);
        if (kind == KC_SINK_LOW) {
            if (!f->pool.write(f->low_fd, data, bytes, f->low_off)) return f->fail("short write to low.bin");
            f->low_off += bytes;
            return 0;
        }
        if ((int)root != f->cur_root) {
            if (f->root_fd >= 0 && ::close(f->root_fd) != 0) return f->fail("close failed");
            const std::string path = f->dir + "root_" + std::to_string(root) + ".bin";
            f->root_fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
            if (f->root_fd < 0) return f->fail("failed to open final drain output file " + path);
            f->cur_root = (int)root;
            f->root_off = 0;
        }
        if (bytes && !f->pool.write(f->root_fd, data, bytes, f->root_off)) return f->fail("short write to a root file");
        f->root_off += bytes;
        return 0;
    }
    int fail(const std::string& m) {
        err = m + ": " + std::strerror(errno);
        return 1;
    }
};

int kc_count_fastq(const kc_config* cfg, const char* fastq_path, const char* out_dir, kc_stats* stats) {
    if (!cfg || !fastq_path) return kc_internal_set_error(KC_ERR_INVALID, "null argument");
    FileSink fs;
    fs.dir = with_slash(out_dir ? out_dir : "./tmp/");
    if (::mkdir(fs.dir.c_str(), 0755) != 0 && errno != EEXIST)
        return io_fail("cannot create " + fs.dir + ": " + std::strerror(errno));
    kc_context* ctx = nullptr;
    int rc = kc_create(cfg, &ctx);
    if (rc) return rc;
    // a plain file streams from disk: pieces are read (parallel preads into a
    // small pinned ring) while earlier batches are counted, and the input is
    // not bounded by host memory; gzip input is inflated first
    {
        const int fd = ::open(fastq_path, O_RDONLY);
        if (fd < 0) {
            kc_destroy(ctx);
            return io_fail(std::string("Failed to open file ") + fastq_path + ": " + std::strerror(errno));
        }
        unsigned char magic[2] = {0, 0};
        struct stat st;
        const bool plain = fstat(fd, &st) == 0 && S_ISREG(st.st_mode) &&
                           !(::pread(fd, magic, 2, 0) == 2 && magic[0] == 0x1F && magic[1] == 0x8B);
        if (plain) {
            fs.low_fd = ::open((fs.dir + "low.bin").c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
            if (fs.low_fd < 0) {
                rc = io_fail("Failed to open export file: " + fs.dir + "low.bin");
            } else {
                rc = kc_internal_count_fd_stream(ctx, fd, (uint64_t)st.st_size, &FileSink::call, &fs, stats);
                if (rc == KC_ERR_IO && !fs.err.empty()) io_fail(fs.err);
                if (::close(fs.low_fd) != 0 && rc == KC_OK) rc = io_fail("close of low.bin failed");
                if (fs.root_fd >= 0 && ::close(fs.root_fd) != 0 && rc == KC_OK)
                    rc = io_fail("close of a root file failed");
            }
            ::close(fd);
            kc_destroy(ctx);
            return rc;
        }
        ::close(fd);
    }
    uint8_t* data = nullptr;
    uint64_t n = 0;
    if ((rc = read_fastq(fastq_path, &data, &n)) == KC_OK) {
        fs.low_fd = ::open((fs.dir + "low.bin").c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
        if (fs.low_fd < 0) {
            rc = io_fail("Failed to open export file: " + fs.dir + "low.bin");
        } else {
            rc = kc_count_host_stream(ctx, data, n, &FileSink::call, &fs, stats);
            if (rc == KC_ERR_IO && !fs.err.empty()) io_fail(fs.err);
            if (::close(fs.low_fd) != 0 && rc == KC_OK) rc = io_fail("close of low.bin failed");
            if (fs.root_fd >= 0 && ::close(fs.root_fd) != 0 && rc == KC_OK) rc = io_fail("close of a root file failed");
        }
        kc_host_free(data);
    }
    kc_destroy(ctx);
    return rc;
}

}  // extern "C"
