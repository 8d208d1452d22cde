// es_cambi_cache: the source's CAMBI per frame, kept on disk between runs, so a later run against the same source
// reads it instead of computing it again (the reference's CambiCache, src/cache.hpp:9-29, src/cache.cpp:13-88).
//
// The on-disk format is shared with the reference, so a cache written by either program is read by the other:
//  * directory: the caller's, else $XDG_CACHE_HOME/encode-score, else $HOME/.cache/encode-score;
//  * file name: 16 lower-case hex digits of a 64-bit FNV-1a hash, then ".cambi". The hash runs over the key text
//    "cambi <version> <source bytes> <x0> <y0> <w> <h> <depth>" (version 1), then the source's first min(size, 1 MiB)
//    bytes, then the min(size, 1 MiB) bytes that start at max(size - 1 MiB, 0) (a small file is hashed twice);
//  * content: records of 16 bytes, {int64 pts; double score} in host byte order, appended in batches of 240 and on
//    close. A length that is not a whole number of records (a run stopped in mid-write) loses its partial last
//    record when the cache is opened; a later record of the same pts wins over an earlier one.
// A cache that cannot be opened (no directory, an unreadable source, a failed write) behaves as an empty one that keeps
// nothing. Frames without a timestamp (INT64_MIN) are never looked up or stored.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "es_internal.h"

using namespace es;

namespace {

constexpr int kFormatVersion = 1;             // raised when the CAMBI computation changes its scores
constexpr off_t kSampleBytes = 1 << 20;       // bytes of the source hashed at its start and at its end
constexpr size_t kRecordsPerWrite = 240;
constexpr int64_t kNoTimestamp = INT64_MIN;

struct ScoreRecord {
    int64_t pts;
    double score;
};
static_assert(sizeof(ScoreRecord) == 16, "the cache's records are 16 bytes");

// 64-bit FNV-1a, fed in pieces.
struct Fnv1a64 {
    uint64_t state = 0xcbf29ce484222325ull;
    void feed(const void *bytes, size_t n)
    {
        const unsigned char *p = static_cast<const unsigned char *>(bytes);
        for (const unsigned char *end = p + n; p != end; ++p) state = (state ^ *p) * 0x100000001b3ull;
    }
};

// Reads exactly n bytes at `at` unless the file ends first; returns the bytes read, or -1 on an error.
ssize_t read_at(int fd, unsigned char *dst, size_t n, off_t at)
{
    size_t got = 0;
    while (got < n) {
        const ssize_t r = pread(fd, dst + got, n - got, at + (off_t)got);
        if (r < 0) return -1;
        if (r == 0) break;
        got += (size_t)r;
    }
    return (ssize_t)got;
}

// The cache file's name for a source, or "" when the source cannot be read.
std::string cache_name(const char *source, int x0, int y0, int w, int h, int depth)
{
    const int fd = open(source, O_RDONLY);
    if (fd < 0) return "";
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        return "";
    }
    const off_t size = st.st_size;
    // both samples in one buffer, hashed after the key text
    const off_t head = size < kSampleBytes ? size : kSampleBytes;
    const off_t tail_at = size > kSampleBytes ? size - kSampleBytes : 0;
    std::vector<unsigned char> sample((size_t)(2 * head));
    const ssize_t a = read_at(fd, sample.data(), (size_t)head, 0);
    const ssize_t b = read_at(fd, sample.data() + head, (size_t)head, tail_at);
    close(fd);
    if (a < 0 || b < 0) return "";
    const std::string key = "cambi " + std::to_string(kFormatVersion) + " " + std::to_string((long long)size) + " " +
                            std::to_string(x0) + " " + std::to_string(y0) + " " + std::to_string(w) + " " +
                            std::to_string(h) + " " + std::to_string(depth);
    Fnv1a64 hash;
    hash.feed(key.data(), key.size());
    hash.feed(sample.data(), (size_t)a);
    hash.feed(sample.data() + head, (size_t)b);
    char hex[17];
    std::snprintf(hex, sizeof hex, "%016llx", (unsigned long long)hash.state);
    return std::string(hex) + ".cambi";
}

std::string default_directory()
{
    const char *xdg = std::getenv("XDG_CACHE_HOME");
    if (xdg && *xdg) return xdg;
    const char *home = std::getenv("HOME");
    return home ? std::string(home) + "/.cache" : "";
}

}  // namespace

struct es_cambi_cache {
    std::string path;                              // "" when there is no cache file
    int fd = -1;                                   // open for appending while the cache stores
    std::unordered_map<int64_t, double> known;     // every score read or added
    std::vector<ScoreRecord> unwritten;

    // Reads the records of an opened file, dropping a partial last one. False when the file cannot be used.
    bool load()
    {
        struct stat st;
        if (fstat(fd, &st) != 0) return false;
        const off_t whole = st.st_size - st.st_size % (off_t)sizeof(ScoreRecord);
        if (whole != st.st_size && ftruncate(fd, whole) != 0) return false;
        std::vector<ScoreRecord> records((size_t)(whole / (off_t)sizeof(ScoreRecord)));
        if (read_at(fd, reinterpret_cast<unsigned char *>(records.data()), (size_t)whole, 0) != (ssize_t)whole) return false;
        for (const ScoreRecord &r : records) known[r.pts] = r.score;
        return true;
    }
    void stop_storing()
    {
        if (fd >= 0) close(fd);
        fd = -1;
    }
    void write_out()
    {
        if (unwritten.empty()) return;
        const size_t bytes = unwritten.size() * sizeof(ScoreRecord);
        if (fd >= 0 && write(fd, unwritten.data(), bytes) != (ssize_t)bytes) stop_storing();
        unwritten.clear();
    }
    ~es_cambi_cache()
    {
        write_out();
        stop_storing();
    }
};

extern "C" {

int es_cambi_cache_open(const char *path, int x0, int y0, int w, int h, int depth, const char *dir, es_cambi_cache **out)
{
    return guarded([&] {
        require(path != nullptr && out != nullptr, "es_cambi_cache_open: NULL argument");
        auto c = std::make_unique<es_cambi_cache>();
        std::string where;
        if (dir) {
            where = dir;
        } else {
            const std::string base = default_directory();
            if (!base.empty()) {
                mkdir(base.c_str(), 0755);
                where = base + "/encode-score";
            }
        }
        const std::string name = where.empty() ? "" : cache_name(path, x0, y0, w, h, depth);
        if (!name.empty()) {
            mkdir(where.c_str(), 0755);
            c->path = where + "/" + name;
            c->fd = open(c->path.c_str(), O_RDWR | O_CREAT | O_APPEND, 0644);
            if (c->fd >= 0 && !c->load()) {
                c->known.clear();
                c->stop_storing();
            }
        }
        *out = c.release();
    });
}

int es_cambi_cache_find(const es_cambi_cache *c, int64_t pts, double *score)
{
    if (!c || pts == kNoTimestamp) return 0;
    const auto it = c->known.find(pts);
    if (it == c->known.end()) return 0;
    if (score) *score = it->second;
    return 1;
}

int es_cambi_cache_add(es_cambi_cache *c, int64_t pts, double score)
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_cache_add: NULL cache");
        if (c->fd < 0 || pts == kNoTimestamp) return;
        c->known[pts] = score;
        c->unwritten.push_back(ScoreRecord{pts, score});
        if (c->unwritten.size() == kRecordsPerWrite) c->write_out();
    });
}

const char *es_cambi_cache_file(const es_cambi_cache *c) { return c ? c->path.c_str() : ""; }

void es_cambi_cache_close(es_cambi_cache *c) { delete c; }

}  // extern "C"
