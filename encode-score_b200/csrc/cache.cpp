// es_cambi_cache: the source's CAMBI per frame kept on disk between runs, src/cache.hpp / src/cache.cpp in the same
// file format and key, so a cache written by either implementation is read by the other.
//
// The file is named by an FNV-1a hash of "cambi <version> <file size> <x0> <y0> <w> <h> <depth>" followed by the first
// and the last mebibyte of the source file (a renamed or moved source keeps its scores), under
// $XDG_CACHE_HOME/encode-score (else $HOME/.cache/encode-score). It holds 16-byte records {int64 pts; double score},
// appended every 240 scores and on close; a partial record at the end (a run stopped in mid-write) is dropped on
// open. A cache that cannot be opened behaves as an empty one that keeps nothing.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "es_internal.h"

using namespace es;

namespace {
constexpr int kCacheVersion = 1;  // raised when the CAMBI computation changes its scores
constexpr size_t kSample = 1 << 20, kFlush = 240;
constexpr int64_t kNoPts = INT64_MIN;  // a frame without a presentation timestamp

struct Record {
    int64_t pts;
    double score;
};
static_assert(sizeof(Record) == 16, "cache record layout");

uint64_t fnv1a(uint64_t h, const void *data, size_t n)
{
    for (size_t i = 0; i < n; i++) h = (h ^ ((const unsigned char *)data)[i]) * 0x100000001b3ull;
    return h;
}
}  // namespace

struct es_cambi_cache {
    std::string file;
    std::unordered_map<int64_t, double> scores;
    std::vector<Record> pending;
    int fd = -1;

    void flush()
    {
        if (fd >= 0 && !pending.empty() &&
            write(fd, pending.data(), pending.size() * sizeof(Record)) != (ssize_t)(pending.size() * sizeof(Record))) {
            close(fd);
            fd = -1;
        }
        pending.clear();
    }
    ~es_cambi_cache()
    {
        flush();
        if (fd >= 0) close(fd);
    }
};

extern "C" {

int es_cambi_cache_open(const char *path, int x0, int y0, int w, int h, int depth, const char *dir, es_cambi_cache **out)
{
    return guarded([&] {
        require(path != nullptr && out != nullptr, "es_cambi_cache_open: NULL argument");
        auto c = std::make_unique<es_cambi_cache>();
        std::string d;
        if (dir) {
            d = dir;
        } else {
            const char *xdg = std::getenv("XDG_CACHE_HOME"), *home = std::getenv("HOME");
            d = xdg && *xdg ? xdg : home ? std::string(home) + "/.cache" : "";
            if (!d.empty()) {
                mkdir(d.c_str(), 0755);
                d += "/encode-score";
            }
        }
        FILE *f = d.empty() ? nullptr : std::fopen(path, "rb");
        if (f) {
            mkdir(d.c_str(), 0755);
            std::vector<unsigned char> buf(kSample);
            std::fseek(f, 0, SEEK_END);
            const long size = std::ftell(f);
            char key[96];
            const int len = std::snprintf(key, sizeof key, "cambi %d %ld %d %d %d %d %d", kCacheVersion, size, x0, y0, w, h, depth);
            uint64_t hash = fnv1a(0xcbf29ce484222325ull, key, (size_t)len);
            for (long at : {0L, std::max(size - (long)kSample, 0L)}) {
                std::fseek(f, at, SEEK_SET);
                hash = fnv1a(hash, buf.data(), std::fread(buf.data(), 1, kSample, f));
            }
            std::fclose(f);
            char name[40];
            std::snprintf(name, sizeof name, "/%016llx.cambi", (unsigned long long)hash);
            c->file = d + name;
            c->fd = open(c->file.c_str(), O_RDWR | O_CREAT | O_APPEND, 0644);
            if (c->fd >= 0) {
                struct stat st;
                fstat(c->fd, &st);
                const off_t whole = st.st_size / (off_t)sizeof(Record) * (off_t)sizeof(Record);
                if (whole != st.st_size && ftruncate(c->fd, whole) != 0) {
                    close(c->fd);
                    c->fd = -1;
                } else {
                    std::vector<Record> records(whole / sizeof(Record));
                    if (pread(c->fd, records.data(), whole, 0) == whole)
                        for (const Record &r : records) c->scores[r.pts] = r.score;
                }
            }
        }
        *out = c.release();
    });
}

int es_cambi_cache_find(const es_cambi_cache *c, int64_t pts, double *score)
{
    if (!c || pts == kNoPts) return 0;
    const auto it = c->scores.find(pts);
    if (it == c->scores.end()) return 0;
    if (score) *score = it->second;
    return 1;
}

int es_cambi_cache_add(es_cambi_cache *c, int64_t pts, double score)
{
    return guarded([&] {
        require(c != nullptr, "es_cambi_cache_add: NULL cache");
        if (c->fd < 0 || pts == kNoPts) return;
        c->scores[pts] = score;
        c->pending.push_back({pts, score});
        if (c->pending.size() >= kFlush) c->flush();
    });
}

const char *es_cambi_cache_file(const es_cambi_cache *c) { return c ? c->file.c_str() : ""; }

void es_cambi_cache_close(es_cambi_cache *c) { delete c; }

size_t es_per_frame_json(const double *vmaf, const double *cambi, const double *cambi_source, const double *psnr_y, long n,
                         char *buf, size_t size)
{
    // src/main.cpp:767-774: {"vmaf": [...], "cambi": [...], "cambi_source": [...], "psnr_y": [...]}, 6 digits (3 for
    // PSNR), comma-separated without spaces; without VMAF figures, "vmaf": null
    std::string out = "{\"vmaf\": ";
    auto arr = [&](const double *v, int digits) {
        std::string s = "[";
        char tmp[64];
        for (long i = 0; i < n; i++) {
            std::snprintf(tmp, sizeof tmp, "%s%.*f", i ? "," : "", digits, v[i]);
            s += tmp;
        }
        return s + "]";
    };
    out += vmaf ? arr(vmaf, 6) : std::string("null");
    out += ", \"cambi\": " + arr(cambi, 6) + ", \"cambi_source\": " + arr(cambi_source, 6) + ", \"psnr_y\": " + arr(psnr_y, 3) + "}";
    if (buf && size) {
        const size_t k = std::min(size - 1, out.size());
        std::memcpy(buf, out.data(), k);
        buf[k] = '\0';
    }
    return out.size();
}

}  // extern "C"
