// Versioned on-disk caches of a build's host work, in the formats of the reference:
//
// 1. The operator-table cache (fmm-tables/src/cache.rs:1-90): one file per (kind, degree,
//    precision) in a directory the caller supplies, `<kind>-p<pp>-<precision>-c<convention>-
//    v<format>.bin`, a 44-byte little-endian header (magic NDFMMTAB, format version 1,
//    convention version 4 of nd-fmm-math (fmm-math/src/lib.rs:73), kind code, p, bits per
//    value, payload length, FNV-1a 64 checksum of the payload) and the payload: the matrices
//    one after another, each column-major (M2M and L2L: 8 n^2 values, M2L: 316 n^2).  A
//    store writes a uniquely named temporary file in the directory, the header last,
//    syncs it and renames it over the final name; a load checks header length, magic,
//    versions, key, payload length, checksum and structure in that order and rejects a
//    file that fails any.  Files written here and by the reference are interchangeable.
//    The Helmholtz tables of one level (which the reference does not cache) use the same
//    header under kind codes of their own, 65 (M2L, 316 real 2n x n matrices) and 66
//    (M2M then L2L, 16 real 2n x n matrices), with the level's wavenumber k_l (boxes of
//    half-width 1) in the file name as the hexadecimal bits of the double.
// 2. The tuning cache (the reference's TuningCache, fmm-exec/src/tune.rs:118-140): one
//    text file per (device, precision, p): a magic line, the FNV-1a checksum of the body,
//    the key and versions, then one line per decision (`<gradients> <decision> <value>`).
//    Written and rejected under the same rules.
#include <fcntl.h>
#include <unistd.h>

#include <atomic>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "plan.hpp"

namespace fmmb {

namespace {

constexpr char kMagic[8] = {'N', 'D', 'F', 'M', 'M', 'T', 'A', 'B'};
constexpr uint32_t kFormatVersion = 1;
constexpr uint32_t kConventionVersion = 4;  // nd-fmm-math's CONVENTION_VERSION
constexpr size_t kHeaderLen = 44;
constexpr uint64_t kFnvOffset = 0xcbf29ce484222325ULL;
constexpr uint64_t kFnvPrime = 0x00000100000001b3ULL;

uint64_t fnv1a(uint64_t h, const unsigned char* p, size_t n) {
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= kFnvPrime;
    }
    return h;
}

void put_u32(unsigned char* o, uint32_t v) {
    for (int i = 0; i < 4; ++i) o[i] = (unsigned char)(v >> (8 * i));
}
void put_u64(unsigned char* o, uint64_t v) {
    for (int i = 0; i < 8; ++i) o[i] = (unsigned char)(v >> (8 * i));
}
uint32_t get_u32(const unsigned char* o) {
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) v |= (uint32_t)o[i] << (8 * i);
    return v;
}
uint64_t get_u64(const unsigned char* o) {
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v |= (uint64_t)o[i] << (8 * i);
    return v;
}

const char* kind_name(int kind) {
    switch (kind) {
        case kTableM2m: return "m2m";
        case kTableL2l: return "l2l";
        case kTableM2l: return "m2l";
        case kTableHelmholtzM2l: return "hh-m2l";
        case kTableHelmholtzOctant: return "hh-octant";
        default: return "unknown";
    }
}

std::atomic<uint64_t> g_counter{0};

// writes `bytes` to dir/name through a unique temporary file, synced, then renamed
bool atomic_write(const std::string& dir, const std::string& name, const std::vector<unsigned char>& head,
                  const std::vector<unsigned char>& body, std::string* why) {
    const std::string tmp = dir + "/." + name + "." + std::to_string((long)getpid()) + "-" +
                            std::to_string((unsigned long long)g_counter.fetch_add(1)) + ".tmp";
    const int fd = ::open(tmp.c_str(), O_WRONLY | O_CREAT | O_EXCL, 0644);
    if (fd < 0) {
        if (why) *why = tmp + ": " + std::strerror(errno);
        return false;
    }
    auto write_at = [&](const std::vector<unsigned char>& b, off_t at) {
        size_t done = 0;
        while (done < b.size()) {
            const ssize_t w = ::pwrite(fd, b.data() + done, b.size() - done, at + (off_t)done);
            if (w <= 0) return false;
            done += (size_t)w;
        }
        return true;
    };
    // the body first, the header (with the magic) last
    bool ok = write_at(body, (off_t)head.size()) && write_at(head, 0) && ::fsync(fd) == 0;
    ok = (::close(fd) == 0) && ok;
    if (ok) ok = ::rename(tmp.c_str(), (dir + "/" + name).c_str()) == 0;
    if (!ok) {
        if (why) *why = tmp + ": " + std::strerror(errno);
        ::unlink(tmp.c_str());
    }
    return ok;
}

}  // namespace

std::string table_cache_file_name(int kind, int p, double k) {
    char buf[160];
    if (kind == kTableHelmholtzM2l || kind == kTableHelmholtzOctant) {
        uint64_t bits;
        std::memcpy(&bits, &k, sizeof bits);
        std::snprintf(buf, sizeof buf, "%s-p%02d-k%016llx-f64-c%u-v%u.bin", kind_name(kind), p,
                      (unsigned long long)bits, kConventionVersion, kFormatVersion);
    } else {
        std::snprintf(buf, sizeof buf, "%s-p%02d-f64-c%u-v%u.bin", kind_name(kind), p, kConventionVersion,
                      kFormatVersion);
    }
    return buf;
}

bool table_cache_store(const std::string& dir, int kind, int p, double k, const std::vector<double>& values,
                       std::string* why) {
    std::vector<unsigned char> body(values.size() * 8);
    for (size_t i = 0; i < values.size(); ++i) {
        uint64_t b;
        std::memcpy(&b, &values[i], 8);
        put_u64(body.data() + 8 * i, b);
    }
    std::vector<unsigned char> head(kHeaderLen, 0);
    std::memcpy(head.data(), kMagic, 8);
    put_u32(head.data() + 8, kFormatVersion);
    put_u32(head.data() + 12, kConventionVersion);
    put_u32(head.data() + 16, (uint32_t)kind);
    put_u32(head.data() + 20, (uint32_t)p);
    put_u32(head.data() + 24, 64);
    put_u64(head.data() + 28, (uint64_t)body.size());
    put_u64(head.data() + 36, fnv1a(kFnvOffset, body.data(), body.size()));
    return atomic_write(dir, table_cache_file_name(kind, p, k), head, body, why);
}

bool table_cache_load(const std::string& dir, int kind, int p, double k, size_t count, std::vector<double>& values,
                      std::string* why) {
    const std::string path = dir + "/" + table_cache_file_name(kind, p, k);
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        if (why) *why = "missing";
        return false;
    }
    std::vector<unsigned char> all((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    auto reject = [&](const std::string& what) {
        if (why) *why = path + ": " + what;
        return false;
    };
    if (all.size() < kHeaderLen) return reject("shorter than the header");
    if (std::memcmp(all.data(), kMagic, 8) != 0) return reject("wrong magic bytes");
    if (get_u32(all.data() + 8) != kFormatVersion) return reject("format version");
    if (get_u32(all.data() + 12) != kConventionVersion) return reject("convention version");
    if (get_u32(all.data() + 16) != (uint32_t)kind || get_u32(all.data() + 20) != (uint32_t)p ||
        get_u32(all.data() + 24) != 64)
        return reject("key (kind, p, precision)");
    const uint64_t len = get_u64(all.data() + 28);
    if (len != all.size() - kHeaderLen) return reject("payload length");
    if (get_u64(all.data() + 36) != fnv1a(kFnvOffset, all.data() + kHeaderLen, (size_t)len))
        return reject("checksum");
    if (len != 8 * (uint64_t)count) return reject("structure: " + std::to_string(len / 8) + " values");
    values.resize(count);
    for (size_t i = 0; i < count; ++i) {
        const uint64_t b = get_u64(all.data() + kHeaderLen + 8 * i);
        std::memcpy(&values[i], &b, 8);
    }
    return true;
}

// ---- tuning cache ----

namespace {
constexpr const char* kTuningMagic = "fmm-b200 tuning cache";
constexpr int kTuningFormat = 1;
constexpr int kCandidateSet = 1;  // the candidate shapes: P2P warps {1, 2, 4}, L2P/M2P blocks {32, 64, 128}

std::string tuning_body(const TuningKey& key, const std::map<std::string, int>& entries) {
    std::ostringstream b;
    b << "format " << kTuningFormat << "\nconvention " << kConventionVersion << "\ncandidates " << kCandidateSet
      << "\nbackend cuda\ndevice " << key.device << "\ncompiler " << key.compiler << "\nprecision "
      << key.precision << "\np " << key.p << "\n";
    for (const auto& e : entries) b << "entry " << e.first << " " << e.second << "\n";
    return b.str();
}
}  // namespace

std::string tuning_cache_file_name(const TuningKey& key) {
    std::string slug;
    bool dash = false;
    for (char c : key.device) {
        const bool an = (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9');
        if (an) {
            slug += (char)((c >= 'A' && c <= 'Z') ? c - 'A' + 'a' : c);
            dash = false;
        } else if (!dash && !slug.empty()) {
            slug += '-';
            dash = true;
        }
    }
    while (!slug.empty() && slug.back() == '-') slug.pop_back();
    const std::string id = key.device + "\n" + key.compiler;
    uint64_t h = fnv1a(kFnvOffset, reinterpret_cast<const unsigned char*>(id.data()), id.size());
    char buf[256];
    std::snprintf(buf, sizeof buf, "tuning-cuda-%s-%08x-%s-p%02d.txt", slug.c_str(), (unsigned)(uint32_t)h,
                  key.precision.c_str(), key.p);
    return buf;
}

bool tuning_cache_load(const std::string& dir, const TuningKey& key, std::map<std::string, int>& entries,
                       std::string* why) {
    const std::string path = dir + "/" + tuning_cache_file_name(key);
    std::ifstream in(path);
    if (!in) {
        if (why) *why = "missing";
        return false;
    }
    std::string magic, sum_line;
    std::getline(in, magic);
    std::getline(in, sum_line);
    std::string body((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    auto reject = [&](const std::string& what) {
        if (why) *why = path + ": " + what;
        return false;
    };
    if (magic != kTuningMagic) return reject("wrong magic line");
    unsigned long long sum = 0;
    if (std::sscanf(sum_line.c_str(), "checksum %llx", &sum) != 1) return reject("no checksum line");
    if (sum != fnv1a(kFnvOffset, reinterpret_cast<const unsigned char*>(body.data()), body.size()))
        return reject("checksum");
    std::map<std::string, int> got;
    const std::string expect_head = tuning_body(key, {});
    if (body.compare(0, expect_head.size(), expect_head) != 0) return reject("key or versions differ (stale)");
    std::istringstream rest(body.substr(expect_head.size()));
    std::string line;
    while (std::getline(rest, line)) {
        if (line.empty()) continue;
        std::istringstream ls(line);
        std::string word, name;
        int value = 0;
        if (!(ls >> word >> name >> value) || word != "entry") return reject("a malformed line `" + line + "`");
        got[name] = value;
    }
    entries = got;
    return true;
}

bool tuning_cache_store(const std::string& dir, const TuningKey& key, const std::map<std::string, int>& entries,
                        std::string* why) {
    const std::string body = tuning_body(key, entries);
    char sum[64];
    std::snprintf(sum, sizeof sum, "checksum %016llx\n",
                  (unsigned long long)fnv1a(kFnvOffset, reinterpret_cast<const unsigned char*>(body.data()),
                                            body.size()));
    const std::string head = std::string(kTuningMagic) + "\n" + sum;
    return atomic_write(dir, tuning_cache_file_name(key), std::vector<unsigned char>(head.begin(), head.end()),
                        std::vector<unsigned char>(body.begin(), body.end()), why);
}

}  // namespace fmmb
