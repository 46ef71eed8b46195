// Restart files of the solver handles (no reference counterpart: the
// reference keeps no restart file).  One file holds
//   magic (8 bytes, one per solver) | version u32 | precision u32 |
//   extents n[3] i32 (unused ones 1) | parameter-struct size u64 |
//   the handle's parameter struct | t f64 | steps i64 |
//   the state arrays as FP64, in the solver's upload order |
//   FNV-1a 64 of everything before it
// (the 2D MHD handle's own format has two extents and no third; its files keep
// that layout).  FP32 states round-trip exactly through FP64.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cc_step.h"

namespace ccb {

inline void ck_put(std::vector<unsigned char>& b, const void* src, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(src);
    b.insert(b.end(), c, c + n);
}

inline void ck_get(const std::vector<unsigned char>& b, size_t& off, void* dst, size_t n) {
    std::memcpy(dst, b.data() + off, n);
    off += n;
}

// FNV-1a, 64-bit
inline uint64_t ck_fnv1a(const unsigned char* d, size_t n) {
    uint64_t hsh = 1469598103934665603ull;
    for (size_t i = 0; i < n; i++) {
        hsh ^= d[i];
        hsh *= 1099511628211ull;
    }
    return hsh;
}

inline int ck_write_file(const char* path, const std::vector<unsigned char>& b, std::string& err) {
    FILE* fo = std::fopen(path, "wb");
    if (!fo) { err = std::string("cannot open for writing: ") + path; return CC_ERR_IO; }
    const size_t w = std::fwrite(b.data(), 1, b.size(), fo);
    const int cl = std::fclose(fo);
    if (w != b.size() || cl != 0) { err = std::string("short write: ") + path; return CC_ERR_IO; }
    return CC_OK;
}

inline int ck_read_file(const char* path, std::vector<unsigned char>& b, std::string& err) {
    FILE* fi = std::fopen(path, "rb");
    if (!fi) { err = std::string("cannot open for reading: ") + path; return CC_ERR_IO; }
    unsigned char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), fi)) > 0) b.insert(b.end(), chunk, chunk + got);
    const bool rerr = std::ferror(fi) != 0;
    std::fclose(fi);
    if (rerr) { err = std::string("read error: ") + path; return CC_ERR_IO; }
    return CC_OK;
}

constexpr uint32_t CK3_VERSION = 1;

// What a restart file holds besides its arrays.
struct CkMeta {
    uint32_t precision = 0;
    int32_t n[3] = {1, 1, 1};
    double t = 0.0;
    long long steps = 0;
};

inline int ck3_save(const char* path, const char magic[9], const CkMeta& m, const void* params, size_t pbytes,
                    const std::vector<std::vector<double>>& f, std::string& err) {
    std::vector<unsigned char> b;
    ck_put(b, magic, 8);
    const uint32_t ver = CK3_VERSION;
    const uint64_t pb = pbytes;
    ck_put(b, &ver, 4); ck_put(b, &m.precision, 4); ck_put(b, m.n, 12);
    ck_put(b, &pb, 8); ck_put(b, params, pbytes);
    ck_put(b, &m.t, 8); ck_put(b, &m.steps, 8);
    for (const auto& a : f) ck_put(b, a.data(), sizeof(double) * a.size());
    const uint64_t sum = ck_fnv1a(b.data(), b.size());
    ck_put(b, &sum, 8);
    return ck_write_file(path, b, err);
}

// Reads a file written by ck3_save with the same magic and parameter-struct
// size; fills m, params (pbytes) and the arrays, whose sizes follow from the
// file's extents through sizes_of(n).  CC_ERR_ARG for a wrong magic, version,
// checksum or size; CC_ERR_IO when the file cannot be read.
template <class SizesOf>
inline int ck3_load(const char* path, const char magic[9], CkMeta& m, void* params, size_t pbytes,
                    const SizesOf& sizes_of, std::vector<std::vector<double>>& f, std::string& err) {
    std::vector<unsigned char> b;
    if (int r = ck_read_file(path, b, err)) return r;
    const size_t head = 8 + 4 + 4 + 12 + 8;
    if (b.size() < head + 8 || std::memcmp(b.data(), magic, 8) != 0) {
        err = "not a checkpoint of this solver (magic)";
        return CC_ERR_ARG;
    }
    uint64_t sum = 0;
    std::memcpy(&sum, b.data() + b.size() - 8, 8);
    if (sum != ck_fnv1a(b.data(), b.size() - 8)) { err = "checkpoint checksum mismatch"; return CC_ERR_ARG; }
    size_t off = 8;
    uint32_t ver = 0;
    uint64_t pb = 0;
    ck_get(b, off, &ver, 4); ck_get(b, off, &m.precision, 4); ck_get(b, off, m.n, 12);
    ck_get(b, off, &pb, 8);
    if (ver != CK3_VERSION || pb != pbytes || b.size() < off + pb + 16 + 8) {
        err = "checkpoint version mismatch";
        return CC_ERR_ARG;
    }
    ck_get(b, off, params, pbytes);
    ck_get(b, off, &m.t, 8); ck_get(b, off, &m.steps, 8);
    if (m.n[0] < 1 || m.n[1] < 1 || m.n[2] < 1) { err = "checkpoint extents invalid"; return CC_ERR_ARG; }
    const std::vector<size_t> sz = sizes_of(m.n);
    size_t need = off + 8;
    for (size_t k : sz) need += sizeof(double) * k;
    if (need != b.size()) { err = "checkpoint size does not match its grid"; return CC_ERR_ARG; }
    f.clear();
    for (size_t k : sz) {
        f.emplace_back(k);
        ck_get(b, off, f.back().data(), sizeof(double) * k);
    }
    return CC_OK;
}

}  // namespace ccb
