// Output helpers of the drop-in drivers: NumPy .npy files (v1.0 header,
// little-endian float64), written whole or grown one snapshot at a time.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace ccmain {

// NumPy .npy v1.0 header for little-endian float64 of the given shape, padded
// with spaces to 128 bytes so that it can be rewritten in place.
inline std::string npy_header(const std::vector<long long>& shape) {
    std::string dict = "{'descr': '<f8', 'fortran_order': False, 'shape': (";
    for (size_t k = 0; k < shape.size(); k++) {
        dict += std::to_string(shape[k]);
        dict += (shape.size() == 1) ? "," : (k + 1 < shape.size() ? ", " : "");
    }
    dict += "), }";
    const size_t total = 128, pre = 10;
    while (pre + dict.size() + 1 < total) dict += ' ';
    dict += '\n';
    std::string h = "\x93NUMPY";
    h += (char)1;
    h += (char)0;
    const uint16_t len = (uint16_t)dict.size();
    h += (char)(len & 0xff);
    h += (char)(len >> 8);
    return h + dict;
}

inline bool write_npy(const std::string& path, const std::vector<long long>& shape, const double* data, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const std::string h = npy_header(shape);
    bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    ok = ok && std::fwrite(data, sizeof(double), n, f) == n;
    return std::fclose(f) == 0 && ok;
}

// A (Nt, ...) field file appended one snapshot at a time; the header is
// rewritten with the final Nt by finish().
struct SeriesFile {
    FILE* f = nullptr;
    long long nt = 0;
    std::vector<long long> frame;   // shape of one snapshot
    bool open(const std::string& path, const std::vector<long long>& shape) {
        frame = shape;
        f = std::fopen(path.c_str(), "wb");
        if (!f) return false;
        std::vector<long long> s{0};
        s.insert(s.end(), frame.begin(), frame.end());
        const std::string h = npy_header(s);
        return std::fwrite(h.data(), 1, h.size(), f) == h.size();
    }
    bool append(const double* d) {
        size_t n = 1;
        for (long long e : frame) n *= (size_t)e;
        if (std::fwrite(d, sizeof(double), n, f) != n) return false;
        nt++;
        return true;
    }
    bool finish() {
        std::vector<long long> s{nt};
        s.insert(s.end(), frame.begin(), frame.end());
        const std::string h = npy_header(s);
        bool ok = std::fseek(f, 0, SEEK_SET) == 0 && std::fwrite(h.data(), 1, h.size(), f) == h.size();
        ok = (std::fclose(f) == 0) && ok;
        f = nullptr;
        return ok;
    }
};

}  // namespace ccmain
