// ORACLE / TEST INFRASTRUCTURE ONLY.  Runs the reference's own main() from a
// compiled shim library (oracle/_ref/libref_<solver>.so, entry
// ref_<solver>_run_main) in a plain process and writes what its HDF5 writer
// recorded (oracle/hdf5_stub/hdf5.h: cc_h5rec_*) to one binary file:
//   "CCH5REC1", int32 count, then per dataset: int32 name length, name,
//   int32 file-name length, file name, int32 rank, uint64 dims[rank],
//   int64 n_head, double head[n_head], int64 n_last, double last[n_last].
// Read by tests/golden/make_golden.py, which also reads the printed lines.
//   usage: ref_main_record <libref_X.so> <run-main symbol> <out.bin>
#include <dlfcn.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <lib.so> <symbol> <out.bin>\n", argv[0]);
        return 2;
    }
    void* h = dlopen(argv[1], RTLD_NOW);
    if (!h) {
        std::fprintf(stderr, "%s\n", dlerror());
        return 1;
    }
    auto run = reinterpret_cast<int (*)()>(dlsym(h, argv[2]));
    auto count = reinterpret_cast<int (*)()>(dlsym(h, "cc_h5rec_count"));
    auto name = reinterpret_cast<const char* (*)(int)>(dlsym(h, "cc_h5rec_name"));
    auto file = reinterpret_cast<const char* (*)(int)>(dlsym(h, "cc_h5rec_file"));
    auto rank = reinterpret_cast<int (*)(int)>(dlsym(h, "cc_h5rec_rank"));
    auto dims = reinterpret_cast<void (*)(int, unsigned long long*)>(dlsym(h, "cc_h5rec_dims"));
    auto head_len = reinterpret_cast<long long (*)(int)>(dlsym(h, "cc_h5rec_head_len"));
    auto head = reinterpret_cast<void (*)(int, double*)>(dlsym(h, "cc_h5rec_head"));
    auto last_len = reinterpret_cast<long long (*)(int)>(dlsym(h, "cc_h5rec_last_len"));
    auto last = reinterpret_cast<void (*)(int, double*)>(dlsym(h, "cc_h5rec_last"));
    if (!run || !count || !name || !file || !rank || !dims || !head_len || !head || !last_len || !last) {
        std::fprintf(stderr, "missing symbols in %s\n", argv[1]);
        return 1;
    }
    // line-buffered stdout: the reference's per-snapshot lines (t, dt, max
    // |div B|) reach a reader as they are printed, also from a run that is
    // stopped before its HDF5 write
    std::setvbuf(stdout, nullptr, _IOLBF, 0);
    if (int r = run()) return r;
    std::FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    std::fwrite("CCH5REC1", 1, 8, f);
    const int32_t n = count();
    std::fwrite(&n, 4, 1, f);
    for (int i = 0; i < n; i++) {
        for (const char* s : {name(i), file(i)}) {
            const int32_t l = (int32_t)std::strlen(s);
            std::fwrite(&l, 4, 1, f);
            std::fwrite(s, 1, l, f);
        }
        const int32_t rk = rank(i);
        std::fwrite(&rk, 4, 1, f);
        std::vector<unsigned long long> d(rk);
        dims(i, d.data());
        std::fwrite(d.data(), 8, rk, f);
        for (int part = 0; part < 2; part++) {
            const int64_t m = part == 0 ? head_len(i) : last_len(i);
            std::vector<double> v((size_t)m);
            if (part == 0) head(i, v.data()); else last(i, v.data());
            std::fwrite(&m, 8, 1, f);
            std::fwrite(v.data(), 8, (size_t)m, f);
        }
    }
    return std::fclose(f) == 0 ? 0 : 1;
}
