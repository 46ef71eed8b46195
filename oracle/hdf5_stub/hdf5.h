/* Recording stand-in for <hdf5.h>, used only to compile the reference
 * solvers' sources as an oracle (test infrastructure).  libhdf5 is not
 * installed in this image.  Instead of writing a file, the functions the
 * reference's writers call record each dataset in memory: its name, its
 * dimensions (from the dataspace it was created with) and, from the buffer
 * passed to H5Dwrite, every value of a rank-1 dataset and, of a dataset of
 * rank >= 2 (frames along the first axis), the first CC_H5REC_KEEP frames and
 * the last one.  The shim that includes this header exports the record
 * through the cc_h5rec_* C functions at the end; nothing touches a file. */
#ifndef CC_ORACLE_HDF5_STUB_H
#define CC_ORACLE_HDF5_STUB_H
#include <cstring>
#include <string>
#include <vector>

typedef long long hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;
#define H5F_ACC_TRUNC 0
#define H5P_DEFAULT 0
#define H5S_ALL 0
#define H5T_IEEE_F64LE 0
#define H5T_NATIVE_DOUBLE 0

#ifndef CC_H5REC_KEEP
#define CC_H5REC_KEEP 2
#endif

namespace cc_h5rec {
struct Dataset {
    std::string file, name;
    std::vector<hsize_t> dims;
    std::vector<double> head;   // rank 1: all values; rank >= 2: the first CC_H5REC_KEEP frames
    std::vector<double> last;   // rank >= 2: the last frame
};
inline std::vector<Dataset>& sets() { static std::vector<Dataset> s; return s; }
inline std::vector<std::vector<hsize_t>>& spaces() { static std::vector<std::vector<hsize_t>> s; return s; }
inline std::vector<std::string>& files() { static std::vector<std::string> f; return f; }
}  // namespace cc_h5rec

static inline hid_t H5Fcreate(const char* name, unsigned, hid_t, hid_t) {
    cc_h5rec::files().push_back(name ? name : "");
    return (hid_t)cc_h5rec::files().size();
}
static inline herr_t H5Fclose(hid_t) { return 0; }
static inline hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t*) {
    cc_h5rec::spaces().emplace_back(dims, dims + rank);
    return (hid_t)cc_h5rec::spaces().size();
}
static inline herr_t H5Sclose(hid_t) { return 0; }
static inline hid_t H5Dcreate(hid_t file, const char* name, hid_t, hid_t space, hid_t, hid_t, hid_t) {
    cc_h5rec::Dataset d;
    if (file >= 1 && (size_t)file <= cc_h5rec::files().size()) d.file = cc_h5rec::files()[file - 1];
    d.name = name ? name : "";
    if (space >= 1 && (size_t)space <= cc_h5rec::spaces().size()) d.dims = cc_h5rec::spaces()[space - 1];
    cc_h5rec::sets().push_back(d);
    return (hid_t)cc_h5rec::sets().size();
}
static inline hid_t H5Dcreate2(hid_t file, const char* name, hid_t t, hid_t space, hid_t a, hid_t b, hid_t c) {
    return H5Dcreate(file, name, t, space, a, b, c);
}
static inline herr_t H5Dwrite(hid_t ds, hid_t, hid_t, hid_t, hid_t, const void* buf) {
    if (ds < 1 || (size_t)ds > cc_h5rec::sets().size() || !buf) return -1;
    cc_h5rec::Dataset& d = cc_h5rec::sets()[ds - 1];
    const double* a = static_cast<const double*>(buf);
    size_t total = 1;
    for (hsize_t n : d.dims) total *= (size_t)n;
    if (d.dims.size() <= 1) {
        d.head.assign(a, a + total);
    } else {
        const size_t nf = (size_t)d.dims[0], frame = nf ? total / nf : 0;
        const size_t keep = nf < (size_t)CC_H5REC_KEEP ? nf : (size_t)CC_H5REC_KEEP;
        d.head.assign(a, a + keep * frame);
        if (nf) d.last.assign(a + (nf - 1) * frame, a + nf * frame);
    }
    return 0;
}
static inline herr_t H5Dclose(hid_t) { return 0; }

/* the record, for the tests (one copy per shim library) */
extern "C" {
__attribute__((visibility("default"))) int cc_h5rec_count() { return (int)cc_h5rec::sets().size(); }
__attribute__((visibility("default"))) const char* cc_h5rec_name(int i) { return cc_h5rec::sets()[i].name.c_str(); }
__attribute__((visibility("default"))) const char* cc_h5rec_file(int i) { return cc_h5rec::sets()[i].file.c_str(); }
__attribute__((visibility("default"))) int cc_h5rec_rank(int i) { return (int)cc_h5rec::sets()[i].dims.size(); }
__attribute__((visibility("default"))) void cc_h5rec_dims(int i, unsigned long long* out) {
    for (size_t k = 0; k < cc_h5rec::sets()[i].dims.size(); k++) out[k] = cc_h5rec::sets()[i].dims[k];
}
__attribute__((visibility("default"))) long long cc_h5rec_head_len(int i) {
    return (long long)cc_h5rec::sets()[i].head.size();
}
__attribute__((visibility("default"))) void cc_h5rec_head(int i, double* out) {
    const auto& v = cc_h5rec::sets()[i].head;
    if (!v.empty()) std::memcpy(out, v.data(), sizeof(double) * v.size());
}
__attribute__((visibility("default"))) long long cc_h5rec_last_len(int i) {
    return (long long)cc_h5rec::sets()[i].last.size();
}
__attribute__((visibility("default"))) void cc_h5rec_last(int i, double* out) {
    const auto& v = cc_h5rec::sets()[i].last;
    if (!v.empty()) std::memcpy(out, v.data(), sizeof(double) * v.size());
}
__attribute__((visibility("default"))) void cc_h5rec_clear() {
    cc_h5rec::sets().clear();
    cc_h5rec::spaces().clear();
    cc_h5rec::files().clear();
}
}
#endif
