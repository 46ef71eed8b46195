/* Minimal no-op stand-in for <hdf5.h>, used only to compile the reference
 * solvers' sources as an oracle (test infrastructure).  libhdf5 is not
 * installed in this image; the oracle never calls the writers, it only needs
 * the translation units to compile.  Every function returns a dummy handle or
 * success and touches no file. */
#ifndef CC_ORACLE_HDF5_STUB_H
#define CC_ORACLE_HDF5_STUB_H
typedef long long hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;
#define H5F_ACC_TRUNC 0
#define H5P_DEFAULT 0
#define H5S_ALL 0
#define H5T_IEEE_F64LE 0
#define H5T_NATIVE_DOUBLE 0
static inline hid_t H5Fcreate(const char*, unsigned, hid_t, hid_t) { return 1; }
static inline herr_t H5Fclose(hid_t) { return 0; }
static inline hid_t H5Screate_simple(int, const hsize_t*, const hsize_t*) { return 1; }
static inline herr_t H5Sclose(hid_t) { return 0; }
static inline hid_t H5Dcreate(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t) { return 1; }
static inline hid_t H5Dcreate2(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t) { return 1; }
static inline herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void*) { return 0; }
static inline herr_t H5Dclose(hid_t) { return 0; }
#endif
