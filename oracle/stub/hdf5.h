/* No-op stand-in for the HDF5 C API, written for this project.
 *
 * Test infrastructure only. The reference's Mesh.cpp and Field.cpp include
 * <hdf5.h> for their Save/Read routines, which the oracle never calls. This
 * header lets those two files compile without the HDF5 library: every call
 * does nothing and returns 0.
 */
#ifndef SE_ORACLE_HDF5_STUB_H
#define SE_ORACLE_HDF5_STUB_H
typedef long long hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;
enum { H5P_DEFAULT = 0, H5S_ALL = 0, H5F_ACC_TRUNC = 0, H5F_ACC_RDONLY = 0,
       H5S_SELECT_SET = 0, H5T_NATIVE_DOUBLE = 0, H5T_NATIVE_INT = 0,
       H5T_STD_I32BE = 0 };
template <typename... A> static inline hid_t H5Fcreate(A...) { return 0; }
template <typename... A> static inline hid_t H5Fopen(A...) { return 0; }
template <typename... A> static inline herr_t H5Fclose(A...) { return 0; }
template <typename... A> static inline hid_t H5Gopen(A...) { return 0; }
template <typename... A> static inline herr_t H5Gclose(A...) { return 0; }
template <typename... A> static inline hid_t H5Acreate(A...) { return 0; }
template <typename... A> static inline herr_t H5Awrite(A...) { return 0; }
template <typename... A> static inline herr_t H5Aclose(A...) { return 0; }
template <typename... A> static inline hid_t H5Screate_simple(A...) { return 0; }
template <typename... A> static inline herr_t H5Sclose(A...) { return 0; }
template <typename... A> static inline herr_t H5Sselect_all(A...) { return 0; }
template <typename... A> static inline herr_t H5Sselect_hyperslab(A...) { return 0; }
template <typename... A> static inline int H5Sget_simple_extent_dims(A...) { return 0; }
template <typename... A> static inline hid_t H5Dcreate(A...) { return 0; }
template <typename... A> static inline hid_t H5Dopen(A...) { return 0; }
template <typename... A> static inline herr_t H5Dwrite(A...) { return 0; }
template <typename... A> static inline herr_t H5Dread(A...) { return 0; }
template <typename... A> static inline hid_t H5Dget_space(A...) { return 0; }
template <typename... A> static inline herr_t H5Dclose(A...) { return 0; }
#endif
