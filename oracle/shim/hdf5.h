/*
 * Type-only HDF5 stand-in for compiling the reference solver as the CPU oracle
 * (test infrastructure).  The oracle flag sets leave OUTPUT_H5 undefined and
 * src/output_h5.c out of the link, so only the handle types of the reference
 * headers (src/common_object.h:16 includes <hdf5.h> unconditionally) are needed.
 */
#ifndef CH4_ORACLE_HDF5_STUB_H
#define CH4_ORACLE_HDF5_STUB_H
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
#endif
