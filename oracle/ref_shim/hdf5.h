/*
 * In-memory stand-in for <hdf5.h>.  TEST INFRASTRUCTURE ONLY.
 *
 * libhdf5 is not installed here.  The reference writes its results with
 * include/wos/hdf5_io.hpp:15-338; with this header those calls record every
 * dataset (name, shape, element size, bytes) in process memory instead of a
 * file, so the reference's own runner (include/wos/runner.hpp:22-308) can be
 * executed unchanged and its fields read back by the oracle driver
 * (oracle/ref_driver.cpp, refshim_dataset()).
 */
#ifndef WOS_ORACLE_HDF5_SHIM_H
#define WOS_ORACLE_HDF5_SHIM_H

#include <stddef.h>
#include <stdint.h>
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

enum {
    H5P_DEFAULT = 0,
    H5P_FILE_ACCESS = 1,
    H5P_DATASET_XFER = 2,
    H5F_ACC_TRUNC = 2,
    H5FD_MPIO_COLLECTIVE = 1,
    H5S_SELECT_SET = 0,
    H5S_SCALAR = 0,
};

/* Native types: the value is the element size in bytes, plus a tag. */
#define H5T_NATIVE_UCHAR ((hid_t)0x101)
#define H5T_NATIVE_INT ((hid_t)0x204)
#define H5T_NATIVE_DOUBLE ((hid_t)0x308)
#define H5T_NATIVE_LLONG ((hid_t)0x408)
#define H5T_NATIVE_UINT64 ((hid_t)0x508)

hid_t H5Pcreate(hid_t cls);
herr_t H5Pclose(hid_t plist);
herr_t H5Pset_fapl_mpio(hid_t fapl, MPI_Comm comm, MPI_Info info);
herr_t H5Pset_dxpl_mpio(hid_t dxpl, int mode);
hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t file);
hid_t H5Gcreate(hid_t loc, const char *name, hid_t lcpl, hid_t gcpl, hid_t gapl);
herr_t H5Gclose(hid_t group);
hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *maxdims);
hid_t H5Screate(int kind);
herr_t H5Sclose(hid_t space);
herr_t H5Sselect_hyperslab(hid_t space, int op, const hsize_t *start, const hsize_t *stride,
                           const hsize_t *count, const hsize_t *block);
herr_t H5Sselect_none(hid_t space);
hid_t H5Dcreate(hid_t loc, const char *name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl,
                hid_t dapl);
herr_t H5Dwrite(hid_t dataset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t dxpl,
                const void *buf);
herr_t H5Dclose(hid_t dataset);

#ifdef __cplusplus
}
#endif

#endif
