/* No-op HDF5 stand-in for building the reference CPU oracle.
 * HDF5 is not installed in this image; the oracle always runs with the save
 * location set to NULL, so checkpoint I/O is never reached.  Every call is
 * routed to a stub (h5_stub.c) that returns an invalid id / failure.
 * Test infrastructure: never part of the product library. */
#pragma once
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#define H5P_DEFAULT 0
#define H5S_ALL 0
#define H5F_ACC_TRUNC 2u
#define H5F_ACC_RDONLY 0u
#define H5T_STD_I32LE 1
#define H5T_STD_I64LE 2
#define H5T_IEEE_F64LE 3

hid_t t3ns_h5_stub_id(void);
herr_t t3ns_h5_stub_err(void);

#define H5Fcreate(...) t3ns_h5_stub_id()
#define H5Fopen(...) t3ns_h5_stub_id()
#define H5Fclose(...) t3ns_h5_stub_err()
#define H5Gcreate(...) t3ns_h5_stub_id()
#define H5Gopen(...) t3ns_h5_stub_id()
#define H5Gclose(...) t3ns_h5_stub_err()
#define H5Screate_simple(...) t3ns_h5_stub_id()
#define H5Sclose(...) t3ns_h5_stub_err()
#define H5Acreate(...) t3ns_h5_stub_id()
#define H5Aopen(...) t3ns_h5_stub_id()
#define H5Aget_type(...) t3ns_h5_stub_id()
#define H5Awrite(...) t3ns_h5_stub_err()
#define H5Aread(...) t3ns_h5_stub_err()
#define H5Aclose(...) t3ns_h5_stub_err()
#define H5Dcreate(...) t3ns_h5_stub_id()
#define H5Dopen(...) t3ns_h5_stub_id()
#define H5Dget_type(...) t3ns_h5_stub_id()
#define H5Dwrite(...) t3ns_h5_stub_err()
#define H5Dread(...) t3ns_h5_stub_err()
#define H5Dclose(...) t3ns_h5_stub_err()
