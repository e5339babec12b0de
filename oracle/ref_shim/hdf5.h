/*
 * hdf5.h — declares only the two HDF5 types that the reference's
 * checkpoint.h names (hid_t, hvl_t), so that headers including it compile.
 * HDF5 itself is absent on this machine; io_xdmf.c and checkpoint.c are not
 * compiled and are replaced by the no-op stubs in ref_stubs.c.
 * Test infrastructure only.
 */
#ifndef MMSREF_HDF5_H
#define MMSREF_HDF5_H
#include <stddef.h>
#include <stdint.h>
typedef int64_t hid_t;
typedef struct { size_t len; void *p; } hvl_t;
#endif
