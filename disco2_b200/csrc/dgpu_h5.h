/* HDF5 files of 64-bit float datasets in the root group, without an HDF5
 * library: the subset that the reference's checkpoints use
 * (src/IO/io_hdf5.c:15-266).  Host code only. */
#ifndef DGPU_H5_H
#define DGPU_H5_H
#include <stdint.h>

#define H5_MAX_RANK 2

typedef struct {
  const char *name;
  int rank;                    /* 1 or 2 */
  uint64_t dims[H5_MAX_RANK];
  const double *data;          /* row-major, dims[0] * dims[1] values */
} h5_dataset;

/* Writes a new file holding datasets ds[0..n) (n <= 8).  0 on success; on
 * failure a message in err and -1 (bad arguments, I/O) or -2 (no memory). */
int h5_write(const char *path, const h5_dataset *ds, int n, char *err, int errlen);

/* Finds dataset `name` in the root group of `path`: its rank and dims, and,
 * when data is not NULL, rows [row0, row0 + nrows) of its values (rows of
 * dims[1] values for rank 2).  0 on success, -1 with a message in err. */
int h5_read(const char *path, const char *name, int *rank, uint64_t *dims, double *data,
            uint64_t row0, uint64_t nrows, char *err, int errlen);

#endif
