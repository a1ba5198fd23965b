/*
 * Stand-in for hdf5.h when building the reference's checkpoint buffer code
 * (src/IO/io_buffer.c, io_create_destroy.c, io_access.c, io_setup.c) into
 * the oracle (test infrastructure only).  Those files include hdf5.h but
 * call nothing from it; src/IO/io_hdf5.c, which does, is left out.
 */
#ifndef ORACLE_SHIM_HDF5_H
#define ORACLE_SHIM_HDF5_H
#endif
