/*
 * Stand-in declarations for the netCDF-C interface, used ONLY to compile the
 * reference io_utils.c into the oracle under oracle/_ref/.  netCDF is absent
 * from this image; snapshots are never requested by the oracle runs, and every
 * function here is defined in ref_stubs.c as an abort.  Test infrastructure.
 */
#ifndef SM_SHIM_NETCDF_H
#define SM_SHIM_NETCDF_H
#include <stddef.h>

typedef int nc_type;
#define NC_CLOBBER 0
#define NC_GLOBAL (-1)
#define NC_LONG 4
#define NC_FLOAT 5
#define NC_DOUBLE 6

int nc_create(const char *path, int cmode, int *ncidp);
int nc_def_dim(int ncid, const char *name, size_t len, int *idp);
int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimidsp, int *varidp);
int nc_put_att_text(int ncid, int varid, const char *name, size_t len, const char *op);
int nc_put_att_int(int ncid, int varid, const char *name, nc_type xtype, size_t len, const int *op);
int nc_put_att_double(int ncid, int varid, const char *name, nc_type xtype, size_t len, const double *op);
int nc_put_var_double(int ncid, int varid, const double *op);
int nc_put_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, const float *op);
int nc_enddef(int ncid);
int nc_close(int ncid);
const char *nc_strerror(int ncerr);
#endif
