/* netcdf.h -- stand-in declarations for the netCDF calls of the reference's IO module.
 * TEST INFRASTRUCTURE ONLY: every call fails with NC_ENOTBUILT; the reference harness
 * never reads or writes netCDF (it exchanges raw arrays), so these are never reached. */
#ifndef FE_REFSHIM_NETCDF_H
#define FE_REFSHIM_NETCDF_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define NC_NOERR 0
#define NC_ENOTBUILT (-128)
#define NC_NOWRITE 0
#define NC_NETCDF4 0x1000
#define NC_UNLIMITED 0L
#define NC_INT 4
#define NC_FLOAT 5
typedef int nc_type;
int nc_open(const char *path, int mode, int *ncid);
int nc_create(const char *path, int cmode, int *ncid);
int nc_close(int ncid);
int nc_enddef(int ncid);
int nc_def_dim(int ncid, const char *name, size_t len, int *idp);
int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimids, int *varidp);
int nc_inq_dimid(int ncid, const char *name, int *idp);
int nc_inq_dimlen(int ncid, int dimid, size_t *lenp);
int nc_inq_varid(int ncid, const char *name, int *varidp);
int nc_inq_varndims(int ncid, int varid, int *ndimsp);
int nc_inq_vardimid(int ncid, int varid, int *dimidsp);
int nc_get_vara(int ncid, int varid, const size_t *startp, const size_t *countp, void *ip);
int nc_get_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, float *ip);
int nc_put_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, const float *op);
int nc_put_vara_int(int ncid, int varid, const size_t *startp, const size_t *countp, const int *op);
int nc_put_att_text(int ncid, int varid, const char *name, size_t len, const char *op);
const char *nc_strerror(int ncerr);
#ifdef __cplusplus
}
#endif
#endif
