/* netcdf_stub.c -- implementation of oracle/refshim/netcdf.h: every call reports NC_ENOTBUILT. */
#include "netcdf.h"
int nc_open(const char *p, int m, int *n) { (void)p; (void)m; (void)n; return NC_ENOTBUILT; }
int nc_create(const char *p, int m, int *n) { (void)p; (void)m; (void)n; return NC_ENOTBUILT; }
int nc_close(int n) { (void)n; return NC_ENOTBUILT; }
int nc_enddef(int n) { (void)n; return NC_ENOTBUILT; }
int nc_def_dim(int n, const char *s, size_t l, int *i) { (void)n; (void)s; (void)l; (void)i; return NC_ENOTBUILT; }
int nc_def_var(int n, const char *s, nc_type t, int d, const int *di, int *v) { (void)n; (void)s; (void)t; (void)d; (void)di; (void)v; return NC_ENOTBUILT; }
int nc_inq_dimid(int n, const char *s, int *i) { (void)n; (void)s; (void)i; return NC_ENOTBUILT; }
int nc_inq_dimlen(int n, int d, size_t *l) { (void)n; (void)d; (void)l; return NC_ENOTBUILT; }
int nc_inq_varid(int n, const char *s, int *v) { (void)n; (void)s; (void)v; return NC_ENOTBUILT; }
int nc_inq_varndims(int n, int v, int *d) { (void)n; (void)v; (void)d; return NC_ENOTBUILT; }
int nc_inq_vardimid(int n, int v, int *d) { (void)n; (void)v; (void)d; return NC_ENOTBUILT; }
int nc_get_vara(int n, int v, const size_t *s, const size_t *c, void *p) { (void)n; (void)v; (void)s; (void)c; (void)p; return NC_ENOTBUILT; }
int nc_get_vara_float(int n, int v, const size_t *s, const size_t *c, float *p) { (void)n; (void)v; (void)s; (void)c; (void)p; return NC_ENOTBUILT; }
int nc_put_vara_float(int n, int v, const size_t *s, const size_t *c, const float *p) { (void)n; (void)v; (void)s; (void)c; (void)p; return NC_ENOTBUILT; }
int nc_put_vara_int(int n, int v, const size_t *s, const size_t *c, const int *p) { (void)n; (void)v; (void)s; (void)c; (void)p; return NC_ENOTBUILT; }
int nc_put_att_text(int n, int v, const char *s, size_t l, const char *p) { (void)n; (void)v; (void)s; (void)l; (void)p; return NC_ENOTBUILT; }
const char *nc_strerror(int e) { (void)e; return "netCDF is not available in this build"; }
