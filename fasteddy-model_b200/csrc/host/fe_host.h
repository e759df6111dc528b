/* fe_host.h -- the repository's host C layer (parameters, grid, base state, ICs).
 * See fe_host.c for what each step restates from the reference's host modules. */
#ifndef FE_HOST_H
#define FE_HOST_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Read a FastEddy parameter file / text into the global parameter symbols.
 * Returns the number of parameter errors (0 = valid), -1 when the file is missing. */
int fe_host_load_params_file(const char *path);
int fe_host_load_params_text(const char *text);
/* Names of keys present but never queried (space separated); returns their count. */
int fe_host_unused_params(char *buf, int buflen);
/* Topography (i-major Nx*Ny, metres) used by fe_host_init instead of a topoFile. */
int fe_host_set_topography(const float *topo_ij, int nx, int ny);
int fe_host_gaussian_hill(float height, float halfwidth);
int fe_host_write_topofile(const char *path);
/* Allocate host arrays, build grid, metrics, base state, initial condition. */
int fe_host_init(unsigned long long seed);
int fe_host_set_qv_profile(float q_sfc, float q_top, float z_top);
void fe_host_cleanup(void);
size_t fe_host_field_elems(void);
size_t fe_host_plane_elems(void);
const char *fe_host_last_message(void);
/* Write the host state in the reference's raw binary output format (io_binary.c:19-132):
 * every variable the reference registers for output, in its order. path NULL or "":
 * <outPath><outFileBase>_rank_0.<tstep> from the parameter file. Returns 0 or -1. */
int fe_host_write_binary(const char *path, int tstep);
/* Write the host state as the reference's netCDF output (io_netcdf.c:392-717): dimensions time,
 * zIndex, yIndex, xIndex, the registered variables over the interior cells, in the classic
 * 64-bit-offset container. path NULL or "": <outPath><outFileBase>.<tstep>. Returns 0 or -1. */
int fe_host_write_netcdf(const char *path, int tstep);
const char *fe_host_topofile(void);

#ifdef __cplusplus
}
#endif
#endif
