/* ref_io.c -- TEST INFRASTRUCTURE ONLY: writes one output file with the reference's own binary
 * output code (SRC/IO/io_binary.c:19-132), so the repository's writer can be checked byte for
 * byte against it. Host modules only: no CUDA call is made, so this runs without a GPU.
 *
 * Follows the reference's host initialisation order (SRC/FEMAIN/FastEddy.c:72-253, without the
 * FECUDA module), which registers the output variables, then overwrites every registered array
 * with the raw float32 files <INDIR>/<name>.bin and writes <outPath><outFileBase>_rank_0.<TSTEP>.
 *
 * usage: fe_ref_io PARAMFILE INDIR TSTEP
 *        fe_ref_io PARAMFILE OUTDIR dump
 *
 * dump runs the reference's own initial-condition path instead (FastEddy.c:109 seeding,
 * gridSecondaryPreparations, hydro_coreSetBaseState: FastEddy.c:223-238, grid.c:386-803,
 * hydro_core.c:1053-1250) and writes the host inputs of the CUDA path as raw float32 files
 * <OUTDIR>/<name>.bin: coordinates, metrics, base state, initial state and surface arrays.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fempi.h>
#include <parameters.h>
#include <mem_utils.h>
#include <io.h>
#include <grid.h>
#include <hydro_core.h>
#include <time_integration.h>

int ioWriteBinaryoutFileSingleTime(int tstep, int Nx, int Ny, int Nz, int Nh);

static int read_into(const char *dir, const char *name, float *dst, size_t n) {
  char path[2048];
  FILE *f;
  size_t got;
  snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  f = fopen(path, "rb");
  if (!f) {
    fprintf(stderr, "ref_io: missing %s\n", path);
    return -1;
  }
  got = fread(dst, sizeof(float), n, f);
  fclose(f);
  if (got != n) {
    fprintf(stderr, "ref_io: %s has %zu floats, expected %zu\n", path, got, n);
    return -1;
  }
  return 0;
}

static int write_from(const char *dir, const char *name, const float *src, size_t n) {
  char path[2048];
  FILE *f;
  size_t put;
  snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  f = fopen(path, "wb");
  if (!f) return -1;
  put = fwrite(src, sizeof(float), n, f);
  fclose(f);
  return put == n ? 0 : -1;
}

/* the reference's own initial grid, base state and initial state (FastEddy.c:223-238) */
static int dump_initial_state(const char *out) {
  size_t N = (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh) * (Nzp + 2 * Nh);
  size_t N2 = (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh);
  int rc = 0;
  fempi_AllocateBuffers(Nxp, Nyp, Nzp, Nh);
  if (gridSecondaryPreparations() != 0) return 7;
  if (hydro_coreSetBaseState() != 0) return 8;
  rc |= write_from(out, "xPos", xPos, N);
  rc |= write_from(out, "yPos", yPos, N);
  rc |= write_from(out, "zPos", zPos, N);
  rc |= write_from(out, "topoPos", topoPos, N2);
  rc |= write_from(out, "J31", J31, N);
  rc |= write_from(out, "J32", J32, N);
  rc |= write_from(out, "J33", J33, N);
  rc |= write_from(out, "D_Jac", D_Jac, N);
  rc |= write_from(out, "invD_Jac", invD_Jac, N);
  rc |= write_from(out, "baseState", hydroBaseStateFlds, 2 * N);
  rc |= write_from(out, "hydroFlds", hydroFlds, 5 * N);
  if (TKESelector > 0) rc |= write_from(out, "sgstke", sgstkeScalars, (size_t)TKESelector * N);
  if (surflayerSelector > 0) {
    rc |= write_from(out, "tskin", tskin, N2);
    rc |= write_from(out, "fricVel", fricVel, N2);
    rc |= write_from(out, "htFlux", htFlux, N2);
    rc |= write_from(out, "z0m", z0m, N2);
    rc |= write_from(out, "z0t", z0t, N2);
    if (moistureSelector > 0) {
      rc |= write_from(out, "qskin", qskin, N2);
      rc |= write_from(out, "qFlux", qFlux, N2);
    }
  }
  return rc ? 9 : 0;
}

int main(int argc, char **argv) {
  char *desc;
  int rc = 0;
  size_t N, N2;
  const char *in;
  if (argc != 4) {
    fprintf(stderr, "usage: %s PARAMFILE INDIR TSTEP\n", argv[0]);
    return 2;
  }
  in = argv[2];
  fempi_LaunchMPI(argc, argv);
  parameters_init();
  if (parameters_readFile(argv[1]) != 0) return 3;
  queryStringParameter("Description", &desc, PARAM_MANDATORY);
  fempi_GetParams();
  mem_utilsGetParams();
  ioGetParams();
  gridGetParams();
  hydro_coreGetParams();
  timeGetParams();
  srand(mpi_rank_world + 12345); /* FastEddy.c:109 */
  fempi_Init();
  mem_utilsInit();
  ioInit();
  gridInit();
  hydro_coreInit();
  timeInit();
  if (getParameterErrors() != 0) {
    fprintf(stderr, "ref_io: parameter errors\n");
    return 4;
  }
  if (strcmp(argv[3], "dump") == 0) return dump_initial_state(in);
  N = (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh) * (Nzp + 2 * Nh);
  N2 = (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh);
  rc |= read_into(in, "xPos", xPos, N);
  rc |= read_into(in, "yPos", yPos, N);
  rc |= read_into(in, "zPos", zPos, N);
  rc |= read_into(in, "topoPos", topoPos, N2);
  rc |= read_into(in, "hydroFlds", hydroFlds, 5 * N);
  rc |= read_into(in, "hydroPres", hydroPres, N);
  rc |= read_into(in, "hydroFldsFrhs", hydroFldsFrhs, 5 * N);
  if (TKESelector > 0) {
    rc |= read_into(in, "sgstke", sgstkeScalars, (size_t)TKESelector * N);
    rc |= read_into(in, "sgstkeFrhs", sgstkeScalarsFrhs, (size_t)TKESelector * N);
  }
  if (turbulenceSelector > 0) rc |= read_into(in, "taus", hydroTauFlds, 9 * N);
  if (surflayerSelector > 0) {
    rc |= read_into(in, "tskin", tskin, N2);
    rc |= read_into(in, "fricVel", fricVel, N2);
    rc |= read_into(in, "htFlux", htFlux, N2);
    rc |= read_into(in, "invOblen", invOblen, N2);
    rc |= read_into(in, "z0m", z0m, N2);
    rc |= read_into(in, "z0t", z0t, N2);
    if (moistureSelector > 0) {
      rc |= read_into(in, "qskin", qskin, N2);
      rc |= read_into(in, "qFlux", qFlux, N2);
    }
  }
  if (moistureSelector > 0) {
    rc |= read_into(in, "moist", moistScalars, (size_t)moistureNvars * N);
    rc |= read_into(in, "moistFrhs", moistScalarsFrhs, (size_t)moistureNvars * N);
    if (moistureSGSturb > 0) rc |= read_into(in, "moistTaus", moistTauFlds, (size_t)3 * moistureNvars * N);
  }
  if (rc) return 5;
  return ioWriteBinaryoutFileSingleTime(atoi(argv[3]), Nxp, Nyp, Nzp, Nh) == 0 ? 0 : 6;
}
