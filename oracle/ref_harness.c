/* ref_harness.c -- TEST INFRASTRUCTURE ONLY: driver that runs the reference's own CUDA
 * build (compiled from the reference sources into oracle/_ref by oracle/build_ref.py) on
 * inputs supplied as raw float32 files, so the B200 engine and the reference integrate
 * bit-identical initial states.
 *
 * Follows the reference's initialisation order (SRC/FEMAIN/FastEddy.c:72-280), then
 * overwrites every host input of the CUDA path (grid metrics, base state, prognostic
 * state, surface arrays) with the supplied files before the CUDA modules upload them.
 *
 * usage: fe_ref_harness PARAMFILE INDIR OUTDIR run NSTEPS
 *        fe_ref_harness PARAMFILE INDIR OUTDIR time K     (prints one JSON line)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <fempi.h>
#include <parameters.h>
#include <mem_utils.h>
#include <io.h>
#include <grid.h>
#include <hydro_core.h>
#include <time_integration.h>
#include <fecuda.h>
#include <cuda_grid.h>
#include <cuda_hydroCore.h>
#include <cuda_timeInt.h>

static size_t field_elems(void) { return (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh) * (Nzp + 2 * Nh); }
static size_t plane_elems(void) { return (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh); }

static int read_into(const char *dir, const char *name, float *dst, size_t n, int required) {
  char path[2048];
  FILE *f;
  size_t got;
  snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  f = fopen(path, "rb");
  if (!f) {
    if (required) fprintf(stderr, "harness: missing %s\n", path);
    return required ? -1 : 0;
  }
  got = fread(dst, sizeof(float), n, f);
  fclose(f);
  if (got != n) {
    fprintf(stderr, "harness: %s has %zu floats, expected %zu\n", path, got, n);
    return -1;
  }
  return 0;
}

static int write_from(const char *dir, const char *name, const float *src, size_t n) {
  char path[2048];
  FILE *f;
  snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  f = fopen(path, "wb");
  if (!f) return -1;
  fwrite(src, sizeof(float), n, f);
  fclose(f);
  return 0;
}

static double now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char **argv) {
  char *desc;
  int rc = 0, n, it;
  size_t N, N2;
  if (argc != 6) {
    fprintf(stderr, "usage: %s PARAMFILE INDIR OUTDIR run|time N\n", argv[0]);
    return 2;
  }
  n = atoi(argv[5]);
  fempi_LaunchMPI(argc, argv);
  parameters_init();
  if (parameters_readFile(argv[1]) != 0) return 3;
  queryStringParameter("Description", &desc, PARAM_MANDATORY);
  fempi_GetParams();
  mem_utilsGetParams();
  ioGetParams();
  fecuda_GetParams();
  gridGetParams();
  hydro_coreGetParams();
  timeGetParams();
  fempi_Init();
  mem_utilsInit();
  ioInit();
  fecuda_Init();
  gridInit();
  hydro_coreInit();
  timeInit();
  if (getParameterErrors() != 0) {
    fprintf(stderr, "harness: parameter errors\n");
    return 4;
  }
  fempi_AllocateBuffers(Nxp, Nyp, Nzp, Nh);
  gridSecondaryPreparations();
  hydro_coreSetBaseState();

  N = field_elems();
  N2 = plane_elems();
  rc |= read_into(argv[2], "zPos", zPos, N, 1);
  rc |= read_into(argv[2], "J31", J31, N, 1);
  rc |= read_into(argv[2], "J32", J32, N, 1);
  rc |= read_into(argv[2], "J33", J33, N, 1);
  rc |= read_into(argv[2], "D_Jac", D_Jac, N, 1);
  rc |= read_into(argv[2], "invD_Jac", invD_Jac, N, 1);
  rc |= read_into(argv[2], "baseState", hydroBaseStateFlds, 2 * N, 1);
  rc |= read_into(argv[2], "hydroFlds", hydroFlds, 5 * N, 1);
  if (TKESelector > 0) rc |= read_into(argv[2], "sgstke", sgstkeScalars, N, 1);
  if (moistureSelector > 0) rc |= read_into(argv[2], "moist", moistScalars, (size_t)moistureNvars * N, 1);
  if (surflayerSelector > 0) {
    rc |= read_into(argv[2], "z0m", z0m, N2, 1);
    rc |= read_into(argv[2], "z0t", z0t, N2, 1);
    rc |= read_into(argv[2], "htFlux", htFlux, N2, 1);
    rc |= read_into(argv[2], "tskin", tskin, N2, 1);
    rc |= read_into(argv[2], "fricVel", fricVel, N2, 1);
    if (moistureSelector > 0) {
      rc |= read_into(argv[2], "qFlux", qFlux, N2, 1);
      rc |= read_into(argv[2], "qskin", qskin, N2, 1);
    }
  }
  if (rc) return 5;

  cuda_gridInit();
  fecuda_SetBlocksPerGrid((Nxp + 2 * Nh), (Nyp + 2 * Nh), (Nzp + 2 * Nh));
  cuda_hydroCoreInit();
  cuda_timeIntInit();

  it = simTime_itRestart;
  if (strcmp(argv[4], "run") == 0) {
    NtBatch = n;
    cuda_timeIntCommence(it);
    write_from(argv[3], "hydroFlds", hydroFlds, 5 * N);
    write_from(argv[3], "pres", hydroPres, N);
    if (TKESelector > 0) write_from(argv[3], "sgstke", sgstkeScalars, N);
    if (moistureSelector > 0) write_from(argv[3], "moist", moistScalars, (size_t)moistureNvars * N);
    if (surflayerSelector > 0) {
      write_from(argv[3], "fricVel", fricVel, N2);
      write_from(argv[3], "htFlux", htFlux, N2);
      write_from(argv[3], "invOblen", invOblen, N2);
      write_from(argv[3], "tskin", tskin, N2);
    }
  } else {
    /* warm-up batch (also the first-batch host-to-device upload), then batches of K and
     * 2K steps; their difference times K steps without the per-batch copy back */
    double t0, t1, t2, t3;
    NtBatch = 1;
    cuda_timeIntCommence(it);
    it += NtBatch;
    NtBatch = n;
    t0 = now();
    cuda_timeIntCommence(it);
    t1 = now();
    it += NtBatch;
    NtBatch = 2 * n;
    t2 = now();
    cuda_timeIntCommence(it);
    t3 = now();
    printf("{\"ref_batch_K_s\": %.6f, \"ref_batch_2K_s\": %.6f, \"K\": %d, \"ms_per_step\": %.6f, \"cells\": %lld}\n",
           t1 - t0, t3 - t2, n, 1e3 * ((t3 - t2) - (t1 - t0)) / n, (long long)Nxp * Nyp * Nzp);
  }
  cuda_timeIntCleanup();
  cuda_hydroCoreCleanup();
  cuda_gridCleanup();
  fflush(stdout);
  return 0;
}
