/* ref_harness.c -- TEST INFRASTRUCTURE ONLY: driver that runs the reference's own CUDA
 * build (compiled from the reference sources into oracle/_ref by oracle/build_ref.py) on
 * inputs supplied as raw float32 files, so the B200 engine and the reference integrate
 * bit-identical initial states.
 *
 * Follows the reference's initialisation order (SRC/FEMAIN/FastEddy.c:72-280), then
 * overwrites every host input of the CUDA path (grid metrics, base state, prognostic
 * state, surface arrays) with the supplied files before the CUDA modules upload them
 * (unless INDIR is "-", below).
 *
 * usage: fe_ref_harness PARAMFILE INDIR OUTDIR run NSTEPS [qv:SFC,TOP,ZTOP]
 *        fe_ref_harness PARAMFILE INDIR OUTDIR time K [qv:SFC,TOP,ZTOP]   (prints one JSON line)
 *        fe_ref_harness PARAMFILE INDIR OUTDIR frhs STAGE
 *
 * INDIR "-" keeps the reference's own initial state: its grid (from the parameter file's
 * topoFile), its base state and its seeded theta perturbations (FastEddy.c:109,232-238). The
 * reference can only start moisture from a netCDF inFile, so "qv:SFC,TOP,ZTOP" sets
 * rho*q_v [g/kg] on its own grid: SFC at z <= 0, linear to TOP at z = ZTOP, TOP above; q_l = 0.
 *
 * run writes the state after NSTEPS steps, and, when the parameter file sets hydroForcingWrite
 * or hydroSubGridWrite, the tendencies and SGS fluxes the reference copies back with it
 * (cuda_timeIntDevice.cu:198-251: those of the last stage of the last step). frhs evaluates one
 * tendency of RK stage STAGE (0..2) on the supplied state through the reference's own
 * cuda_hydroCoreDeviceBuildFrhs and writes the tendencies and SGS fluxes (the parameter file
 * must set hydroForcingWrite = 1 and hydroSubGridWrite = 1, so the reference allocates them).
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

/* device-level entry points of the reference (extern "C" in its .cu files) */
int cuda_timeIntHydroInitDevice(void);
int cuda_timeIntHydroSynchFromDevice(void);
int cuda_hydroCoreDeviceBuildFrhs(float simTime, int simTime_it, int simTime_itRestart, float dt, int timeStage,
                                  int numRKstages);

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

/* rho q_v from a linear q_v(z) profile on the reference's own grid and density. */
static int set_qv_profile(const char *spec) {
  double qs, qt, zt;
  size_t n = field_elems(), ijk;
  if (sscanf(spec, "qv:%lf,%lf,%lf", &qs, &qt, &zt) != 3 || !(zt > 0.0)) {
    fprintf(stderr, "harness: bad q_v profile '%s'\n", spec);
    return -1;
  }
  if (moistureSelector <= 0 || moistureNvars <= 0) {
    fprintf(stderr, "harness: q_v profile given for a dry case\n");
    return -1;
  }
  for (ijk = 0; ijk < n; ijk++) {
    double z = zPos[ijk], q;
    if (z <= 0.0) q = qs;
    else if (z >= zt) q = qt;
    else q = qs + (qt - qs) * z / zt;
    moistScalars[ijk] = (float)(q * hydroFlds[ijk]);
    if (moistureNvars > 1) moistScalars[n + ijk] = 0.0f;
  }
  return 0;
}

/* The tendencies and SGS fluxes the batch copy-back brought to the host. */
static void write_forcing(const char *dir) {
  size_t N = field_elems();
  if (hydroForcingWrite == 1 || hydroForcingLog == 1) {
    write_from(dir, "hydroFrhs", hydroFldsFrhs, 5 * N);
    if (TKESelector > 0) write_from(dir, "sgstkeFrhs", sgstkeScalarsFrhs, N);
    if (moistureSelector > 0) write_from(dir, "moistFrhs", moistScalarsFrhs, (size_t)moistureNvars * N);
  }
  if (hydroSubGridWrite == 1) {
    if (turbulenceSelector > 0) write_from(dir, "taus", hydroTauFlds, 9 * N);
    if (moistureSGSturb == 1 && moistureSelector > 0) write_from(dir, "moistTaus", moistTauFlds, (size_t)moistureNvars * 3 * N);
  }
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
  if (argc != 6 && argc != 7) {
    fprintf(stderr, "usage: %s PARAMFILE INDIR|- OUTDIR run|time|frhs N [qv:SFC,TOP,ZTOP]\n", argv[0]);
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
  srand(mpi_rank_world + 12345); /* FastEddy.c:109 */
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
  if (strcmp(argv[2], "-") != 0) {
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
  }
  if (argc == 7 && set_qv_profile(argv[6]) != 0) return 5;
  if (rc) return 5;

  cuda_gridInit();
  fecuda_SetBlocksPerGrid((Nxp + 2 * Nh), (Nyp + 2 * Nh), (Nzp + 2 * Nh));
  cuda_hydroCoreInit();
  cuda_timeIntInit();

  it = simTime_itRestart;
  if (strcmp(argv[4], "frhs") == 0) {
    /* one tendency evaluation of stage n on the uploaded state; the parameter file sets
     * hydroForcingWrite and hydroSubGridWrite so the host arrays exist and are copied back */
    if (n < 0 || n > 2) return 2;
    cuda_timeIntHydroInitDevice();
    cuda_hydroCoreDeviceBuildFrhs(simTime, simTime_it, simTime_itRestart, dt, n, numRKstages);
    cuda_timeIntHydroSynchFromDevice();
    write_from(argv[3], "pres", hydroPres, N);
    write_forcing(argv[3]);
  } else if (strcmp(argv[4], "run") == 0) {
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
    write_forcing(argv[3]);
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
