/* fasteddy_b200.h -- C ABI of the B200-native FastEddy hot path.
 *
 * Two layers, both plain C (no C++ or torch types, plain pointers and sizes):
 *
 * 1. The reference-named drop-in entry points (section A). They have exactly the
 *    signatures the FastEddy driver binds (reference SRC/FEMAIN/FastEddy.c:123,256,
 *    263-280,379,451-461) and read their inputs from the same global host symbols the
 *    reference CUDA layer reads (grid extents, metric arrays, prognostic arrays,
 *    physics selectors; see fe_refglobals.h). They return 0 on success and a nonzero
 *    FE_ERR_* code on failure; unlike the reference (fecuda_Device_cu.h:26-35) they
 *    never call exit().
 *
 * 2. The engine API (section B): an explicit domain handle, used by the entry points
 *    above, by the ensemble launcher and directly by tests and benchmarks.
 *
 * Field layout everywhere at this boundary is the reference's: a field of a domain
 * with interior extents Nx,Ny,Nz and halo width Nh=3 is a float array of
 * (Nx+6)*(Ny+6)*(Nz+6) values indexed ijk = i*(Ny+6)*(Nz+6) + j*(Nz+6) + k
 * (k fastest, the iStride/jStride of every reference device routine), multi-field blocks
 * concatenate fields with that stride, momentum/scalars in flux form (rho*phi).
 */
#ifndef FASTEDDY_B200_H
#define FASTEDDY_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- error codes */
#define FE_OK               0
#define FE_ERR_CUDA         1   /* a CUDA runtime call failed (message via fe_last_error) */
#define FE_ERR_CONFIG       2   /* unsupported or inconsistent configuration */
#define FE_ERR_ARG          3   /* NULL handle/pointer or bad size */
#define FE_ERR_STATE        4   /* call out of order (e.g. advance before set_state) */
#define FE_ERR_NOMEM        5   /* device allocation failed */
#define FE_ERR_NONFINITE    6   /* the state contains NaN/Inf after a batch */
#define FE_ERR_NO_DEVICE    7   /* no CUDA device visible */

/* ======================================================= A. reference-named ABI */
/* Each entry replaces the same-named function of the reference CUDA layer. */

/* replaces SRC/FECUDA/fecuda.c:38 fecuda_GetParams(): reads the tBx/tBy/tBz keys through the
 * reference's parameter reader when the program links it (they stay mandatory keys); the
 * engine chooses its own launch shapes. */
int fecuda_GetParams(void);
/* replaces SRC/FECUDA/fecuda.h:35 fecuda_Init(): selects device (rank % numDevices). */
int fecuda_Init(void);
/* replaces SRC/FECUDA/fecuda.h:45 fecuda_SetBlocksPerGrid(): halo-inclusive extents;
 * accepted for interface compatibility (launch geometry is chosen by the engine). */
int fecuda_SetBlocksPerGrid(int Nx, int Ny, int Nz);
/* replaces SRC/FECUDA/fecuda.h:55 / :60: single-GPU domains need no halo buffers. */
int fecuda_AllocateHaloBuffers(int Nxp, int Nyp, int Nzp, int Nh);
int fecuda_DeallocateHaloBuffers(void);
/* replaces SRC/FECUDA/fecuda.h:40 fecuda_Cleanup(). */
int fecuda_Cleanup(void);
/* replaces SRC/GRID/CUDA/cuda_grid.h:30 cuda_gridInit(): uploads zPos and metrics. */
int cuda_gridInit(void);
/* replaces SRC/GRID/CUDA/cuda_grid.h:35 cuda_gridCleanup(). */
int cuda_gridCleanup(void);
/* replaces SRC/HYDRO_CORE/CUDA/cuda_hydroCore.h:30 cuda_hydroCoreInit(): creates the
 * device domain from the physics globals and uploads the base state. */
int cuda_hydroCoreInit(void);
/* replaces SRC/HYDRO_CORE/CUDA/cuda_hydroCore.h:35 cuda_hydroCoreCleanup(). */
int cuda_hydroCoreCleanup(void);
/* replaces SRC/TIME_INTEGRATION/CUDA/cuda_timeInt.h:30 cuda_timeIntInit(): uploads the
 * prognostic state and surface arrays. */
int cuda_timeIntInit(void);
/* replaces SRC/TIME_INTEGRATION/CUDA/cuda_timeInt.h:35 cuda_timeIntCleanup(). */
int cuda_timeIntCleanup(void);
/* replaces SRC/TIME_INTEGRATION/CUDA/cuda_timeInt.h:40 cuda_timeIntCommence(it):
 * advances NtBatch RK3 steps (re-uploading the host state when it==simTime_itRestart),
 * then copies state, perturbation pressure and surface arrays back to the host
 * globals and advances simTime / simTime_it, as cuda_timeIntDevice.cu:105-157. */
int cuda_timeIntCommence(int it);
/* replaces SRC/HYDRO_CORE/CUDA/cuda_hydroCoreDevice_cu.h:97 (device-level twin):
 * evaluates the tendency of RK stage `timeStage` (0..2) from the device state into
 * the device Frhs buffers without committing; read it back with fe_get_frhs(). */
int cuda_hydroCoreDeviceBuildFrhs(float simTime, int simTime_it, int simTime_itRestart,
                                  float dt, int timeStage, int numRKstages);
/* replaces SRC/TIME_INTEGRATION/CUDA/cuda_timeIntDevice_cu.h:57/:62 twins. */
int cuda_timeIntHydroInitDevice(void);
int cuda_timeIntHydroSynchFromDevice(void);

/* ===================================================================== B. engine */
typedef struct fe_domain fe_domain;
typedef struct fe_ensemble fe_ensemble;
typedef struct fe_comm fe_comm;

/* Physics configuration of one domain. Names and meanings follow the reference's
 * parameter keys (SRC/HYDRO_CORE/hydro_core.c:197-395, SRC/GRID/grid.c:68-88,
 * SRC/TIME_INTEGRATION/time_integration.c:51-64); derived constants follow
 * hydro_core.c:941-967. Fill with fe_config_defaults() then override. */
typedef struct fe_config {
  int Nx, Ny, Nz, Nh;                 /* interior extents per rank, halo width (3) */
  float dX, dY, dZ;                   /* d_xi, d_eta, d_zeta */
  float dt;
  int simTime_itRestart;
  int hydroBCs;                       /* only 2 (periodic horizontal, ABL vertical) */
  int pgfSelector, buoyancySelector, coriolisSelector;
  int turbulenceSelector, TKESelector, TKEAdvSelector;
  float TKEAdvSelector_b_hyb, c_s, c_k;
  int advectionSelector;              /* 0 upwind, 1 QUICK, 2 HYB34, 3 HYB56, 4 WENO3, 5 WENO5, 6 centred 2nd */
  float b_hyb;
  int diffusionSelector, filterSelector, lsfSelector;   /* diffusion must be 0; filter and lsf 0 or 1 */
  int surflayerSelector;              /* 0, 1 (heat flux) or 2 (skin temperature) */
  float surflayer_z0, surflayer_z0t, surflayer_wth, surflayer_tr, surflayer_wq, surflayer_qr;
  int surflayer_qskin_input, surflayer_stab, surflayer_idealsine;
  float surflayer_ideal_ts, surflayer_ideal_te, surflayer_ideal_amp;
  float surflayer_ideal_qts, surflayer_ideal_qte, surflayer_ideal_qamp;
  int moistureSelector, moistureNvars, moistureAdvSelectorQv;
  float moistureAdvSelectorQv_b;
  int moistureAdvSelectorQi, moistureSGSturb, moistureCond;
  float moistureCondTscale;
  int moistureCondBasePres;
  float moistureMPcallTscale;
  int dampingLayerSelector;
  float dampingLayerDepth;
  float U_g, V_g, z_Ug, z_Vg, Ug_grad, Vg_grad;
  float corioConstHorz, corioConstVert, corioLS_fact;
  int physics_oneRKonly;
  float temp_grnd, pres_grnd;
  float R_gas, R_vapor, Rv_Rg, cp_gas, cv_gas, accel_g, R_cp, cp_R, cp_cv, refPressure, kappa, L_v;
  float filter_6th_coeff;             /* 6th-order vertical filter factor on rho w (filterSelector = 1) */
  /* large-scale forcing (lsfSelector = 1): piecewise-linear profiles in z (surface value, values
   * at zlev1 and zlev2, constant above), per hour; w drives the subsidence terms */
  int lsf_horMnSubTerms;              /* 1: subsidence of the slab-mean u, v, theta, q_v */
  float lsf_freq;                     /* seconds between applications */
  float lsf_w_surf, lsf_w_lev1, lsf_w_lev2, lsf_w_zlev1, lsf_w_zlev2;
  float lsf_th_surf, lsf_th_lev1, lsf_th_lev2, lsf_th_zlev1, lsf_th_zlev2;
  float lsf_qv_surf, lsf_qv_lev1, lsf_qv_lev2, lsf_qv_zlev1, lsf_qv_zlev2;
} fe_config;

/* Reference defaults (hydro_core.c:197-395 defaults, hydro_core.c:941-952 constants). */
void fe_config_defaults(fe_config *cfg);
/* Recompute the derived constants (cp, ratios, Coriolis factors from latitude). */
void fe_config_derive(fe_config *cfg, float coriolisLatitude);

int fe_device_count(void);
/* Check a configuration as fe_create does (selector ranges as hydro_core.c:221-349 checks
 * them, and what this path supports); FE_OK or FE_ERR_CONFIG/FE_ERR_ARG with fe_last_error(). */
int fe_check_config(const fe_config *cfg);
/* Create a domain on `device`; checks the configuration and allocates device memory. */
int fe_create(const fe_config *cfg, int device, fe_domain **out);
int fe_destroy(fe_domain *d);
/* Bytes of device memory held by the domain. */
size_t fe_device_bytes(const fe_domain *d);

/* Grid inputs, reference layout, halo-inclusive, one field each. */
int fe_set_grid(fe_domain *d, const float *zPos, const float *J31, const float *J32,
                const float *J33, const float *D_Jac, const float *invD_Jac);
/* Base state: rho_BS and (rho*theta)_BS, two concatenated fields (hydroBaseStateFlds). */
int fe_set_base_state(fe_domain *d, const float *baseStateFlds);
/* Prognostic state: hydroFlds (5 fields), sgstke (TKESelector fields or NULL),
 * moist (moistureNvars fields or NULL). Halos are filled on the device. */
int fe_set_state(fe_domain *d, const float *hydroFlds, const float *sgstke, const float *moist);
/* Surface 2-D arrays ((Nx+6)*(Ny+6) each, any may be NULL when unused). */
int fe_set_surface(fe_domain *d, const float *z0m, const float *z0t, const float *htFlux,
                   const float *tskin, const float *fricVel, const float *qFlux, const float *qskin);
/* Simulation clock (simTime, simTime_it) the next step starts from. */
int fe_set_clock(fe_domain *d, float simTime, int simTime_it);
int fe_get_clock(const fe_domain *d, float *simTime, int *simTime_it);

/* Advance `nsteps` RK3 steps on the domain's stream (asynchronous; see fe_sync). */
int fe_advance(fe_domain *d, int nsteps);
/* Block until queued work of the domain finished; reports device errors. */
int fe_sync(fe_domain *d);
/* CUDA stream (cudaStream_t) the domain launches on, for event timing. */
void *fe_stream(fe_domain *d);

int fe_get_state(fe_domain *d, float *hydroFlds, float *sgstke, float *moist, float *pres);
int fe_get_surface(fe_domain *d, float *cd, float *ch, float *fricVel, float *htFlux,
                   float *invOblen, float *tskin, float *qFlux, float *qskin);

/* Tendency of RK stage `stage` (0..2) from the current state, no commit. */
int fe_build_frhs(fe_domain *d, int stage);
/* Copy the tendencies of the last fe_build_frhs (same field blocks as fe_get_state)
 * and, if taus != NULL, the 9 SGS stress/flux fields (order of hydroTauFlds). */
int fe_get_frhs(fe_domain *d, float *hydroFrhs, float *sgstkeFrhs, float *moistFrhs, float *taus);
/* With on != 0, every later fe_advance keeps the tendencies of the last RK stage of its last
 * step in the buffer fe_get_frhs reads: what the reference holds in its Frhs arrays after a
 * batch and copies back when hydroForcingWrite or hydroForcingLog is set
 * (cuda_timeIntDevice.cu:210-224). That step then runs outside the step graph. */
int fe_set_forcing_capture(fe_domain *d, int on);
/* The SGS stresses and heat fluxes (9 fields, order of hydroTauFlds) and the moisture SGS
 * fluxes (3 per moisture species, order of moistTauFlds: species-major, x, y, z) of the last
 * physics stage evaluated, the arrays cuda_timeIntDevice.cu:238-251 copies back. Either
 * pointer may be NULL. */
int fe_get_sgs_fluxes(fe_domain *d, float *taus, float *moistTaus);

/* Count NaN/Inf values in the interior prognostic state (device reduction). */
int fe_count_nonfinite(fe_domain *d, long long *count);
/* FP64 domain means of the interior prognostic fields (device reduction with FP64
 * accumulation); means has room for 5 + TKESelector + moistureNvars values. */
int fe_domain_means(fe_domain *d, double *means);

/* Launch-shape control: threads per block along k and j of the stencil kernels and
 * the number of i-planes each thread block marches (0 = engine default). */
int fe_set_tiling(fe_domain *d, int tk, int tj, int ti);
/* Form of the fused stage kernel. FE_KERNEL_MARCH (the default): thread blocks of 32 levels
 * by tj rows (4 or 8) march ni planes along i with the x stencil in registers and the y/z
 * stencils in shared memory. FE_KERNEL_CELL: one thread per cell, tiled by fe_set_tiling.
 * tj/ni <= 0 select the defaults: tj = 8 and the ni chosen at creation (the most of 64, 32, 16, 8
 * planes per block that leaves 20 waves of two thread blocks per SM, else 8). */
#define FE_KERNEL_CELL 0
#define FE_KERNEL_MARCH 1
int fe_set_stage_kernel(fe_domain *d, int kind, int tj, int ni);
int fe_get_stage_kernel(const fe_domain *d, int *kind, int *tj, int *ni);
/* Form of the last RK stage's SGS physics with the march stage kernel: rows = 8 or 16 evaluates
 * the closure's stresses and fluxes and the tendencies they give in one i-marching kernel with
 * tiles of 32 levels x rows that keeps them on chip; 0 runs them as separate kernels through the
 * scratch fields (the form the learned closure and the per-cell stage kernel always use). Results
 * are equal bit for bit. */
int fe_set_sgs_kernel(fe_domain *d, int rows);
/* The fused SGS kernel's tile rows (0, 8 or 16) and planes per thread block; and both read back.
 * fe_autotune times the fused SGS kernel's shapes too and keeps the fastest. */
int fe_set_sgs_shape(fe_domain *d, int rows, int ni);
int fe_get_sgs_shape(const fe_domain *d, int *rows, int *ni);
/* Pick the stage-kernel form and launch shape by timing the candidates (the autotuner);
 * tk/tj/ti receive the cell-kernel tiling, fe_get_stage_kernel the chosen form. */
int fe_autotune(fe_domain *d, int *tk, int *tj, int *ti);
/* Page-lock an existing host buffer for faster copies (cudaHostRegister) and undo it. */
int fe_host_register(void *ptr, size_t bytes);
int fe_host_unregister(void *ptr);
/* Time `reps` back-to-back launches of the fused dynamics stage kernel (the RK3 second
 * stage, whose output buffer every step rewrites, so the model state is unchanged) with
 * CUDA events on the domain's stream; *ms receives the mean time per launch. */
int fe_time_stage_kernel(fe_domain *d, int reps, float *ms);
/* Number of engine kernel launches enqueued since creation (for bookkeeping). */
long long fe_launch_count(const fe_domain *d);

/* Ensembles: advance several domains (different sizes allowed, same device) with one
 * captured CUDA graph per step batch. When every member runs the dry flavour with the fused
 * SGS kernel (prognostic TKE, HYB56, no moisture, no subsidence means, no network, not
 * decomposed), a step is one launch per kernel over the tiles of all members (a work list of
 * (member, tile) items with the members' parameters in device tables), else one graph branch per
 * member; both give the members' own results bit for bit. The members' settings and tile shapes
 * are read when the ensemble first advances. fe_ensemble_set_batched(e, 0) keeps the branches. */
int fe_ensemble_create(fe_domain **members, int n, fe_ensemble **out);
int fe_ensemble_advance(fe_ensemble *e, int nsteps);
int fe_ensemble_sync(fe_ensemble *e);
void *fe_ensemble_stream(fe_ensemble *e);
int fe_ensemble_destroy(fe_ensemble *e);
int fe_ensemble_set_batched(fe_ensemble *e, int on);
int fe_ensemble_is_batched(const fe_ensemble *e);
/* Kernel launches enqueued for the ensemble and its members since creation. */
long long fe_ensemble_launch_count(const fe_ensemble *e);

/* Domain decomposition over px x py slabs, FastEddy's numProcsX x numProcsY ranks
 * (fempi.c:98-160 rank grid: rx = r % px, ry = r / px; periodic neighbours fempi.c:226-245).
 * Each slab is a domain created with Nx = Nx_global/px, Ny = Ny_global/py and given the
 * halo-inclusive slab of the global inputs. Every RK stage's commit writes the slab's cells
 * and, for cells within 3 of a slab edge, their images in the neighbouring slabs' halos: the
 * per-stage exchange of cuda_hydroCoreDevice.cu:276-314 (fecuda_SendRecvWestEast/EastWest/
 * SouthNorth/NorthSouth, fecuda_Utils.cu:205-418) fused into the commit as peer stores.
 * Set the decomposition before the inputs (the initial boundary fill then keeps the given
 * slab halos). Not with lsf_horMnSubTerms = 1 (its slab means span the domain).
 *
 * All slabs on one device, in this process: slabs[r] for rank r; the group advances with
 * fe_ensemble_advance (stages of all slabs in lock step) and is released by
 * fe_ensemble_destroy. */
int fe_slab_group_create(fe_domain **slabs, int px, int py, fe_ensemble **out);
/* One slab per process (one GPU each): exchange the slabs' state-arena handles
 * (fe_arena_ipc_handle, fe_ipc_handle_bytes() bytes) among the ranks, then give each slab
 * the handles of its 8 neighbours, handles[(dx+1)*3 + (dy+1)] for dx, dy in {-1,0,1}
 * (NULL where the neighbour is the slab itself), and a stage barrier: a communicator of all
 * ranks (fe_comm_create from the unique id rank 0 made with fe_comm_unique_id, of
 * fe_comm_unique_id_bytes() bytes, passed to every rank). All ranks advance the same steps. */
size_t fe_ipc_handle_bytes(void);
int fe_arena_ipc_handle(fe_domain *d, void *out, size_t bytes);
int fe_set_halo_peers(fe_domain *d, int px, int py, const void *const *handles);
/* Unmap the neighbours' arenas (after every rank's last step); the slab is undecomposed again. */
int fe_clear_halo_peers(fe_domain *d);
size_t fe_comm_unique_id_bytes(void);
int fe_comm_unique_id(void *out, size_t bytes);
int fe_comm_create(const void *uid, int nranks, int rank, int device, fe_comm **out);
int fe_comm_destroy(fe_comm *c);
int fe_set_halo_comm(fe_domain *d, fe_comm *c);

/* Checkpoint / resume: the prognostic state, the 11 surface planes and the clock in one host
 * buffer of fe_checkpoint_bytes() bytes (a header checks the domain shape on load); with
 * large-scale subsidence (lsf_horMnSubTerms = 1) also the previous step's last-stage input,
 * whose halo values the next slab means read. Loading
 * into a domain with the same grid and base state and advancing repeats the run that wrote it
 * bit for bit (the reference restarts through its netCDF inFile, io_netcdf.c:106-300). */
size_t fe_checkpoint_bytes(const fe_domain *d);
int fe_checkpoint_save(fe_domain *d, void *buf, size_t bytes);
int fe_checkpoint_load(fe_domain *d, const void *buf, size_t bytes);

/* ======================================================= C. learned SGS closure */
/* No counterpart in the reference: a small network that replaces the 9 stresses and heat
 * fluxes of the TKE closure (cudaDevice_hydroCoreCalcTaus_PrognosticTKE_DeviatoricTerm,
 * SRC/HYDRO_CORE/CUDA/cuda_sgsTurbDevice.cu:308-367) where the SGS divergence consumes them
 * (cuda_hydroCoreDevice.cu:759-768); the TKE closure stays the fallback (no network set).
 *
 * Inputs per stress point (FE_SGS_NIN): the 9 velocity-gradient halves of the closure's
 * staggered strain rates g11 g12 g13 g21 g22 g23 g31 g32 g33, the buoyancy frequency N^2 and
 * the grid scale (dx dy dz D)^(1/3). Outputs (FE_SGS_NOUT): tau/rho in the closure's field
 * order tau11 tau21 tau31 tau32 tau22 tau33 tauTH1 tauTH2 tauTH3. Network 11 -> 64 -> 64 ->
 * 64 -> 9 with tanh, BF16 weights/activations on the tensor cores, FP32 accumulation;
 * inputs standardised with (in_mu, in_sig), outputs tau/rho = out_mu + out_sig * y.
 * Parameters (fe_mlp_param_count() FP32 values): W1[64][16] (columns 11..15 unused), b1[64],
 * W2[64][64], b2[64], W3[64][64], b3[64], W4[16][64] (rows 9..15 unused), b4[16]. */
#define FE_SGS_NIN 11
#define FE_SGS_NOUT 9
typedef struct fe_mlp fe_mlp;
long long fe_mlp_param_count(void);
int fe_mlp_create(int device, unsigned long long seed, fe_mlp **out); /* Glorot-uniform weights */
int fe_mlp_destroy(fe_mlp *m);
int fe_mlp_set_params(fe_mlp *m, const float *params); /* also resets the optimiser */
int fe_mlp_get_params(fe_mlp *m, float *params);
int fe_mlp_set_norm(fe_mlp *m, const float *in_mu, const float *in_sig, const float *out_mu, const float *out_sig);
int fe_mlp_get_norm(fe_mlp *m, float *in_mu, float *in_sig, float *out_mu, float *out_sig);
/* Training set: host arrays X[n][11] (inputs), T[n][9] (targets tau/rho); shuffled once with
 * `seed`; fit_norm != 0 sets the standardisation to the set's means and deviations. */
int fe_mlp_set_data(fe_mlp *m, const float *X, const float *T, long long n, unsigned long long seed, int fit_norm);
/* Loss (mean over samples and outputs of the squared standardised error) and its gradient
 * (fe_mlp_param_count() values) over samples [first, first+count) of the set, in set order. */
int fe_mlp_gradient(fe_mlp *m, long long first, long long count, float *grad, double *loss);
/* `steps` Adam steps (beta 0.9/0.999) on consecutive shuffled batches; loss_hist (may be NULL)
 * receives the loss of every step. */
int fe_mlp_train(fe_mlp *m, int steps, long long batch, float lr, double *loss_hist);
/* Network outputs tau/rho for host inputs X[n][11] into Y[n][9]. */
int fe_mlp_predict(fe_mlp *m, const float *X, long long n, float *Y);
/* Mean device time (CUDA events) of a gradient evaluation (train != 0) or an inference over
 * the first `batch` samples of the set. */
int fe_mlp_time(fe_mlp *m, int train, long long batch, int reps, float *ms);
/* Report (and clear) an expired tensor-core wait of the network's kernels. */
int fe_mlp_check(fe_mlp *m);
/* Use the network for the domain's SGS stresses (NULL: the TKE closure). */
int fe_set_sgs_mlp(fe_domain *d, fe_mlp *m);
/* Evaluate the domain's closure on its current state and sample every `every`-th interior cell
 * (row-major i, j, k; every >= 1): inputs X[n][11], stresses tau[n][9], density rho[n] with
 * n = ceil(cells/every) (any NULL is skipped). */
int fe_sgs_sample(fe_domain *d, long long every, float *X, float *tau, float *rho);
/* Coarse-grain the state of `fine` (2Nx x 2Ny x 2Nz over the same physical domain) by a
 * 2x2x2 box filter into the state of `coarse`, and write the subfilter stresses and heat
 * fluxes of every coarse interior cell divided by the filtered density (plus the fine
 * model's own closure stresses) to tau_target[cells][9] (may be NULL). */
int fe_coarsen(fe_domain *fine, fe_domain *coarse, float *tau_target);

/* ---------------------------------------------- allocation-free tendency evaluation */
/* No counterpart in the reference. For callers that cannot allocate device memory (pool
 * allocators that own all device memory, embedders whose memory footprint is fixed after
 * start-up): evaluates the tendency of
 * RK stage `stage` like fe_build_frhs, but all scratch lives in one static device array of
 * FE_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds until exit. Limit:
 * (Nx+6)(Ny+6)(Nz+6) <= fe_noalloc_max_cells() (about 799k cells). All pointers are device
 * pointers in the reference layout; `state` (5 + TKE + moisture fields) must have its halo
 * cells filled (as fe_get_state returns them); `surface` holds the 11 planes cd, ch, cq,
 * fricVel, htFlux, tskin, invOblen, z0m, z0t, qFlux, qskin and is updated in place on a
 * physics stage; `frhs` receives the interior tendencies. Every call looks up the array's
 * device address on the caller's current device (so a reset device or a re-created context is
 * followed). Calls share the array, so calls that overlap on the GPU (other streams, other
 * threads) race. The configuration is checked as fe_check_config does, and further limited to
 * HYB56/WENO5 advection without the explicit filter or large-scale forcing.
 * Runs on `stream` (a cudaStream_t, NULL = legacy default stream) and synchronises it. */
#define FE_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
typedef struct fe_noalloc_args {
  const float *zPos, *J31, *J32, *J33, *D_Jac, *invD_Jac;
  const float *baseState;
  const float *state;
  float *surface;
  float *frhs;
} fe_noalloc_args;
long long fe_noalloc_max_cells(void);
int fe_frhs_noalloc(const fe_config *cfg, int stage, float simTime, int simTime_it, const fe_noalloc_args *args,
                    void *stream);
const char *fe_noalloc_last_error(void);

/* Text of the last error of the calling thread. */
const char *fe_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
