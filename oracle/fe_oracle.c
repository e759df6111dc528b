/* fe_oracle.c -- TEST INFRASTRUCTURE ONLY (see fe_oracle.h): serial FP64 restatement of
 * the reference hot path, used by tests as the checker of the CUDA path.
 *
 * Every array is double precision in the reference's halo-inclusive layout
 * ijk = (i*(Ny+2Nh) + j)*(Nz+2Nh) + k. The stage follows the reference's kernel order
 * (SRC/HYDRO_CORE/CUDA/cuda_hydroCoreDevice.cu:246-426 then
 * SRC/TIME_INTEGRATION/CUDA/cuda_timeIntDevice.cu:131-146), one operator at a time over
 * all its cells, so values the reference reads from other threads are always the ones
 * of the current stage (its Commence corner halos and the sgstke_ls[k-1] read in
 * CalcEddyDiff are races on the GPU; here they are resolved in program order).
 * Transcendentals are libm double; no CUDA math is reproduced.
 */
#include "fe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct ora_domain {
  fe_config c;
  int nxh, nyh, nzh;              /* halo-inclusive extents */
  size_t n, n2;                   /* elements per 3-D / 2-D field */
  int iMin, iMax, jMin, jMax, kMin, kMax;
  double dX, dY, dZ, dXi, dYi, dZi;
  int nmoist, ntke;
  double simTime;
  int simTime_it;
  /* grid and base state */
  double *zPos, *J31, *J32, *J33, *D, *invD, *rhoBS, *thBS;
  /* state */
  double *fld[5], *tke, *moist[2];
  double *fld0[5], *tke0, *moist0[2];
  double *F[5], *Ftke, *Fmoist[3];
  double *rhoInv, *pres, *ucf, *vcf, *wcf;
  double *tau[9], *Km, *ls, *dedx[3], *mtau[6], *fcond;
  /* surface */
  double *cd, *ch, *cq, *fricVel, *htFlux, *tskin, *invOblen, *z0m, *z0t, *qFlux, *qskin;
  /* large-scale forcing: slab means of rho, rho u, rho v, rho theta, rho q_v per level */
  double *lsfProf;
  int lsfN;
  /* decomposed directions: their halo columns hold the neighbouring slabs' cells */
  int peerX, peerY;
};

#define IX(o, i, j, k) (((size_t)(i) * (size_t)(o)->nyh + (size_t)(j)) * (size_t)(o)->nzh + (size_t)(k))
#define IJ(o, i, j) ((size_t)(i) * (size_t)(o)->nyh + (size_t)(j))

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

int ora_create(const fe_config *cfg, ora_domain **out) {
  ora_domain *o;
  int f;
  if (!cfg || !out || cfg->Nh != 3) return FE_ERR_ARG;
  o = (ora_domain *)calloc(1, sizeof(ora_domain));
  if (!o) return FE_ERR_NOMEM;
  o->c = *cfg;
  o->nxh = cfg->Nx + 6; o->nyh = cfg->Ny + 6; o->nzh = cfg->Nz + 6;
  o->n = (size_t)o->nxh * o->nyh * o->nzh;
  o->n2 = (size_t)o->nxh * o->nyh;
  o->iMin = 3; o->iMax = cfg->Nx + 3; o->jMin = 3; o->jMax = cfg->Ny + 3; o->kMin = 3; o->kMax = cfg->Nz + 3;
  o->dX = cfg->dX; o->dY = cfg->dY; o->dZ = cfg->dZ;
  o->dXi = 1.0 / cfg->dX; o->dYi = 1.0 / cfg->dY; o->dZi = 1.0 / cfg->dZ;
  o->ntke = (cfg->turbulenceSelector > 0 && cfg->TKESelector > 0) ? 1 : 0;
  o->nmoist = cfg->moistureSelector > 0 ? cfg->moistureNvars : 0;
  o->zPos = dalloc(o->n); o->J31 = dalloc(o->n); o->J32 = dalloc(o->n); o->J33 = dalloc(o->n);
  o->D = dalloc(o->n); o->invD = dalloc(o->n); o->rhoBS = dalloc(o->n); o->thBS = dalloc(o->n);
  for (f = 0; f < 5; f++) { o->fld[f] = dalloc(o->n); o->fld0[f] = dalloc(o->n); o->F[f] = dalloc(o->n); }
  o->tke = dalloc(o->n); o->tke0 = dalloc(o->n); o->Ftke = dalloc(o->n);
  for (f = 0; f < 2; f++) { o->moist[f] = dalloc(o->n); o->moist0[f] = dalloc(o->n); }
  for (f = 0; f < 3; f++) o->Fmoist[f] = dalloc(o->n);
  o->rhoInv = dalloc(o->n); o->pres = dalloc(o->n);
  o->ucf = dalloc(o->n); o->vcf = dalloc(o->n); o->wcf = dalloc(o->n);
  for (f = 0; f < 9; f++) o->tau[f] = dalloc(o->n);
  o->Km = dalloc(o->n); o->ls = dalloc(o->n);
  for (f = 0; f < 3; f++) o->dedx[f] = dalloc(o->n);
  for (f = 0; f < 6; f++) o->mtau[f] = dalloc(o->n);
  o->fcond = dalloc(o->n);
  o->cd = dalloc(o->n2); o->ch = dalloc(o->n2); o->cq = dalloc(o->n2); o->fricVel = dalloc(o->n2);
  o->htFlux = dalloc(o->n2); o->tskin = dalloc(o->n2); o->invOblen = dalloc(o->n2); o->z0m = dalloc(o->n2);
  o->z0t = dalloc(o->n2); o->qFlux = dalloc(o->n2); o->qskin = dalloc(o->n2);
  o->lsfProf = dalloc((size_t)5 * o->nzh);
  o->lsfN = cfg->lsfSelector > 0 ? (int)lroundf(cfg->lsf_freq / cfg->dt) : 1;
  if (o->lsfN < 1) o->lsfN = 1;
  if (!o->fcond || !o->qskin || !o->lsfProf) { ora_destroy(o); return FE_ERR_NOMEM; }
  *out = o;
  return FE_OK;
}

void ora_destroy(ora_domain *o) {
  int f;
  if (!o) return;
  free(o->zPos); free(o->J31); free(o->J32); free(o->J33); free(o->D); free(o->invD); free(o->rhoBS); free(o->thBS);
  for (f = 0; f < 5; f++) { free(o->fld[f]); free(o->fld0[f]); free(o->F[f]); }
  free(o->tke); free(o->tke0); free(o->Ftke);
  for (f = 0; f < 2; f++) { free(o->moist[f]); free(o->moist0[f]); }
  for (f = 0; f < 3; f++) free(o->Fmoist[f]);
  free(o->rhoInv); free(o->pres); free(o->ucf); free(o->vcf); free(o->wcf);
  for (f = 0; f < 9; f++) free(o->tau[f]);
  free(o->Km); free(o->ls);
  for (f = 0; f < 3; f++) free(o->dedx[f]);
  for (f = 0; f < 6; f++) free(o->mtau[f]);
  free(o->fcond);
  free(o->cd); free(o->ch); free(o->cq); free(o->fricVel); free(o->htFlux); free(o->tskin); free(o->invOblen);
  free(o->z0m); free(o->z0t); free(o->qFlux); free(o->qskin);
  free(o->lsfProf);
  free(o);
}

static void f2d(double *dst, const float *src, size_t n) {
  size_t i;
  if (!src) return;
  for (i = 0; i < n; i++) dst[i] = src[i];
}

int ora_set_grid(ora_domain *o, const float *zPos, const float *J31, const float *J32, const float *J33,
                 const float *D_Jac, const float *invD_Jac) {
  f2d(o->zPos, zPos, o->n); f2d(o->J31, J31, o->n); f2d(o->J32, J32, o->n); f2d(o->J33, J33, o->n);
  f2d(o->D, D_Jac, o->n); f2d(o->invD, invD_Jac, o->n);
  return FE_OK;
}

int ora_set_base_state(ora_domain *o, const float *bs) {
  f2d(o->rhoBS, bs, o->n);
  f2d(o->thBS, bs + o->n, o->n);
  return FE_OK;
}

int ora_set_state(ora_domain *o, const float *hydro, const float *sgstke, const float *moist) {
  int f;
  for (f = 0; f < 5; f++) f2d(o->fld[f], hydro + (size_t)f * o->n, o->n);
  if (o->ntke && sgstke) f2d(o->tke, sgstke, o->n);
  for (f = 0; f < o->nmoist; f++)
    if (moist) f2d(o->moist[f], moist + (size_t)f * o->n, o->n);
  return FE_OK;
}

int ora_set_state_f64(ora_domain *o, const double *hydro, const double *sgstke, const double *moist) {
  int f;
  for (f = 0; f < 5; f++) memcpy(o->fld[f], hydro + (size_t)f * o->n, o->n * sizeof(double));
  if (o->ntke && sgstke) memcpy(o->tke, sgstke, o->n * sizeof(double));
  for (f = 0; f < o->nmoist; f++)
    if (moist) memcpy(o->moist[f], moist + (size_t)f * o->n, o->n * sizeof(double));
  return FE_OK;
}

int ora_set_surface(ora_domain *o, const float *z0m, const float *z0t, const float *htFlux, const float *tskin,
                    const float *fricVel, const float *qFlux, const float *qskin) {
  f2d(o->z0m, z0m, o->n2); f2d(o->z0t, z0t, o->n2); f2d(o->htFlux, htFlux, o->n2); f2d(o->tskin, tskin, o->n2);
  f2d(o->fricVel, fricVel, o->n2); f2d(o->qFlux, qFlux, o->n2); f2d(o->qskin, qskin, o->n2);
  return FE_OK;
}

int ora_set_clock(ora_domain *o, double simTime, int simTime_it) {
  o->simTime = simTime;
  o->simTime_it = simTime_it;
  return FE_OK;
}

/* ------------------------------------------------------------------ boundary conditions */
/* Momentum base-state value (cuda_BCsDevice.cu:183-211). fld: 1=u, 2=v, else w. */
static double momentum_bs(const ora_domain *o, int fld, double z, double rho) {
  double zg = 0, vg = 0, grad = 0;
  if (fld == 1) { zg = o->c.z_Ug; vg = o->c.U_g; grad = o->c.Ug_grad; }
  else if (fld == 2) { zg = o->c.z_Vg; vg = o->c.V_g; grad = o->c.Vg_grad; }
  if (z < zg) return vg * rho;
  return (vg + grad * (z - zg)) * rho;
}

/* kind: 0 = base state below/above (rho, theta: cuda_BCsDevice.cu:120-150),
 *       1 = momentum (bottom copy, top geostrophic, :152-181),
 *       2 = bottom copy / top base (TKE with zero base, hydroCoreDevice.cu:516-529),
 *       3 = zero gradient both ends (moisture, :213-241). Then periodic x, then y
 *       (:67-118), applied in that order over all columns. */
static void apply_bcs(ora_domain *o, double *f, int kind, int momfld, const double *base) {
  int i, j, k;
  int Nxh = o->nxh, Nyh = o->nyh, kMin = o->kMin, kMax = o->kMax, iMin = o->iMin, iMax = o->iMax;
  int jMin = o->jMin, jMax = o->jMax;
  for (i = 0; i < Nxh; i++)
    for (j = 0; j < Nyh; j++) {
      for (k = 0; k < kMin; k++) {
        if (kind == 0) f[IX(o, i, j, k)] = base[IX(o, i, j, k)];
        else f[IX(o, i, j, k)] = f[IX(o, i, j, kMin)];
      }
      for (k = kMax; k < kMax + 3; k++) {
        if (kind == 0) f[IX(o, i, j, k)] = base[IX(o, i, j, k)];
        else if (kind == 1) f[IX(o, i, j, k)] = momentum_bs(o, momfld, o->zPos[IX(o, i, j, kMax - 1)], o->rhoBS[IX(o, i, j, kMax - 1)]);
        else if (kind == 2) f[IX(o, i, j, k)] = 0.0;
        else f[IX(o, i, j, k)] = f[IX(o, i, j, kMax - 1)];
      }
    }
  if (!o->peerX)
    for (j = 0; j < Nyh; j++)
      for (k = 0; k < o->nzh; k++) {
        for (i = 0; i < iMin; i++) f[IX(o, i, j, k)] = f[IX(o, iMax - 3 + i, j, k)];
        for (i = iMax; i < iMax + 3; i++) f[IX(o, i, j, k)] = f[IX(o, i - iMax + 3, j, k)];
      }
  if (!o->peerY)
    for (i = 0; i < Nxh; i++)
      for (k = 0; k < o->nzh; k++) {
        for (j = 0; j < jMin; j++) f[IX(o, i, j, k)] = f[IX(o, i, jMax - 3 + j, k)];
        for (j = jMax; j < jMax + 3; j++) f[IX(o, i, j, k)] = f[IX(o, i, j - jMax + 3, k)];
      }
}

/* A slab of a decomposed domain (fempi.c:98-160 rank grid): the caller writes the x (y) halo
   columns from the neighbouring slabs before every stage (the exchange of
   cuda_hydroCoreDevice.cu:276-314); the boundary pass then keeps them and applies only the
   vertical rules on them. */
int ora_set_decomposition(ora_domain *o, int peerX, int peerY) {
  o->peerX = peerX != 0;
  o->peerY = peerY != 0;
  return FE_OK;
}

/* ------------------------------------------------------------------ advection */
static double sgn1(double x) { return copysign(1.0, x); }

/* HYB56 flux divergence (cuda_advectionDevice.cu:318-380), b = b_hyb. */
static double hyb56(const ora_domain *o, const double *s, int i, int j, int k, double b) {
  size_t c = IX(o, i, j, k);
  size_t si = (size_t)o->nyh * o->nzh, sj = (size_t)o->nzh, sk = 1;
  size_t st[3] = {si, sj, sk};
  const double *vel[3] = {o->ucf, o->vcf, o->wcf};
  double div = 0.0;
  int d;
  for (d = 0; d < 3; d++) {
    size_t q = st[d];
    double p1 = s[c + q], p2 = s[c + 2 * q], p3 = s[c + 3 * q], z0 = s[c], m1 = s[c - q], m2 = s[c - 2 * q], m3 = s[c - 3 * q];
    double fp = (37.0 * (p1 + z0) - 8.0 * (p2 + m1) + (p3 + m2) -
                 (1.0 - b) * sgn1(vel[d][c + q]) * ((p3 - m2) - 5.0 * (p2 - m1) + 10.0 * (p1 - z0))) / 60.0;
    double fm = (37.0 * (z0 + m1) - 8.0 * (p1 + m2) + (p2 + m3) -
                 (1.0 - b) * sgn1(vel[d][c]) * ((p2 - m3) - 5.0 * (p1 - m2) + 10.0 * (z0 - m1))) / 60.0;
    div += vel[d][c + q] * fp - vel[d][c] * fm;
  }
  return -o->invD[c] * div;
}

/* WENO5 face value on the upwind side: stencil a,b,c,d,e = s[-2..+2] around the
 * left cell of the face (cuda_advectionDevice.cu:626-926). */
static double weno5_face(double a, double b, double c, double d, double e) {
  double g1 = 0.1, g2 = 0.6, g3 = 0.3, tol = 1e-6;
  double f1 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
  double f2 = -(1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
  double f3 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
  double b1 = (13.0 / 12.0) * pow(a - 2.0 * b + c, 2.0) + 0.25 * pow(a - 4.0 * b + 3.0 * c, 2.0);
  double b2 = (13.0 / 12.0) * pow(b - 2.0 * c + d, 2.0) + 0.25 * pow(b - d, 2.0);
  double b3 = (13.0 / 12.0) * pow(c - 2.0 * d + e, 2.0) + 0.25 * pow(3.0 * c - 4.0 * d + e, 2.0);
  double w1 = g1 / pow(tol + b1, 2.0), w2 = g2 / pow(tol + b2, 2.0), w3 = g3 / pow(tol + b3, 2.0);
  double ws = w1 + w2 + w3;
  return (w1 / ws) * f1 + (w2 / ws) * f2 + (w3 / ws) * f3;
}

static double weno5(const ora_domain *o, const double *s, int i, int j, int k) {
  size_t c = IX(o, i, j, k);
  size_t si = (size_t)o->nyh * o->nzh, sj = (size_t)o->nzh, sk = 1;
  size_t st[3] = {si, sj, sk};
  const double *vel[3] = {o->ucf, o->vcf, o->wcf};
  double tot = 0.0;
  int d;
  for (d = 0; d < 3; d++) {
    size_t q = st[d];
    double m3 = s[c - 3 * q], m2 = s[c - 2 * q], m1 = s[c - q], z0 = s[c], p1 = s[c + q], p2 = s[c + 2 * q], p3 = s[c + 3 * q];
    double fpP = weno5_face(m2, m1, z0, p1, p2);
    double fpN = weno5_face(p3, p2, p1, z0, m1);
    double fmP = weno5_face(m3, m2, m1, z0, p1);
    double fmN = weno5_face(p2, p1, z0, m1, m2);
    double sp = sgn1(vel[d][c + q]), sm = sgn1(vel[d][c]);
    double fp = 0.5 * (1.0 + sp) * fpP + 0.5 * (1.0 - sp) * fpN;
    double fm = 0.5 * (1.0 + sm) * fmP + 0.5 * (1.0 - sm) * fmN;
    tot += -o->invD[c] * (vel[d][c + q] * fp - vel[d][c] * fm);
  }
  return tot;
}

/* Face value of the lower-order schemes on the face between cells z0 (lower) and p1 (upper),
 * stencil m1..p2; u = face velocity (cuda_advectionDevice.cu:126-312, 382-623):
 *   0 upwind  max(0,u) z0 + min(0,u) p1 (returned divided by u: the flux is u times the value)
 *   1 QUICK   [max(0,u)(6 z0 + 3 p1 - m1) + min(0,u)(6 p1 + 3 z0 - p2)] / 8, likewise
 *   2 HYB34   (7(p1+z0) - (p2+m1) + (1-b) sgn(u) ((p2-m1) - 3(p1-z0))) / 12
 *   4 WENO3   two-candidate WENO on the upwind side, weights g/(tol+beta)^2, g = 1/3, 2/3
 *   6 centred (z0 + p1) / 2 */
static double weno3_side(double a, double b, double c) {
  double g1 = 1.0 / 3.0, g2 = 2.0 / 3.0, tol = 1e-6;
  double f1 = -0.5 * a + 1.5 * b, f2 = 0.5 * b + 0.5 * c;
  double w1 = g1 / pow(tol + pow(b - a, 2.0), 2.0), w2 = g2 / pow(tol + pow(c - b, 2.0), 2.0);
  return (w1 / (w1 + w2)) * f1 + (w2 / (w1 + w2)) * f2;
}

static double low_order_face(int sel, double m1, double z0, double p1, double p2, double u, double b) {
  double up = u > 0.0;
  switch (sel) {
    case 0: return up ? z0 : p1;
    case 1: return up ? (6.0 * z0 + 3.0 * p1 - m1) / 8.0 : (6.0 * p1 + 3.0 * z0 - p2) / 8.0;
    case 2: return (7.0 * (p1 + z0) - (p2 + m1) + (1.0 - b) * sgn1(u) * ((p2 - m1) - 3.0 * (p1 - z0))) / 12.0;
    case 4: return sgn1(u) > 0.0 ? weno3_side(m1, z0, p1) : weno3_side(p2, p1, z0);
    default: return 0.5 * (z0 + p1);
  }
}

/* Flux divergence of a lower-order scheme: -invD sum_d (u+ f+ - u- f-). */
static double low_order(const ora_domain *o, const double *s, int i, int j, int k, int sel, double b) {
  size_t c = IX(o, i, j, k);
  size_t st[3] = {(size_t)o->nyh * o->nzh, (size_t)o->nzh, 1};
  const double *vel[3] = {o->ucf, o->vcf, o->wcf};
  double div = 0.0;
  int d;
  for (d = 0; d < 3; d++) {
    size_t q = st[d];
    double m2 = s[c - 2 * q], m1 = s[c - q], z0 = s[c], p1 = s[c + q], p2 = s[c + 2 * q];
    double fp = low_order_face(sel, m1, z0, p1, p2, vel[d][c + q], b);
    double fm = low_order_face(sel, m2, m1, z0, p1, vel[d][c], b);
    div += vel[d][c + q] * fp - vel[d][c] * fm;
  }
  return -o->invD[c] * div;
}

static double advect(const ora_domain *o, const double *s, int i, int j, int k, int sel, double b) {
  if (sel == 3) return hyb56(o, s, i, j, k, b);
  if (sel == 5) return weno5(o, s, i, j, k);
  return low_order(o, s, i, j, k, sel, b);
}

/* q_l's scheme (moistureAdvSelectorQi: 0 upwind, 1 WENO3, 2 WENO5; cuda_hydroCoreDevice.cu:725-736). */
static double advect_ql(const ora_domain *o, const double *s, int i, int j, int k, int qi) {
  if (qi == 2) return weno5(o, s, i, j, k);
  return low_order(o, s, i, j, k, qi == 1 ? 4 : 0, 0.0);
}

/* 6th-order vertical filter of rho w (cuda_filtersDevice.cu:73-122): flux-limited so that it
 * only diffuses down-gradient; coefficient 0.015625 filter_6th_coeff / dt. */
static double filter6(const ora_domain *o, const double *s, int i, int j, int k) {
  size_t c = IX(o, i, j, k);
  double coef = 0.015625 * o->c.filter_6th_coeff / o->c.dt;
  double fm = 10.0 * (s[c] - s[c - 1]) - 5.0 * (s[c + 1] - s[c - 2]) + (s[c + 2] - s[c - 3]);
  double fp = 10.0 * (s[c + 1] - s[c]) - 5.0 * (s[c + 2] - s[c - 1]) + (s[c + 3] - s[c - 2]);
  if (signbit((s[c] - s[c - 1]) * fm)) fm = 0.0;
  if (signbit((s[c + 1] - s[c]) * fp)) fp = 0.0;
  return coef * (fp - fm);
}

/* ------------------------------------------------------------------ surface layer */
/* Land-surface update (cuda_surfaceLayerDevice.cu:112-195 dry, :199-318 moist). */
static void surface_lsm(ora_domain *o, int i, int j, int stage) {
  size_t ij = IJ(o, i, j), c = IX(o, i, j, o->kMin);
  int moist = o->c.moistureSelector > 0;
  double pi = acos(-1.0);
  double dt = o->c.dt;
  int temp_freq = (int)lround(10.0 / dt);
  double temp_freq_f = temp_freq;
  double z0 = o->z0m[ij], z1 = 0.5 / (o->dZi * o->J33[c]);
  double z1oz0 = (z1 + z0) / z0, z0t = o->z0t[ij], z1ozt0 = (z1 + z0t) / z0t;
  double rho = o->fld[0][c];
  double u1 = o->fld[1][c] / rho, v1 = o->fld[2][c] / rho;
  double U1 = sqrt(u1 * u1 + v1 * v1), th1 = o->fld[4][c] / rho;
  double q1 = moist ? o->moist[0][c] / rho : 0.0;
  double rcp = pow(o->c.refPressure / o->c.pres_grnd, o->c.R_cp);
  double qsk_input = o->qskin[ij];
  double simTime = o->simTime;
  int it = o->simTime_it, itr = o->c.simTime_itRestart;
  if (it == itr && it == 0) {
    o->cd[ij] = pow(o->c.kappa, 2.0) / pow(log(z1oz0), 2.0);
    o->ch[ij] = pow(o->c.kappa, 2.0) / pow(log(z1ozt0), 2.0);
    if (moist) o->cq[ij] = pow(o->c.kappa, 2.0) / pow(log(z1ozt0), 2.0);
  } else if (it == itr && it != 0) {
    double th0 = o->tskin[ij] * rcp;
    o->cd[ij] = pow(o->fricVel[ij], 2.0) / pow(U1, 2.0);
    o->ch[ij] = o->htFlux[ij] / (U1 * (th0 - th1));
    if (moist) o->cq[ij] = o->qFlux[ij] / (U1 * (o->qskin[ij] - q1));
  }
  if (o->c.surflayerSelector == 1) {
    if (o->c.surflayer_idealsine == 1) {
      double ts = o->c.surflayer_ideal_ts, te = o->c.surflayer_ideal_te;
      o->htFlux[ij] = (simTime > ts && simTime <= te)
                          ? o->c.surflayer_wth + o->c.surflayer_ideal_amp * sin(pi * (simTime - ts) / (te - ts))
                          : o->c.surflayer_wth;
      if (moist) {
        double qts = o->c.surflayer_ideal_qts, qte = o->c.surflayer_ideal_qte;
        o->qFlux[ij] = (simTime > qts && simTime <= qte) ? o->c.surflayer_ideal_qamp * sin(pi * (simTime - qts) / (qte - qts))
                                                         : o->c.surflayer_wq;
      }
    }
  } else if (o->c.surflayerSelector == 2) {
    double tsk_c, qsk_c = 0.0;
    if ((it % temp_freq) == 0 && stage == 2) {
      double ts = o->c.surflayer_ideal_ts, te = o->c.surflayer_ideal_te;
      if (o->c.surflayer_idealsine == 1 && simTime > ts && simTime < te + dt * temp_freq_f) {
        double prev = simTime - temp_freq_f * dt;
        if (prev < ts) prev = ts;
        tsk_c = o->tskin[ij] + o->c.surflayer_ideal_amp * (sin(pi * (simTime - ts) / (te - ts)) - sin(pi * (prev - ts) / (te - ts)));
        if (moist) {
          double qts = o->c.surflayer_ideal_qts, qte = o->c.surflayer_ideal_qte;
          qsk_c = o->qskin[ij] + o->c.surflayer_ideal_qamp * (sin(pi * (simTime - qts) / (qte - qts)) - sin(pi * (prev - qts) / (qte - qts)));
        }
      } else {
        tsk_c = o->tskin[ij] + o->c.surflayer_tr * dt * temp_freq_f / 3600.0;
        if (moist) qsk_c = o->qskin[ij] + o->c.surflayer_qr * dt * temp_freq_f / 3600.0;
      }
      o->tskin[ij] = tsk_c;
      if (moist) o->qskin[ij] = qsk_c;
    } else {
      tsk_c = o->tskin[ij];
      if (moist) qsk_c = o->qskin[ij];
    }
    o->htFlux[ij] = o->ch[ij] * U1 * (tsk_c * rcp - th1);
    if (moist) {
      o->qFlux[ij] = o->cq[ij] * U1 * (qsk_c - q1);
      if (o->c.surflayer_qskin_input == 1) o->qskin[ij] = qsk_input;
    }
  }
}

/* Monin-Obukhov iteration (cuda_surfaceLayerDevice.cu:322-414 dry, :418-521 moist). */
static void surface_most(ora_domain *o, int i, int j) {
  size_t ij = IJ(o, i, j), c = IX(o, i, j, o->kMin);
  int moist = o->c.moistureSelector > 0;
  double pi = acos(-1.0), beta = 5.0, ol_lim = 1.0;
  double kap = o->c.kappa, g = o->c.accel_g;
  int it_max = o->c.surflayer_stab == 0 ? 5 : 1, it_n = 0;
  double z0 = o->z0m[ij], z1 = 0.5 / (o->dZi * o->J33[c]);
  double z1oz0 = (z1 + z0) / z0, z0t = o->z0t[ij], z1ozt0 = (z1 + z0t) / z0t;
  double rho = o->fld[0][c], uu = o->fld[1][c], vv = o->fld[2][c];
  double u1 = uu / rho, v1 = vv / rho, U1 = sqrt(u1 * u1 + v1 * v1), th1 = o->fld[4][c] / rho;
  double th0 = o->tskin[ij] * pow(o->c.refPressure / o->c.pres_grnd, o->c.R_cp);
  double q1 = moist ? o->moist[0][c] / rho : 0.0, q0 = moist ? o->qskin[ij] : 0.0;
  double cd0 = o->cd[ij], cdi = 0, chi = 0, cqi = 0, tx, ty, zol, psim, psih;
  do {
    tx = -cd0 * U1 * u1;
    ty = -cd0 * U1 * v1;
    o->fricVel[ij] = pow(tx * tx + ty * ty, 0.25);
    it_n++;
    if (o->c.surflayer_stab == 0) {
      if (o->fricVel[ij] > 0.0) {
        double iol = -(kap * g * o->htFlux[ij]) / (pow(o->fricVel[ij], 3.0) * th1);
        o->invOblen[ij] = fmax(fmin(iol, ol_lim), -ol_lim);
      } else {
        o->invOblen[ij] = -ol_lim;
      }
    } else {
      o->invOblen[ij] = 0.0;
    }
    zol = o->invOblen[ij] * (z1 + z0);
    if (zol < 0.0) {
      double xi = pow(1.0 - 16.0 * zol, 0.25);
      psim = log(0.5 * (1.0 + xi * xi) * pow(0.5 * (1.0 + xi), 2.0)) - 2.0 * atan(xi) + 0.5 * pi;
      psih = 2.0 * log(0.5 * (1.0 + xi * xi));
    } else {
      psim = -beta * zol;
      psih = -beta * zol;
    }
    cdi = kap * kap / pow(log(z1oz0) - psim, 2.0);
    chi = kap * kap / ((log(z1ozt0) - psim) * (log(z1ozt0) - psih));
    cqi = chi;
    if (o->c.surflayerSelector > 1) {
      o->htFlux[ij] = chi * U1 * (th0 - th1);
      if (moist) o->qFlux[ij] = cqi * U1 * (q0 - q1);
    }
    cd0 = cdi;
  } while (it_n <= it_max);
  o->cd[ij] = cdi;
  o->ch[ij] = chi;
  if (moist) o->cq[ij] = cqi;
  tx = -cdi * sqrt(pow(uu / rho, 2.0) + pow(vv / rho, 2.0)) * uu;
  ty = -cdi * sqrt(pow(uu / rho, 2.0) + pow(vv / rho, 2.0)) * vv;
  o->tau[2][c] = tx;
  o->tau[3][c] = ty;
  o->fricVel[ij] = pow(tx * tx + ty * ty, 0.25);
  o->tau[8][c] = o->htFlux[ij] * rho;
  if (moist) o->mtau[2][c] = o->qFlux[ij] * rho;
  o->invOblen[ij] = -(kap * g * o->htFlux[ij]) / (pow(o->fricVel[ij], 3.0) * th1);
}

/* ------------------------------------------------------------------ one tendency */
/* ------------------------------------------------------------------ large-scale forcing */
/* Steps that take the slab means and apply the forcing (cuda_timeIntDevice.cu:125-127,
 * cuda_hydroCoreDevice.cu:401-406). */
static int lsf_means_step(const ora_domain *o) {
  return o->c.lsfSelector > 0 && o->c.lsf_horMnSubTerms == 1 && o->simTime_it > o->c.simTime_itRestart &&
         o->simTime_it % o->lsfN == 0;
}
static int lsf_force_step(const ora_domain *o) {
  int d = o->simTime_it - o->c.simTime_itRestart;
  return o->c.lsfSelector > 0 && d > 0 && d >= o->lsfN && o->simTime_it % o->lsfN == 0;
}

/* Slab means over every column of the halo-inclusive plane (cuda_largeScaleForcingsDevice.cu:96-138,
 * fecuda_PlugIns.cu:25-45) of the arrays as they are: at the start of a step their halo cells
 * hold the boundary values of the previous step's last-stage input, as the reference's do. */
static void lsf_slab_means(ora_domain *o) {
  const double *src[5] = {o->fld[0], o->fld[1], o->fld[2], o->fld[4], o->nmoist > 0 ? o->moist[0] : NULL};
  double inv = 1.0 / ((double)o->nxh * (double)o->nyh);
  int f, i, j, k;
  for (f = 0; f < 5; f++)
    for (k = 0; k < o->nzh; k++) {
      double sum = 0.0;
      if (src[f])
        for (i = 0; i < o->nxh; i++)
          for (j = 0; j < o->nyh; j++) sum += src[f][IX(o, i, j, k)];
      o->lsfProf[f * o->nzh + k] = sum * inv;
    }
}

/* Piecewise-linear forcing profile (surface, lev1 at zlev1, lev2 at zlev2, constant above)
 * times rho, per second over the application interval (cuda_largeScaleForcingsDevice.cu:177-230). */
static double lsf_profile(double surf, double lev1, double lev2, double z1, double z2, double z, double rho,
                          int nsteps) {
  double f;
  if (z <= z1) f = (surf + (lev1 - surf) / z1 * z) * rho;
  else if (z <= z2) f = (lev1 + (lev2 - lev1) / (z2 - z1) * (z - z1)) * rho;
  else f = lev2 * rho;
  return f * nsteps / 3600.0;
}

static int build_frhs(ora_domain *o, int stage, int fresh_means);

int ora_build_frhs(ora_domain *o, int stage) { return build_frhs(o, stage, 1); }

/* fresh_means: a tendency evaluated on its own takes the slab means of its input state (after
 * its boundary values are set); inside a step they were taken at the step's start. */
static int build_frhs(ora_domain *o, int stage, int fresh_means) {
  const fe_config *C = &o->c;
  int i, j, k, f;
  int iMin = o->iMin, iMax = o->iMax, jMin = o->jMin, jMax = o->jMax, kMin = o->kMin, kMax = o->kMax;
  size_t si = (size_t)o->nyh * o->nzh, sj = (size_t)o->nzh;
  double dXi = o->dXi, dYi = o->dYi, dZi = o->dZi;
  int physics = (C->physics_oneRKonly == 0) || (stage == 2);
  int turb = C->turbulenceSelector > 0 && physics;
  int moistOn = o->nmoist > 0;
  double c1 = C->R_gas / pow(C->refPressure, C->R_cp);
  double *rho = o->fld[0], *u = o->fld[1], *v = o->fld[2], *w = o->fld[3], *th = o->fld[4];

  /* 1. Commence: BCs and zeroed tendencies (cuda_hydroCoreDevice.cu:431-556) */
  apply_bcs(o, o->fld[0], 0, 0, o->rhoBS);
  apply_bcs(o, o->fld[1], 1, 1, NULL);
  apply_bcs(o, o->fld[2], 1, 2, NULL);
  apply_bcs(o, o->fld[3], 1, 3, NULL);
  apply_bcs(o, o->fld[4], 0, 0, o->thBS);
  for (f = 0; f < 5; f++) memset(o->F[f], 0, o->n * sizeof(double));
  memset(o->Km, 0, o->n * sizeof(double));
  memset(o->Ftke, 0, o->n * sizeof(double));
  if (o->ntke) apply_bcs(o, o->tke, 2, 0, NULL);
  for (f = 0; f < 3; f++) memset(o->Fmoist[f], 0, o->n * sizeof(double));
  for (f = 0; f < o->nmoist; f++) apply_bcs(o, o->moist[f], 3, 0, NULL);

  /* 2. rho^-1 and perturbation pressure (cuda_hydroCoreDevice.cu:558-589,
   *    cuda_pressureDevice.cu:53-113) */
  for (i = 0; i < o->nxh; i++)
    for (j = 0; j < o->nyh; j++)
      for (k = 0; k < o->nzh; k++) {
        size_t c = IX(o, i, j, k), t = c;
        double rtm;
        o->rhoInv[c] = 1.0 / fmax(rho[c], 1e-6);
        if (k > 0 && k < kMin) t = IX(o, i, j, kMin);
        else if (k >= kMax) t = IX(o, i, j, kMax - 1);
        rtm = th[t];
        if (moistOn) rtm = th[t] * (1.0 + C->Rv_Rg * o->moist[0][t] / rho[t] * 1e-3);
        o->pres[c] = pow(rtm * c1, C->cp_cv) - pow(o->thBS[t] * c1, C->cp_cv);
      }

  /* 3a. cell-face velocities (cuda_advectionDevice.cu:54-121) */
  memset(o->ucf, 0, o->n * sizeof(double));
  memset(o->vcf, 0, o->n * sizeof(double));
  memset(o->wcf, 0, o->n * sizeof(double));
  for (i = iMin; i <= iMax; i++)
    for (j = jMin; j <= jMax; j++)
      for (k = kMin; k <= kMax; k++) {
        size_t c = IX(o, i, j, k), im = c - si, jm = c - sj, km = c - 1;
        o->ucf[c] = 0.5 * dXi * ((o->D[c] / rho[c]) * (u[c] + w[c] * o->J31[c]) + (o->D[im] / rho[im]) * (u[im] + w[im] * o->J31[im]));
        o->vcf[c] = 0.5 * dYi * ((o->D[c] / rho[c]) * (v[c] + w[c] * o->J32[c]) + (o->D[jm] / rho[jm]) * (v[jm] + w[jm] * o->J32[jm]));
        o->wcf[c] = 0.5 * dZi * ((o->D[c] / rho[c]) * (w[c] * o->J33[c]) + (o->D[km] / rho[km]) * (w[km] * o->J33[km]));
        if (k == kMin || k >= kMax) o->wcf[c] = 0.0;
      }

  /* 3b. pressure-gradient force (cuda_pressureDevice.cu:118-194) */
  if (C->pgfSelector > 0)
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++)
        for (k = kMin; k < kMax; k++) {
          size_t c = IX(o, i, j, k);
          double *p = o->pres, fac = 1.0;
          double dpx = p[c + si] - p[c - si], dpy = p[c + sj] - p[c - sj], dpz = p[c + 1] - p[c - 1];
          if (moistOn) {
            double rmd = 1.0;
            for (f = 0; f < o->nmoist; f++) rmd += o->moist[f][c] / rho[c] * 1e-3;
            fac = 1.0 / rmd;
          }
          o->F[1][c] -= fac * 0.5 * dXi * dpx;
          o->F[2][c] -= fac * 0.5 * dYi * dpy;
          o->F[3][c] -= fac * 0.5 * (dXi * o->J31[c] * dpx + dYi * o->J32[c] * dpy + dZi * o->J33[c] * dpz);
        }

  /* 3c. SGS turbulence, last stage only (cuda_hydroCoreDevice.cu:836-891) */
  if (turb) {
    double *ri = o->rhoInv;
    double **T = o->tau;
    /* strain rates and theta gradients (cuda_sgsTurbDevice.cu:60-197) on the ring */
    for (i = iMin - 1; i < iMax + 1; i++)
      for (j = jMin - 1; j < jMax + 1; j++)
        for (k = kMin; k < kMax + 1; k++) {
          size_t c = IX(o, i, j, k), a = c - si, b = c - sj, d = c - 1, ab = c - si - sj, ad = c - si - 1, bd = c - sj - 1,
                 abd = c - si - sj - 1;
          double J1 = o->J31[c], J2 = o->J32[c], J3 = o->J33[c];
#define U_(x) (u[x] * ri[x])
#define V_(x) (v[x] * ri[x])
#define W_(x) (w[x] * ri[x])
#define TH_(x) (th[x] * ri[x])
          T[0][c] = dXi * (U_(c) - U_(a));
          T[4][c] = dYi * (V_(c) - V_(b));
          T[5][c] = J1 * dXi * (W_(c) - W_(a)) + J2 * dYi * (W_(c) - W_(b)) + J3 * dZi * (W_(c) - W_(d));
          T[1][c] = 0.5 * (0.5 * (dXi * (V_(c) - V_(a)) + dXi * (V_(b) - V_(ab))) +
                           0.5 * (dYi * (U_(c) - U_(b)) + dYi * (U_(a) - U_(ab))));
          T[2][c] = 0.5 * (0.5 * (dXi * (W_(c) - W_(a)) + dXi * (W_(d) - W_(ad))) +
                           0.5 * (J1 * dXi * (U_(c) - U_(a)) + J1 * dXi * (U_(d) - U_(ad))) +
                           0.25 * (J2 * dYi * (U_(c) - U_(b)) + J2 * dYi * (U_(a) - U_(ab)) + J2 * dYi * (U_(d) - U_(bd)) +
                                   J2 * dYi * (U_(ad) - U_(abd))) +
                           0.5 * (J3 * dZi * (U_(c) - U_(d)) + J3 * dZi * (U_(a) - U_(ad))));
          T[3][c] = 0.5 * (0.5 * (dYi * (W_(c) - W_(b)) + dYi * (W_(d) - W_(bd))) +
                           0.25 * (J1 * dXi * (V_(c) - V_(a)) + J1 * dXi * (V_(b) - V_(ab)) + J1 * dXi * (V_(d) - V_(ad)) +
                                   J1 * dXi * (V_(bd) - V_(abd))) +
                           0.5 * (J2 * dYi * (V_(c) - V_(b)) + J2 * dYi * (V_(d) - V_(bd))) +
                           0.5 * (J3 * dZi * (V_(c) - V_(d)) + J3 * dZi * (V_(b) - V_(bd))));
          T[6][c] = dXi * (TH_(c) - TH_(a));
          T[7][c] = dYi * (TH_(c) - TH_(b));
          T[8][c] = J1 * dXi * (TH_(c) - TH_(a)) + J2 * dYi * (TH_(c) - TH_(b)) + J3 * dZi * (TH_(c) - TH_(d));
        }
    /* moisture gradients to faces (cuda_sgsTurbDevice.cu:372-402) */
    if (moistOn && C->moistureSGSturb > 0)
      for (f = 0; f < o->nmoist; f++)
        for (i = iMin - 1; i < iMax + 1; i++)
          for (j = jMin - 1; j < jMax + 1; j++)
            for (k = kMin - 1; k < kMax + 1; k++) {
              size_t c = IX(o, i, j, k);
              double *q = o->moist[f];
              double qc = q[c] * ri[c], qa = q[c - si] * ri[c - si], qb = q[c - sj] * ri[c - sj], qd = q[c - 1] * ri[c - 1];
              o->mtau[3 * f + 0][c] = dXi * (qc - qa);
              o->mtau[3 * f + 1][c] = dYi * (qc - qb);
              o->mtau[3 * f + 2][c] = o->J31[c] * dXi * (qc - qa) + o->J32[c] * dYi * (qc - qb) + o->J33[c] * dZi * (qc - qd);
            }
    if (o->ntke) {
      /* length scale (cuda_sgstkeDevice.cu:96-151) */
      for (i = iMin - 1; i < iMax + 1; i++)
        for (j = jMin - 1; j < jMax + 1; j++)
          for (k = kMin - 1; k < kMax + 1; k++) {
            size_t c = IX(o, i, j, k);
            double dthdz = 0.5 * (o->J31[c] * dXi * (TH_(c + si) - TH_(c - si)) + o->J32[c] * dYi * (TH_(c + sj) - TH_(c - sj)) +
                                  o->J33[c] * dZi * (TH_(c + 1) - TH_(c - 1)));
            double N2 = (C->accel_g / TH_(c)) * dthdz;
            double len2 = pow((double)o->dX * o->dY * o->dZ * o->D[c], 1.0 / 3.0);
            if (N2 > 0.0) {
              double e = o->tke[c] * ri[c];
              double len1 = 0.76 * pow(e, 0.5) * pow(N2, -0.5);
              o->ls[c] = fmax(fmin(len1, len2), 1e-2);
            } else {
              o->ls[c] = len2;
            }
          }
      /* Km (cuda_sgsTurbDevice.cu:202-254, Lilly branch) */
      for (i = iMin - 1; i < iMax + 1; i++)
        for (j = jMin - 1; j < jMax + 1; j++)
          for (k = kMin; k < kMax + 1; k++) {
            size_t c = IX(o, i, j, k);
            double e0 = o->tke[c] * ri[c], e1 = o->tke[c - 1] * ri[c - 1];
            o->Km[c] += C->c_k * 0.5 * (o->ls[c] * pow(e0, 0.5) + o->ls[c - 1] * pow(e1, 0.5));
          }
      /* grad e (cuda_sgstkeDevice.cu:309-343) */
      for (i = iMin - 1; i < iMax + 1; i++)
        for (j = jMin - 1; j < jMax + 1; j++)
          for (k = kMin - 1; k < kMax + 1; k++) {
            size_t c = IX(o, i, j, k);
            double *e = o->tke;
            double ex = e[c + si] * ri[c + si] - e[c - si] * ri[c - si];
            double ey = e[c + sj] * ri[c + sj] - e[c - sj] * ri[c - sj];
            double ez = e[c + 1] * ri[c + 1] - e[c - 1] * ri[c - 1];
            o->dedx[0][c] = 0.5 * (dXi * ex);
            o->dedx[1][c] = 0.5 * (dYi * ey);
            o->dedx[2][c] = 0.5 * (o->J31[c] * dXi * ex + o->J32[c] * dYi * ey + o->J33[c] * dZi * ez);
          }
      /* stresses with the deviatoric TKE term (cuda_sgsTurbDevice.cu:308-367) */
      for (i = iMin - 1; i < iMax + 1; i++)
        for (j = jMin - 1; j < jMax + 1; j++)
          for (k = kMin; k < kMax + 1; k++) {
            size_t c = IX(o, i, j, k), a = c - si, b = c - sj, d = c - 1;
            double delta = pow((double)o->dX * o->dY * o->dZ * o->D[c], 1.0 / 3.0);
            double invPr = 1.0 + 2.0 * o->ls[c] / delta;
            double r = rho[c], km = o->Km[c];
            double dev = (2.0 / 3.0) * r *
                         (km * (dXi * (u[c] / r - u[a] / rho[a]) + dYi * (v[c] / r - v[b] / rho[b]) +
                                o->J31[c] * dXi * (w[c] / r - w[a] / rho[a]) + o->J32[c] * dYi * (w[c] / r - w[b] / rho[b]) +
                                o->J33[c] * dZi * (w[c] / r - w[d] / rho[d])) +
                          o->tke[c] / r);
            T[0][c] = -2.0 * r * km * T[0][c] + dev;
            T[1][c] = -2.0 * r * km * T[1][c];
            T[2][c] = -2.0 * r * km * T[2][c];
            T[3][c] = -2.0 * r * km * T[3][c];
            T[4][c] = -2.0 * r * km * T[4][c] + dev;
            T[5][c] = -2.0 * r * km * T[5][c] + dev;
            T[6][c] = -r * km * invPr * T[6][c];
            T[7][c] = -r * km * invPr * T[7][c];
            T[8][c] = -r * km * invPr * T[8][c];
          }
    } else {
      /* Smagorinsky (cuda_sgsTurbDevice.cu:226-238, 259-302) */
      for (i = iMin - 1; i < iMax + 1; i++)
        for (j = jMin - 1; j < jMax + 1; j++)
          for (k = kMin; k < kMax + 1; k++) {
            size_t c = IX(o, i, j, k);
            double delta = pow((double)o->dX * o->dY * o->dZ * o->D[c], 1.0 / 3.0);
            double t1 = 0.5 * (T[0][c] * T[0][c] + T[4][c] * T[4][c] + T[5][c] * T[5][c]) + T[1][c] * T[1][c] +
                        T[2][c] * T[2][c] + T[3][c] * T[3][c];
            double N2 = C->accel_g / TH_(c) * T[8][c];
            double t2 = N2 * 3.0;
            double km, invPr, r = rho[c];
            o->Km[c] += (C->c_s * delta) * (C->c_s * delta) * sqrt(fmax(0.0, t1 - fmax(0.0, t2)));
            km = o->Km[c];
            invPr = 1.0 + 2.0 * delta / delta;
            for (f = 0; f < 6; f++) T[f][c] = -2.0 * r * km * T[f][c];
            for (f = 6; f < 9; f++) T[f][c] = -r * km * invPr * T[f][c];
          }
    }
    /* moisture SGS fluxes (cuda_sgsTurbDevice.cu:407-442) */
    if (moistOn && C->moistureSGSturb > 0)
      for (f = 0; f < o->nmoist; f++)
        for (i = iMin - 1; i < iMax + 1; i++)
          for (j = jMin - 1; j < jMax + 1; j++)
            for (k = kMin; k < kMax + 1; k++) {
              size_t c = IX(o, i, j, k);
              double delta = pow((double)o->dX * o->dY * o->dZ * o->D[c], 1.0 / 3.0);
              double lsc = o->ntke ? o->ls[c] : delta;
              double invPr = 1.0 + 2.0 * lsc / delta;
              int m;
              for (m = 0; m < 3; m++) o->mtau[3 * f + m][c] = -rho[c] * o->Km[c] * invPr * o->mtau[3 * f + m][c];
            }
#undef U_
#undef V_
#undef W_
#undef TH_
  }

  /* 3d. surface layer at k = kMin (cuda_hydroCoreDevice.cu:907-945) */
  if (C->surflayerSelector > 0 && physics)
    for (i = iMin; i <= iMax + 1; i++)
      for (j = jMin; j <= jMax + 1; j++) {
        surface_lsm(o, i, j, stage);
        surface_most(o, i, j);
      }

  /* 4. advection, Rayleigh, buoyancy, Coriolis, SGS mixing (cuda_hydroCoreDevice.cu:591-778) */
  for (i = iMin; i < iMax; i++)
    for (j = jMin; j < jMax; j++)
      for (k = kMin; k < kMax; k++) {
        size_t c = IX(o, i, j, k);
        for (f = 0; f < 5; f++) {
          o->F[f][c] += advect(o, o->fld[f], i, j, k, C->advectionSelector, C->b_hyb);
          if (f == 3) {
            if (C->dampingLayerSelector > 0) {
              size_t top = IX(o, i, j, kMax - 1);
              double z = o->zPos[c], zt = o->zPos[top];
              if (z >= zt - C->dampingLayerDepth) {
                double wbs = momentum_bs(o, 3, z, o->rhoBS[c]);
                double s = sin(0.5 * acos(-1.0) * (1.0 - (zt - z) / C->dampingLayerDepth));
                o->F[3][c] -= 0.2 * rho[c] * (s * s) * (w[c] / rho[c] - wbs / o->rhoBS[c]);
              }
            }
            if (C->buoyancySelector > 0) {
              double r = rho[c];
              if (moistOn && o->nmoist == 1) {
                double rm = r + o->moist[0][c] * 1e-3;
                o->F[3][c] -= (r / rm) * C->accel_g * (rm - o->rhoBS[c]);
              } else if (moistOn && o->nmoist == 2) {
                double rm = r + o->moist[0][c] * 1e-3 + o->moist[1][c] * 1e-3;
                o->F[3][c] -= (r / rm) * C->accel_g * (rm - o->rhoBS[c]);
              } else {
                o->F[3][c] -= C->accel_g * (r - o->rhoBS[c]);
              }
            }
          }
        }
        if (o->ntke) o->Ftke[c] += advect(o, o->tke, i, j, k, C->TKEAdvSelector, C->TKEAdvSelector_b_hyb);
        for (f = 0; f < o->nmoist; f++) {
          if (f == 0) o->Fmoist[0][c] += advect(o, o->moist[0], i, j, k, C->moistureAdvSelectorQv, C->moistureAdvSelectorQv_b);
          else o->Fmoist[f][c] += advect_ql(o, o->moist[f], i, j, k, C->moistureAdvSelectorQi);
        }
        if (C->coriolisSelector > 0) {
          double z = o->zPos[c], rb = o->rhoBS[c], r = rho[c];
          double ubs = momentum_bs(o, 1, z, rb), vbs = momentum_bs(o, 2, z, rb), wbs = momentum_bs(o, 3, z, rb);
          double fh = C->corioConstHorz, fv = C->corioConstVert, ls = C->corioLS_fact;
          o->F[1][c] += fh * (v[c] / r - ls * vbs / rb) - fv * (w[c] / r - ls * wbs / rb);
          o->F[2][c] -= fh * (u[c] / r - ls * ubs / rb);
          o->F[3][c] += fv * (u[c] / r - ls * ubs / rb);
        }
      }
  if (turb) {
    double **T = o->tau;
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++)
        for (k = kMin; k < kMax; k++) {
          size_t c = IX(o, i, j, k), ip = c + si, jp = c + sj, kp = c + 1;
          double J1 = o->J31[c], J2 = o->J32[c], J3 = o->J33[c];
          o->F[1][c] -= dXi * (T[0][ip] - T[0][c]) + dYi * (T[1][jp] - T[1][c]) + J1 * dXi * (T[2][ip] - T[2][c]) +
                        J2 * dYi * (T[2][jp] - T[2][c]) + J3 * dZi * (T[2][kp] - T[2][c]);
          o->F[2][c] -= dXi * (T[1][ip] - T[1][c]) + dYi * (T[4][jp] - T[4][c]) + J1 * dXi * (T[3][ip] - T[3][c]) +
                        J2 * dYi * (T[3][jp] - T[3][c]) + J3 * dZi * (T[3][kp] - T[3][c]);
          o->F[3][c] -= dXi * (T[2][ip] - T[2][c]) + dYi * (T[3][jp] - T[3][c]) + J1 * dXi * (T[5][ip] - T[5][c]) +
                        J2 * dYi * (T[5][jp] - T[5][c]) + J3 * dZi * (T[5][kp] - T[5][c]);
          o->F[4][c] -= dXi * (T[6][ip] - T[6][c]) + dYi * (T[7][jp] - T[7][c]) + J1 * dXi * (T[8][ip] - T[8][c]) +
                        J2 * dYi * (T[8][jp] - T[8][c]) + J3 * dZi * (T[8][kp] - T[8][c]);
          if (moistOn && C->moistureSGSturb > 0)
            for (f = 0; f < o->nmoist; f++) {
              double **M = &o->mtau[3 * f];
              o->Fmoist[f][c] -= dXi * (M[0][ip] - M[0][c]) + dYi * (M[1][jp] - M[1][c]) + J1 * dXi * (M[2][ip] - M[2][c]) +
                                 J2 * dYi * (M[2][jp] - M[2][c]) + J3 * dZi * (M[2][kp] - M[2][c]);
            }
        }
  }

  /* 5. SGS TKE budget (cuda_sgstkeDevice.cu:68-92, 155-397) */
  if (physics && o->ntke) {
    double **T = o->tau, *ri = o->rhoInv, *e = o->tke;
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++)
        for (k = kMin; k < kMax; k++) {
          size_t c = IX(o, i, j, k), ip = c + si, im = c - si, jp = c + sj, jm = c - sj, kp = c + 1, km = c - 1;
          double J1 = o->J31[c], J2 = o->J32[c], J3 = o->J33[c];
          double delta = pow((double)o->dX * o->dY * o->dZ * o->D[c], 1.0 / 3.0);
          double ce = 1.9 * C->c_k + (0.93 - 1.9 * C->c_k) * o->ls[c] / delta;
          double ec = e[c] * ri[c];
          double dux, duy, duz, dvx, dvy, dvz, dwx, dwy, dwz, tt;
          /* buoyancy */
          o->Ftke[c] += C->accel_g / (th[c] * ri[c]) * T[8][c];
          /* dissipation */
          o->Ftke[c] += -ce * e[c] * pow(ec, 0.5) / o->ls[c];
          /* shear production */
#define G_(q, x) (q[x] * ri[x])
          dux = 0.5 * (dXi * (G_(u, ip) - G_(u, im)));
          duy = 0.5 * (dYi * (G_(u, jp) - G_(u, jm)));
          duz = 0.5 * (J1 * dXi * (G_(u, ip) - G_(u, im)) + J2 * dYi * (G_(u, jp) - G_(u, jm)) + J3 * dZi * (G_(u, kp) - G_(u, km)));
          dvx = 0.5 * (dXi * (G_(v, ip) - G_(v, im)));
          dvy = 0.5 * (dYi * (G_(v, jp) - G_(v, jm)));
          dvz = 0.5 * (J1 * dXi * (G_(v, ip) - G_(v, im)) + J2 * dYi * (G_(v, jp) - G_(v, jm)) + J3 * dZi * (G_(v, kp) - G_(v, km)));
          dwx = 0.5 * (dXi * (G_(w, ip) - G_(w, im)));
          dwy = 0.5 * (dYi * (G_(w, jp) - G_(w, jm)));
          dwz = 0.5 * (J1 * dXi * (G_(w, ip) - G_(w, im)) + J2 * dYi * (G_(w, jp) - G_(w, jm)) + J3 * dZi * (G_(w, kp) - G_(w, km)));
#undef G_
          o->Ftke[c] += -T[0][c] * dux - T[1][c] * duy - T[2][c] * duz - T[1][c] * dvx - T[4][c] * dvy - T[3][c] * dvz -
                        T[2][c] * dwx - T[3][c] * dwy - T[5][c] * dwz;
          /* turbulent transport */
          {
            double *Km = o->Km, **de = o->dedx;
            double tx = -(dXi * (de[0][ip] * Km[ip] * rho[ip] - de[0][im] * Km[im] * rho[im]));
            double ty = -(dYi * (de[1][jp] * Km[jp] * rho[jp] - de[1][jm] * Km[jm] * rho[jm]));
            double tz = -(J1 * dXi * (de[2][ip] * Km[ip] * rho[ip] - de[2][im] * Km[im] * rho[im]) +
                          J2 * dYi * (de[2][jp] * Km[jp] * rho[jp] - de[2][jm] * Km[jm] * rho[jm]) +
                          J3 * dZi * (de[2][kp] * Km[kp] * rho[kp] - de[2][km] * Km[km] * rho[km]));
            tt = -(tx + ty + tz);
          }
          o->Ftke[c] += tt;
        }
  }

  /* 6. saturation adjustment (cuda_moistureDevice.cu:80-247) every MP call */
  if (physics && moistOn && C->moistureCond > 0 && o->nmoist > 1) {
    int freq = (int)lround(fmax(C->moistureMPcallTscale, C->dt) / C->dt);
    if (freq < 1) freq = 1;
    if (o->simTime_it % freq == 0) {
      static const double a[9] = {6.11239921, 0.443987641, 0.142986287e-1, 0.264847430e-3, 0.302950461e-5,
                                  0.206739458e-7, 0.640689451e-10, -0.952447341e-13, -0.976195544e-15};
      static const double ai[9] = {6.11147274, 0.503160820, 0.188439774e-1, 0.420895665e-3, 0.615021634e-5,
                                   0.602588177e-7, 0.385852041e-9, 0.146898966e-11, 0.252751365e-14};
      double *ri = o->rhoInv;
      for (i = iMin; i < iMax; i++)
        for (j = jMin; j < jMax; j++)
          for (k = kMin; k < kMax; k++) {
            size_t c = IX(o, i, j, k);
            double thd = th[c] * ri[c];
            double prd = C->moistureCondBasePres == 1 ? pow(o->thBS[c] * c1, C->cp_cv) : pow(th[c] * c1, C->cp_cv);
            double Td = thd * pow(prd / C->refPressure, C->R_cp);
            const double *cf = Td >= 273.15 ? a : ai;
            double Tc = fmax(-80.0, Td - 273.16), pvs, ffor = 0, flim, rv, rvs, fc, pr_d2, Td2;
            int m;
            pvs = cf[8];
            for (m = 7; m >= 0; m--) pvs = cf[m] + Tc * pvs;
            pvs = fmin(0.99 * prd, pvs * 100.0);
            flim = o->moist[1][c] * 1e-3;
            if (C->moistureCond == 1) {
              ffor = o->moist[0][c] * 1e-3 - pvs / (C->R_vapor * Td);
            } else if (C->moistureCond == 2) {
              rv = o->moist[0][c] * 1e-3;
              rvs = pvs / (C->R_vapor * Td);
              ffor = (rv - rvs) / (1.0 + (C->L_v * C->L_v * rvs * ri[c] / (C->cp_gas * C->R_vapor * Td * Td)));
            } else {
              rv = o->moist[0][c] * 1e-3;
              rvs = pvs / (prd - pvs) / C->Rv_Rg;
              rvs = rvs / ri[c];
              ffor = (rv - rvs) / (1.0 + (C->L_v * C->L_v * rvs * ri[c] / (C->cp_gas * C->R_vapor * Td * Td)));
            }
            fc = (fmax(ffor, 0.0) - fmax(fmin(flim, -ffor), 0.0)) / C->moistureCondTscale;
            o->fcond[c] = fc;
            o->Fmoist[0][c] -= fc * 1e3;
            o->Fmoist[1][c] += fc * 1e3;
            pr_d2 = pow(th[c] * c1, C->cp_cv);
            Td2 = thd * pow(pr_d2 / C->refPressure, C->R_cp);
            o->F[4][c] += ((thd * C->L_v) / (Td2 * C->cp_gas)) * fc;
          }
    }
  }

  /* 7. large-scale forcing in the last stage (cuda_largeScaleForcingsDevice.cu:155-252); the
   * subsidence terms multiply the rho-weighted w_ls by rho once more, as the reference does */
  if (stage == 2 && lsf_force_step(o)) {
    double *P = o->lsfProf;
    int nz = o->nzh, ns = o->lsfN;
    if (fresh_means && C->lsf_horMnSubTerms == 1) lsf_slab_means(o);
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++)
        for (k = kMin; k < kMax; k++) {
          size_t c = IX(o, i, j, k);
          double z = o->zPos[c], r = rho[c];
          o->F[4][c] += lsf_profile(C->lsf_th_surf, C->lsf_th_lev1, C->lsf_th_lev2, C->lsf_th_zlev1, C->lsf_th_zlev2, z, r, ns);
          if (moistOn)
            o->Fmoist[0][c] += lsf_profile(C->lsf_qv_surf, C->lsf_qv_lev1, C->lsf_qv_lev2, C->lsf_qv_zlev1, C->lsf_qv_zlev2, z, r, ns);
          if (C->lsf_horMnSubTerms == 1) {
            double fw = lsf_profile(C->lsf_w_surf, C->lsf_w_lev1, C->lsf_w_lev2, C->lsf_w_zlev1, C->lsf_w_zlev2, z, r, ns);
            double dz = o->zPos[c + 1] - o->zPos[c - 1];
#define DMEAN(q) (P[(q) * nz + k + 1] / P[k + 1] - P[(q) * nz + k - 1] / P[k - 1])
            o->F[1][c] -= fw * r * DMEAN(1) / dz;
            o->F[2][c] -= fw * r * DMEAN(2) / dz;
            o->F[4][c] -= fw * r * DMEAN(3) / dz;
            if (moistOn) o->Fmoist[0][c] -= fw * r * DMEAN(4) / dz;
#undef DMEAN
          }
        }
  }

  /* 8. explicit filter of rho w, every stage (cuda_hydroCoreDevice.cu:414-416) */
  if (C->filterSelector > 0)
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++)
        for (k = kMin; k < kMax; k++) o->F[3][IX(o, i, j, k)] += filter6(o, w, i, j, k);
  return FE_OK;
}

/* WS2002 RK3 commit (cuda_RKschemes.cu:21-157) with positive-definite TKE/moisture. */
static void commit(ora_domain *o, int stage) {
  int i, j, k, f;
  double dt = o->c.dt;
  double fac = stage == 0 ? dt / 3.0 : (stage == 1 ? 0.5 * dt : dt);
  for (i = o->iMin; i < o->iMax; i++)
    for (j = o->jMin; j < o->jMax; j++)
      for (k = o->kMin; k < o->kMax; k++) {
        size_t c = IX(o, i, j, k);
        for (f = 0; f < 5; f++) {
          if (stage == 0) o->fld0[f][c] = o->fld[f][c];
          o->fld[f][c] = o->fld0[f][c] + fac * o->F[f][c];
        }
        if (o->ntke) {
          if (stage == 0) o->tke0[c] = o->tke[c];
          o->tke[c] = fmax(o->tke0[c] + fac * o->Ftke[c], 1e-10);
        }
        for (f = 0; f < o->nmoist; f++) {
          if (stage == 0) o->moist0[f][c] = o->moist[f][c];
          o->moist[f][c] = fmax(o->moist0[f][c] + fac * o->Fmoist[f][c], 0.0);
        }
      }
}

int ora_rk_stage(ora_domain *o, int stage) {
  int rc = build_frhs(o, stage, 0);
  if (rc != FE_OK) return rc;
  commit(o, stage);
  return FE_OK;
}

int ora_step(ora_domain *o, int nsteps) {
  int s, st;
  for (s = 0; s < nsteps; s++) {
    if (lsf_means_step(o)) lsf_slab_means(o);
    for (st = 0; st < 3; st++) ora_rk_stage(o, st);
    o->simTime = (double)(float)((float)o->simTime + (float)o->c.dt);
    o->simTime_it += 1;
  }
  return FE_OK;
}

int ora_get_state(ora_domain *o, double *hydro, double *sgstke, double *moist, double *pres) {
  int f;
  if (hydro)
    for (f = 0; f < 5; f++) memcpy(hydro + (size_t)f * o->n, o->fld[f], o->n * sizeof(double));
  if (sgstke && o->ntke) memcpy(sgstke, o->tke, o->n * sizeof(double));
  if (moist)
    for (f = 0; f < o->nmoist; f++) memcpy(moist + (size_t)f * o->n, o->moist[f], o->n * sizeof(double));
  if (pres) memcpy(pres, o->pres, o->n * sizeof(double));
  return FE_OK;
}

int ora_get_frhs(ora_domain *o, double *hydroFrhs, double *sgstkeFrhs, double *moistFrhs, double *taus) {
  int f;
  if (hydroFrhs)
    for (f = 0; f < 5; f++) memcpy(hydroFrhs + (size_t)f * o->n, o->F[f], o->n * sizeof(double));
  if (sgstkeFrhs && o->ntke) memcpy(sgstkeFrhs, o->Ftke, o->n * sizeof(double));
  if (moistFrhs)
    for (f = 0; f < o->nmoist; f++) memcpy(moistFrhs + (size_t)f * o->n, o->Fmoist[f], o->n * sizeof(double));
  if (taus)
    for (f = 0; f < 9; f++) memcpy(taus + (size_t)f * o->n, o->tau[f], o->n * sizeof(double));
  return FE_OK;
}

int ora_get_surface(ora_domain *o, double *cd, double *ch, double *fricVel, double *htFlux, double *invOblen,
                    double *tskin, double *qFlux, double *qskin) {
  size_t b = o->n2 * sizeof(double);
  if (cd) memcpy(cd, o->cd, b);
  if (ch) memcpy(ch, o->ch, b);
  if (fricVel) memcpy(fricVel, o->fricVel, b);
  if (htFlux) memcpy(htFlux, o->htFlux, b);
  if (invOblen) memcpy(invOblen, o->invOblen, b);
  if (tskin) memcpy(tskin, o->tskin, b);
  if (qFlux) memcpy(qFlux, o->qFlux, b);
  if (qskin) memcpy(qskin, o->qskin, b);
  return FE_OK;
}
