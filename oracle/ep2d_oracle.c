/*
 * ep2d_oracle.c -- CPU oracle (test infrastructure; never part of the product path).
 *
 * A plain-C, FP64 restatement of the reference's solver, beacon1143/EffPlast2D
 * (no release tag; the mounted sources carry no revision), file EffPlast2D.cu:
 *   kernels      ComputeDisp :3-35, ComputeStress :37-98, ComputeJ2 :100-145,
 *                ComputePlasticity :147-177
 *   host chain   ComputeEffModuli :179-229, ComputeEffParams :311-698,
 *                SetMaterials :708-769, FindMaxAbs :805-822, getDeltaP_* :825-882,
 *                getTauInfty_honest :925-942, analytic solution :989-1292,
 *                effective moduli :1412-1539, constructor :1541-1612
 * and the pa.dat derivation of get_sigma_2D.m:3-32.
 *
 * Arithmetic follows the reference's expressions term by term and in the same order.
 * It is compiled with -ffp-contract=off, so it does not reproduce the fused
 * multiply-adds the CUDA compiler may form in the reference kernels; agreement with
 * the reference's GPU output is therefore to rounding, not bitwise (the tests state
 * their tolerances).  Host-side reductions (averages, boundary sums, hole area) keep
 * the reference's loop order.
 *
 * The kernel pore mask is evaluated once at creation with the kernel's expression;
 * the reference re-evaluates the same expression on the same inputs every iteration,
 * which gives the same mask.  P0 is identically zero (SetInitPressure :770-783 assigns
 * 0.0 inside and outside the pore), so it is not stored.
 *
 * Parallelism: the four kernel passes are OpenMP-parallel over rows (element-wise,
 * so results do not depend on the thread count); every reduction is sequential.
 */
#include "ep2d_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NSTEP_MAX EP2D_MAX_STEPS
#define NT_MAX 64

struct orc_state {
  long nX, nY;
  double pa[EP2D_NPARS];
  int nl;
  long long niter;
  double eiter;
  long check_every;
  /* derived, EffPlast2D.cu:1563-1573, 1609-1611 */
  double dX, dY, dT, K0, G0, E0, nu0, rad, Y, nPores, porosity, lX, lY;
  /* device-role arrays (the *_cuda arrays of the reference) */
  double *K, *G, *P, *tauXX, *tauYY, *tauXY, *tauXYav, *J2, *J2XY, *Ux, *Uy, *Vx, *Vy;
  /* host copies (the *_cpu arrays after their D2H copies) */
  double *hP, *htauXX, *htauYY, *htauXY, *hUx, *hUy;
  uint8_t *node_in, *corner_in;
  /* get_sigma_2D.m's Plast / PlastXY (:64-65, set at :126-138): 1 where the trial J2 has
   * exceeded coh at any iteration since tracking began */
  int track;
  uint8_t *plast, *plast_xy;
  /* step records (EffPlast2D.h:108-117) */
  int nts[NSTEP_MAX];
  ep2d_step_record rec[NSTEP_MAX][NT_MAX];
  double* checks[NSTEP_MAX][NT_MAX];
  int nchecks[NSTEP_MAX][NT_MAX];
  double curEffStrain[3];
  double loadType_[3];
  int have_step0;
  ep2d_moduli an, an_per, num, num_per;
};

static double* zalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

static long fw(const orc_state* s, int f) {
  switch (f) {
    case EP2D_FIELD_TAUXY: case EP2D_FIELD_J2XY: return s->nX - 1;
    case EP2D_FIELD_UX: case EP2D_FIELD_VX: return s->nX + 1;
    default: return s->nX;
  }
}
static long fh(const orc_state* s, int f) {
  switch (f) {
    case EP2D_FIELD_TAUXY: case EP2D_FIELD_J2XY: return s->nY - 1;
    case EP2D_FIELD_UY: case EP2D_FIELD_VY: return s->nY + 1;
    default: return s->nY;
  }
}
static double* fptr(orc_state* s, int f) {
  switch (f) {
    case EP2D_FIELD_P: return s->P;
    case EP2D_FIELD_TAUXX: return s->tauXX;
    case EP2D_FIELD_TAUYY: return s->tauYY;
    case EP2D_FIELD_TAUXY: return s->tauXY;
    case EP2D_FIELD_TAUXYAV: return s->tauXYav;
    case EP2D_FIELD_J2: return s->J2;
    case EP2D_FIELD_J2XY: return s->J2XY;
    case EP2D_FIELD_UX: return s->Ux;
    case EP2D_FIELD_UY: return s->Uy;
    case EP2D_FIELD_VX: return s->Vx;
    case EP2D_FIELD_VY: return s->Vy;
    case EP2D_FIELD_K: return s->K;
    case EP2D_FIELD_G: return s->G;
    default: return NULL;
  }
}

int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* ComputeStress's pore test at node (i, j), EffPlast2D.cu:79-82 */
static int kernel_node_in(const orc_state* s, int i, int j) {
  const long nX = s->nX, nY = s->nY;
  const double dX = s->dX, dY = s->dY, rad = s->rad, N = s->nPores;
  for (int k = 0; k < N; k++) {
    for (int l = 0; l < N; l++) {
      const double a = -0.5 * dX * (nX - 1) + dX * i - 0.5 * dX * (nX - 1) * (1.0 - 1.0 / N) + (dX * (nX - 1) / N) * k;
      const double b = -0.5 * dY * (nY - 1) + dY * j - 0.5 * dY * (nY - 1) * (1.0 - 1.0 / N) + (dY * (nY - 1) / N) * l;
      if (sqrt(a * a + b * b) < rad) return 1;
    }
  }
  return 0;
}
/* ComputeStress's pore test at corner (i, j), EffPlast2D.cu:89-92 */
static int kernel_corner_in(const orc_state* s, int i, int j) {
  const long nX = s->nX, nY = s->nY;
  const double dX = s->dX, dY = s->dY, rad = s->rad, N = s->nPores;
  for (int k = 0; k < N; k++) {
    for (int l = 0; l < N; l++) {
      const double a = -0.5 * dX * (nX - 2) + dX * i - 0.5 * dX * (nX - 1) * (1.0 - 1.0 / N) + (dX * (nX - 1) / N) * k;
      const double b = -0.5 * dY * (nY - 2) + dY * j - 0.5 * dY * (nY - 1) * (1.0 - 1.0 / N) + (dY * (nY - 1) / N) * l;
      if (sqrt(a * a + b * b) < rad) return 1;
    }
  }
  return 0;
}
/* the host-side pore test of SetMaterials / ComputeEffParams (EffPlast2D.cu:719-720,
 * 523-524, 539-540) at physical position (x, y) */
static int host_in_pore(const orc_state* s, double x, double y) {
  const double Lx = s->dX * (s->nX - 1);
  const double Ly = s->dY * (s->nY - 1);
  const double nPores = s->nPores, rad = s->rad;
  for (int k = 0; k < nPores; k++) {
    for (int l = 0; l < nPores; l++) {
      if (sqrt((x - 0.5 * Lx * (1.0 - 1.0 / nPores) + (Lx / nPores) * k) * (x - 0.5 * Lx * (1.0 - 1.0 / nPores) + (Lx / nPores) * k) +
               (y - 0.5 * Ly * (1.0 - 1.0 / nPores) + (Ly / nPores) * l) * (y - 0.5 * Ly * (1.0 - 1.0 / nPores) + (Ly / nPores) * l)) < rad)
        return 1;
    }
  }
  return 0;
}

/* SetMaterials, EffPlast2D.cu:708-728 (the dilated empty_spaces set feeds only the
 * deprecated getdPhi, EffPlast2D.cu:971-986, and is not restated) */
static void set_materials(orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  for (int i = 0; i < nX; i++) {
    for (int j = 0; j < nY; j++) {
      s->K[j * nX + i] = s->K0;
      s->G[j * nX + i] = s->G0;
      const double x = -0.5 * s->dX * (nX - 1) + s->dX * i;
      const double y = -0.5 * s->dY * (nY - 1) + s->dY * j;
      if (host_in_pore(s, x, y)) {
        s->K[j * nX + i] = 0.01 * s->K0;
        s->G[j * nX + i] = 0.01 * s->G0;
      }
    }
  }
}

int orc_create(const ep2d_params* p, orc_state** out) {
  if (!p || !out) return EP2D_ERR_ARG;
  if (p->nx < 4 || p->ny < 4 || p->nl < 1 || p->nl > EP2D_MAX_STEPS || p->check_every < 1) return EP2D_ERR_ARG;
  orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
  if (!s) return EP2D_ERR_NOMEM;
  s->nX = p->nx;
  s->nY = p->ny;
  memcpy(s->pa, p->pa, sizeof(s->pa));
  s->nl = p->nl;
  s->niter = p->niter;
  s->eiter = p->eiter;
  s->check_every = p->check_every;
  s->dX = s->pa[0];
  s->dY = s->pa[1];
  s->dT = s->pa[2];
  s->K0 = s->pa[3];
  s->G0 = s->pa[4];
  s->E0 = 9.0 * s->K0 * s->G0 / (3.0 * s->K0 + s->G0);
  s->nu0 = (1.5 * s->K0 - s->G0) / (3.0 * s->K0 + s->G0);
  s->rad = s->pa[9];
  s->Y = s->pa[8] / sqrt(2.0);
  s->nPores = s->pa[10];
  const long nX = s->nX, nY = s->nY;
  s->lX = (nX - 1) * s->dX;
  s->lY = (nY - 1) * s->dY;
  s->porosity = 3.1415926 * s->rad * s->rad * s->nPores * s->nPores / (s->lX * s->lY);

  const size_t nn = (size_t)nX * nY, nc = (size_t)(nX - 1) * (nY - 1);
  const size_t nux = (size_t)(nX + 1) * nY, nuy = (size_t)nX * (nY + 1);
  s->K = zalloc(nn); s->G = zalloc(nn); s->P = zalloc(nn); s->tauXX = zalloc(nn);
  s->tauYY = zalloc(nn); s->tauXYav = zalloc(nn); s->J2 = zalloc(nn);
  s->tauXY = zalloc(nc); s->J2XY = zalloc(nc);
  s->Ux = zalloc(nux); s->Vx = zalloc(nux); s->Uy = zalloc(nuy); s->Vy = zalloc(nuy);
  s->hP = zalloc(nn); s->htauXX = zalloc(nn); s->htauYY = zalloc(nn); s->htauXY = zalloc(nc);
  s->hUx = zalloc(nux); s->hUy = zalloc(nuy);
  s->node_in = (uint8_t*)calloc(nn, 1);
  s->corner_in = (uint8_t*)calloc(nc, 1);
  s->plast = (uint8_t*)calloc(nn, 1);
  s->plast_xy = (uint8_t*)calloc(nc ? nc : 1, 1);
  s->track = 0;
  set_materials(s);
  for (int j = 0; j < nY; j++)
    for (int i = 0; i < nX; i++) s->node_in[j * nX + i] = (uint8_t)kernel_node_in(s, i, j);
  for (int j = 0; j < nY - 1; j++)
    for (int i = 0; i < nX - 1; i++) s->corner_in[j * (nX - 1) + i] = (uint8_t)kernel_corner_in(s, i, j);
  for (int a = 0; a < NSTEP_MAX; a++) s->nts[a] = 0;
  *out = s;
  return EP2D_OK;
}

int orc_destroy(orc_state* s) {
  if (!s) return EP2D_OK;
  double* arrs[] = {s->K, s->G, s->P, s->tauXX, s->tauYY, s->tauXY, s->tauXYav, s->J2, s->J2XY,
                    s->Ux, s->Uy, s->Vx, s->Vy, s->hP, s->htauXX, s->htauYY, s->htauXY, s->hUx, s->hUy};
  for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++) free(arrs[a]);
  for (int a = 0; a < NSTEP_MAX; a++)
    for (int t = 0; t < NT_MAX; t++) free(s->checks[a][t]);
  free(s->node_in);
  free(s->corner_in);
  free(s->plast);
  free(s->plast_xy);
  free(s);
  return EP2D_OK;
}

int orc_get_masks(orc_state* s, uint8_t* node_mask, uint8_t* corner_mask) {
  if (!s) return EP2D_ERR_ARG;
  if (node_mask) memcpy(node_mask, s->node_in, (size_t)s->nX * s->nY);
  if (corner_mask) memcpy(corner_mask, s->corner_in, (size_t)(s->nX - 1) * (s->nY - 1));
  return EP2D_OK;
}

/* ---- the four kernels -------------------------------------------------------- */

/* ComputeStress, EffPlast2D.cu:37-98 */
static void k_stress(orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  const double dX = s->dX, dY = s->dY;
  const double *Ux = s->Ux, *Uy = s->Uy, *K = s->K, *G = s->G;
  double *P = s->P, *tauXX = s->tauXX, *tauYY = s->tauYY, *tauXY = s->tauXY;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < nY; j++) {
    for (long i = 0; i < nX; i++) {
      const double divU = (Ux[j * (nX + 1) + i + 1] - Ux[j * (nX + 1) + i]) / dX + (Uy[(j + 1) * nX + i] - Uy[j * nX + i]) / dY;
      P[j * nX + i] = 0.0 - K[j * nX + i] * divU;
      tauXX[j * nX + i] = 2.0 * G[j * nX + i] * ((Ux[j * (nX + 1) + i + 1] - Ux[j * (nX + 1) + i]) / dX - divU / 3.0);
      tauYY[j * nX + i] = 2.0 * G[j * nX + i] * ((Uy[(j + 1) * nX + i] - Uy[j * nX + i]) / dY - divU / 3.0);
      if (i < nX - 1 && j < nY - 1) {
        tauXY[j * (nX - 1) + i] = 0.25 * (G[j * nX + i] + G[j * nX + i + 1] + G[(j + 1) * nX + i] + G[(j + 1) * nX + i + 1]) *
            ((Ux[(j + 1) * (nX + 1) + i + 1] - Ux[j * (nX + 1) + i + 1]) / dY + (Uy[(j + 1) * nX + i + 1] - Uy[(j + 1) * nX + i]) / dX);
      }
      if (s->node_in[j * nX + i]) {
        P[j * nX + i] = 0.0;
        tauXX[j * nX + i] = 0.0;
        tauYY[j * nX + i] = 0.0;
      }
      if (i < nX - 1 && j < nY - 1 && s->corner_in[j * (nX - 1) + i]) tauXY[j * (nX - 1) + i] = 0.0;
    }
  }
}

/* ComputeJ2, EffPlast2D.cu:100-145.  The nine edge/corner stencils of :109-135 all
 * average the 2x2 corner block starting at (clamp(i-1,0,nX-3), clamp(j-1,0,nY-3)),
 * summed in the same order; that is how they are written here. */
static void k_j2(orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  const double *tauXX = s->tauXX, *tauYY = s->tauYY, *tauXY = s->tauXY;
  double *tauXYav = s->tauXYav, *J2 = s->J2, *J2XY = s->J2XY;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < nY; j++) {
    for (long i = 0; i < nX; i++) {
      long ci = i - 1, cj = j - 1;
      if (ci < 0) ci = 0;
      if (ci > nX - 3) ci = nX - 3;
      if (cj < 0) cj = 0;
      if (cj > nY - 3) cj = nY - 3;
      tauXYav[j * nX + i] = 0.25 * (tauXY[cj * (nX - 1) + ci] + tauXY[cj * (nX - 1) + ci + 1] + tauXY[(cj + 1) * (nX - 1) + ci] + tauXY[(cj + 1) * (nX - 1) + ci + 1]);
      J2[j * nX + i] = sqrt(tauXX[j * nX + i] * tauXX[j * nX + i] + tauYY[j * nX + i] * tauYY[j * nX + i] + 2.0 * tauXYav[j * nX + i] * tauXYav[j * nX + i]);
      if (i < nX - 1 && j < nY - 1) {
        const double sx = tauXX[j * nX + i] + tauXX[j * nX + i + 1] + tauXX[(j + 1) * nX + i] + tauXX[(j + 1) * nX + i + 1];
        const double sy = tauYY[j * nX + i] + tauYY[j * nX + i + 1] + tauYY[(j + 1) * nX + i] + tauYY[(j + 1) * nX + i + 1];
        J2XY[j * (nX - 1) + i] = sqrt(0.0625 * sx * sx + 0.0625 * sy * sy + 2.0 * tauXY[j * (nX - 1) + i] * tauXY[j * (nX - 1) + i]);
      }
    }
  }
}

/* ComputePlasticity, EffPlast2D.cu:147-177 */
static void k_plast(orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  const double coh = s->pa[8];
  double *tauXX = s->tauXX, *tauYY = s->tauYY, *tauXY = s->tauXY, *tauXYav = s->tauXYav, *J2 = s->J2;
  const double* J2XY = s->J2XY;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < nY; j++) {
    for (long i = 0; i < nX; i++) {
      if (J2[j * nX + i] > coh) {
        if (s->track) s->plast[j * nX + i] = 1; /* Plast(iPlast) = 1.0, get_sigma_2D.m:130 */
        tauXX[j * nX + i] *= coh / J2[j * nX + i];
        tauYY[j * nX + i] *= coh / J2[j * nX + i];
        tauXYav[j * nX + i] *= coh / J2[j * nX + i];
        J2[j * nX + i] = sqrt(tauXX[j * nX + i] * tauXX[j * nX + i] + tauYY[j * nX + i] * tauYY[j * nX + i] + 2.0 * tauXYav[j * nX + i] * tauXYav[j * nX + i]);
      }
      if (i < nX - 1 && j < nY - 1) {
        if (J2XY[j * (nX - 1) + i] > coh) {
          if (s->track) s->plast_xy[j * (nX - 1) + i] = 1; /* PlastXY(iPlastXY) = 1.0, :136 */
          tauXY[j * (nX - 1) + i] *= coh / J2XY[j * (nX - 1) + i];
        }
      }
    }
  }
}

/* ComputeDisp, EffPlast2D.cu:3-35 */
static void k_disp(orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  const double dX = s->pa[0], dY = s->pa[1], dT = s->pa[2], rho = s->pa[5], dampX = s->pa[6], dampY = s->pa[7];
  double *Ux = s->Ux, *Uy = s->Uy, *Vx = s->Vx, *Vy = s->Vy;
  const double *P = s->P, *tauXX = s->tauXX, *tauYY = s->tauYY, *tauXY = s->tauXY;
#pragma omp parallel for schedule(static)
  for (long j = 0; j < nY; j++) {
    for (long i = 0; i < nX; i++) {
      if (i > 0 && i < nX && j > 0 && j < nY - 1) {
        Vx[j * (nX + 1) + i] = Vx[j * (nX + 1) + i] * (1.0 - dT * dampX) + (dT / rho) * ((
            -P[j * nX + i] + P[j * nX + i - 1] + tauXX[j * nX + i] - tauXX[j * nX + i - 1]) / dX + (
            tauXY[j * (nX - 1) + i - 1] - tauXY[(j - 1) * (nX - 1) + i - 1]) / dY);
      }
      if (i > 0 && i < nX - 1 && j > 0 && j < nY) {
        Vy[j * nX + i] = Vy[j * nX + i] * (1.0 - dT * dampY) + (dT / rho) * ((
            -P[j * nX + i] + P[(j - 1) * nX + i] + tauYY[j * nX + i] - tauYY[(j - 1) * nX + i]) / dY + (
            tauXY[(j - 1) * (nX - 1) + i] - tauXY[(j - 1) * (nX - 1) + i - 1]) / dX);
      }
      Ux[j * (nX + 1) + i] = Ux[j * (nX + 1) + i] + Vx[j * (nX + 1) + i] * dT;
      Uy[j * nX + i] = Uy[j * nX + i] + Vy[j * nX + i] * dT;
    }
  }
}

static void one_iteration(orc_state* s) {
  k_stress(s);
  if (s->nl > 1) {
    k_j2(s);
    k_plast(s);
  }
  k_disp(s);
}

int orc_iterate(orc_state* s, int64_t n) {
  if (!s || n < 0) return EP2D_ERR_ARG;
  for (int64_t it = 0; it < n; it++) one_iteration(s);
  return EP2D_OK;
}

int orc_get_field(orc_state* s, int32_t f, double* out) {
  if (!s || !out || f < 0 || f >= EP2D_NFIELDS) return EP2D_ERR_ARG;
  memcpy(out, fptr(s, f), sizeof(double) * (size_t)fw(s, f) * fh(s, f));
  return EP2D_OK;
}
int orc_set_field(orc_state* s, int32_t f, const double* in) {
  if (!s || !in || f < 0 || f >= EP2D_NFIELDS) return EP2D_ERR_ARG;
  memcpy(fptr(s, f), in, sizeof(double) * (size_t)fw(s, f) * fh(s, f));
  return EP2D_OK;
}

/* ---- host chain -------------------------------------------------------------- */

/* FindMaxAbs(const double*, int), EffPlast2D.cu:805-813 */
static double find_max_abs_arr(const double* a, size_t n) {
  double m = 0.0;
  for (size_t i = 0; i < n; i++)
    if (fabs(a[i]) > fabs(m)) m = fabs(a[i]);
  return m;
}
/* FindMaxAbs(const std::vector<double>&), EffPlast2D.cu:814-822: returns the signed
 * element of largest magnitude */
static double find_max_abs_vec(const double* v, int n) {
  double m = 0.0;
  for (int i = 0; i < n; i++)
    if (fabs(v[i]) > fabs(m)) m = v[i];
  return m;
}
static double std_max(double a, double b) { return (a < b) ? b : a; }

/* getDeltaP_honest, EffPlast2D.cu:825-853 (flat index j*nX + nY-1 kept as written) */
static double delta_p_honest(const orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  const double *P = s->hP, *txx = s->htauXX, *tyy = s->htauYY;
  double dPx = 0.0, dPy = 0.0;
  for (long i = 1; i < nX - 1; i++) {
    dPx += txx[0 * nX + i] - P[0 * nX + i];
    dPx += tyy[0 * nX + i] - P[0 * nX + i];
    dPx += txx[(nY - 1) * nX + i] - P[(nY - 1) * nX + i];
    dPx += tyy[(nY - 1) * nX + i] - P[(nY - 1) * nX + i];
  }
  dPx /= (nX - 2);
  for (long j = 1; j < nY - 1; j++) {
    dPy += txx[j * nX + 0] - P[j * nX + 0];
    dPy += tyy[j * nX + 0] - P[j * nX + 0];
    dPy += txx[j * nX + nY - 1] - P[j * nX + nY - 1];
    dPy += tyy[j * nX + nY - 1] - P[j * nX + nY - 1];
  }
  dPy /= (nY - 2);
  return -0.125 * (dPx + dPy);
}

/* getDeltaP_periodic, EffPlast2D.cu:854-882 (integer divisions and the mixed
 * double bound of :872 kept as written) */
static double delta_p_periodic(const orc_state* s) {
  if (s->nPores <= 2) return 0.0;
  const long nX = s->nX, nY = s->nY;
  const double *P = s->hP, *txx = s->htauXX, *tyy = s->htauYY;
  const int nP = (int)s->nPores;
  double dPx = 0.0, dPy = 0.0;
  for (long i = nX / nP; i < nX * (nP - 1) / nP; i++) {
    dPx += txx[nY / nP * nX + i] - P[nY / nP * nX + i];
    dPx += tyy[nY / nP * nX + i] - P[nY / nP * nX + i];
    dPx += txx[nY * (nP - 1) / nP * nX + i] - P[nY * (nP - 1) / nP * nX + i];
    dPx += tyy[nY * (nP - 1) / nP * nX + i] - P[nY * (nP - 1) / nP * nX + i];
  }
  dPx /= nX * (nP - 2) / nP;
  for (long j = nY / nP; j < nY * (nP - 1) / s->nPores; j++) {
    dPy += txx[j * nX + nX / nP] - P[j * nX + nX / nP];
    dPy += tyy[j * nX + nX / nP] - P[j * nX + nX / nP];
    dPy += txx[j * nX + nX * (nP - 2) / nP] - P[j * nX + nX * (nP - 2) / nP];
    dPy += tyy[j * nX + nX * (nP - 2) / nP] - P[j * nX + nX * (nP - 2) / nP];
  }
  dPy /= nY * (nP - 2) / nP;
  return -0.125 * (dPx + dPy);
}

/* getTauInfty_honest, EffPlast2D.cu:925-942 */
static double tau_infty_honest(const orc_state* s) {
  const long nX = s->nX, nY = s->nY;
  const double *txx = s->htauXX, *tyy = s->htauYY;
  double tx = 0.0, ty = 0.0;
  for (long i = 1; i < nX - 1; i++) {
    tx += txx[0 * nX + i] - tyy[0 * nX + i];
    tx += txx[(nY - 1) * nX + i] - tyy[(nY - 1) * nX + i];
  }
  tx /= (nX - 2);
  for (long j = 1; j < nY - 1; j++) {
    ty += txx[j * nX + 0] - tyy[j * nX + 0];
    ty += txx[j * nX + nY - 1] - tyy[j * nX + nY - 1];
  }
  ty /= (nY - 2);
  return -0.125 * (tx + ty);
}

static void add_check(orc_state* s, int step, int it, double e) {
  int n = s->nchecks[step][it];
  double* p = (double*)realloc(s->checks[step][it], sizeof(double) * (size_t)(n + 1));
  if (!p) return;
  p[n] = e;
  s->checks[step][it] = p;
  s->nchecks[step][it] = n + 1;
}

/* ComputeEffParams, EffPlast2D.cu:311-698 (printing omitted) */
int orc_solve_step(orc_state* s, int32_t step, double loadStepValue, const double loadType[3],
                   int32_t nTimeSteps, ep2d_step_record* out) {
  if (!s || !loadType || step < 0 || step >= s->nl || nTimeSteps < 1 || nTimeSteps > NT_MAX) return EP2D_ERR_ARG;
  if (step > 0 && !s->have_step0) return EP2D_ERR_STATE;
  const long nX = s->nX, nY = s->nY;
  const double dX = s->dX, dY = s->dY, dT = s->dT;
  const size_t nux = (size_t)(nX + 1) * nY, nuy = (size_t)nX * (nY + 1);
  const size_t nn = (size_t)nX * nY, nc = (size_t)(nX - 1) * (nY - 1);
  s->nts[step] = nTimeSteps;
  for (int t = 0; t < NT_MAX; t++) {
    free(s->checks[step][t]);
    s->checks[step][t] = NULL;
    s->nchecks[step][t] = 0;
  }

  if (step == 0) {
    s->curEffStrain[0] = s->curEffStrain[1] = s->curEffStrain[2] = 0.0;
    memset(s->hUx, 0, sizeof(double) * nux);
    memset(s->hUy, 0, sizeof(double) * nuy);
    s->have_step0 = 1;
  } else {
    memcpy(s->hUx, s->Ux, sizeof(double) * nux);
    memcpy(s->hUy, s->Uy, sizeof(double) * nuy);
  }

  for (int it = 0; it < nTimeSteps; it++) {
    ep2d_step_record* r = &s->rec[step][it];
    memset(r, 0, sizeof(*r));
    r->step = step;
    r->time_step = it;
    const double dUxdx = loadStepValue * loadType[0] / (double)nTimeSteps;
    const double dUydy = loadStepValue * loadType[1] / (double)nTimeSteps;
    const double dUxdy = loadStepValue * loadType[2] / (double)nTimeSteps;
    const double dUydx = dUxdy;
    s->curEffStrain[0] += dUxdx;
    s->curEffStrain[1] += dUydy;
    s->curEffStrain[2] += dUxdy;
    memcpy(r->macro_strain, s->curEffStrain, sizeof(r->macro_strain));

    if (it > 0) {
      memcpy(s->hUx, s->Ux, sizeof(double) * nux);
      memcpy(s->hUy, s->Uy, sizeof(double) * nuy);
    }
    /* affine preload, EffPlast2D.cu:370-381 */
    for (int i = 0; i < nX + 1; i++)
      for (int j = 0; j < nY; j++)
        s->hUx[j * (nX + 1) + i] += (-0.5 * dX * nX + dX * i) * dUxdx + (-0.5 * dY * (nY - 1) + dY * j) * dUxdy;
    memcpy(s->Ux, s->hUx, sizeof(double) * nux);
    for (int i = 0; i < nX; i++)
      for (int j = 0; j < nY + 1; j++)
        s->hUy[j * nX + i] += (-0.5 * dY * nY + dY * j) * dUydy + (-0.5 * dX * (nX - 1) + dX * i) * dUydx;
    memcpy(s->Uy, s->hUy, sizeof(double) * nuy);

    /* iteration loop, EffPlast2D.cu:386-428 */
    double error = 0.0;
    long long iters = s->niter;
    int converged = 0;
    for (long long iter = 0; iter < s->niter; iter++) {
      one_iteration(s);
      if ((iter + 1) % s->check_every == 0) {
        error = (find_max_abs_arr(s->Vx, nux) / (dX * (nX - 1)) + find_max_abs_arr(s->Vy, nuy) / (dY * (nY - 1))) * dT /
                (std_max(fabs(s->curEffStrain[0]), std_max(s->curEffStrain[1], s->curEffStrain[2])));
        add_check(s, step, it, error);
        r->n_checks++;
        if (error < s->eiter) {
          iters = iter + 1;
          converged = 1;
          break;
        }
      }
    }
    r->iterations = iters;
    r->converged = converged;
    r->error = error;

    /* averaging, EffPlast2D.cu:430-503 */
    memcpy(s->hP, s->P, sizeof(double) * nn);
    memcpy(s->htauXX, s->tauXX, sizeof(double) * nn);
    memcpy(s->htauYY, s->tauYY, sizeof(double) * nn);
    memcpy(s->htauXY, s->tauXY, sizeof(double) * nc);
    memcpy(s->hUx, s->Ux, sizeof(double) * nux);
    memcpy(s->hUy, s->Uy, sizeof(double) * nuy);
    const double *P = s->hP, *txx = s->htauXX, *tyy = s->htauYY, *txy = s->htauXY, *Ux = s->hUx, *Uy = s->hUy;
    const double nu0 = s->nu0;
    const int perOffsetX = (int)(nX / s->nPores);
    const int perOffsetY = (int)(nY / s->nPores);
    double* sg = r->sigma;
    double* sp = r->sigma_per;
    double* ep = r->eps_per;
    for (int i = 1; i < nX - 1; i++) {
      for (int j = 1; j < nY - 1; j++) {
        sg[0] += txx[j * nX + i] - P[j * nX + i];
        sg[1] += tyy[j * nX + i] - P[j * nX + i];
        if (i < nX - 1 && j < nY - 1) sg[2] += txy[j * (nX - 1) + i];
        sg[2] += nu0 * (txx[j * nX + i] + tyy[j * nX + i] - 2.0 * P[j * nX + i]);
        if (i > perOffsetX && i < nX - perOffsetX && j > perOffsetY && j < nY - perOffsetY) {
          sp[0] += txx[j * nX + i] - P[j * nX + i];
          sp[1] += tyy[j * nX + i] - P[j * nX + i];
          sp[2] += 0.25 * (txy[(j - 1) * (nX - 1) + i - 1] + txy[(j - 1) * (nX - 1) + i] + txy[j * (nX - 1) + i - 1] + txy[j * (nX - 1) + i]);
          sp[3] += nu0 * (txx[j * nX + i] + tyy[j * nX + i] - 2.0 * P[j * nX + i]);
          ep[0] += (Ux[j * (nX + 1) + i + 1] - Ux[j * (nX + 1) + i]) / dX;
          ep[1] += (Uy[(j + 1) * nX + i] - Uy[j * nX + i]) / dY;
          ep[2] += 0.125 * (
              (Ux[j * (nX + 1) + i] - Ux[(j - 1) * (nX + 1) + i]) / dY + (Uy[j * nX + i] - Uy[j * nX + i - 1]) / dX +
              (Ux[j * (nX + 1) + i + 1] - Ux[(j - 1) * (nX + 1) + i + 1]) / dY + (Uy[j * nX + i + 1] - Uy[j * nX + i]) / dX +
              (Ux[(j + 1) * (nX + 1) + i] - Ux[j * (nX + 1) + i]) / dY + (Uy[(j + 1) * nX + i] - Uy[(j + 1) * nX + i - 1]) / dX +
              (Ux[(j + 1) * (nX + 1) + i + 1] - Ux[j * (nX + 1) + i + 1]) / dY + (Uy[(j + 1) * nX + i + 1] - Uy[(j + 1) * nX + i]) / dX);
        }
      }
    }
    sg[0] /= nX * nY;
    sg[1] /= nX * nY;
    sg[2] /= (nX - 1) * (nY - 1);
    sg[3] /= nX * nY;
    const long inner = (nX - 2 * perOffsetX) * (nY - 2 * perOffsetY);
    for (int a = 0; a < 4; a++) sp[a] /= inner;
    for (int a = 0; a < 3; a++) ep[a] /= inner;

    r->delta_p = delta_p_honest(s);
    r->delta_p_per = delta_p_periodic(s);
    r->tau_infty = tau_infty_honest(s);

    /* zero host U in the pores, EffPlast2D.cu:514-547 */
    for (int i = 0; i < nX + 1; i++)
      for (int j = 0; j < nY; j++)
        if (host_in_pore(s, -0.5 * dX * nX + dX * i, -0.5 * dY * (nY - 1) + dY * j)) s->hUx[j * (nX + 1) + i] = 0.0;
    for (int i = 0; i < nX; i++)
      for (int j = 0; j < nY + 1; j++)
        if (host_in_pore(s, -0.5 * dX * (nX - 1) + dX * i, -0.5 * dY * nY + dY * j)) s->hUy[j * nX + i] = 0.0;

    /* hole area, EffPlast2D.cu:549-607 */
    const double nPores = s->nPores, rad = s->rad;
    double HoleAreaPi = 0.0, InternalHoleAreaPi = 0.0;
    for (int k = 0; k < nPores; k++) {
      for (int l = 0; l < nPores; l++) {
        const double cxdX = 0.5 * (nX - 1) * (1.0 - 1.0 / nPores) - ((double)(nX - 1) / nPores) * k;
        const double cydY = 0.5 * (nY - 1) * (1.0 - 1.0 / nPores) - ((double)(nY - 1) / nPores) * l;
        const size_t cyIdx = (size_t)(cydY + 0.5 * (nY - 1));
        size_t rxIdx = (size_t)(cxdX - rad / dX + 0.5 * nX);
        double left[5], right[5], bottom[5], top[5];
        for (int q = 0; q < 5; q++) left[q] = s->hUx[cyIdx * (nX + 1) + rxIdx - 1 + q];
        rxIdx = (size_t)(cxdX + rad / dX + 0.5 * nX);
        for (int q = 0; q < 5; q++) right[q] = s->hUx[cyIdx * (nX + 1) + rxIdx - 2 + q];
        const size_t cxIdx = (size_t)(cxdX + 0.5 * (nX - 1));
        size_t ryIdx = (size_t)(cydY - rad / dY + 0.5 * nY);
        for (int q = 0; q < 5; q++) bottom[q] = s->hUy[(ryIdx - 1 + q) * nX + cxIdx];
        ryIdx = (size_t)(cydY + rad / dY + 0.5 * nY);
        for (int q = 0; q < 5; q++) top[q] = s->hUy[(ryIdx - 2 + q) * nX + cxIdx];
        const double dRx = -0.5 * (find_max_abs_vec(left, 5) - find_max_abs_vec(right, 5));
        const double dRy = -0.5 * (find_max_abs_vec(bottom, 5) - find_max_abs_vec(top, 5));
        HoleAreaPi += (rad + dRx) * (rad + dRy);
        if (k > 0 && l > 0 && k < nPores - 1 && l < nPores - 1) InternalHoleAreaPi += (rad + dRx) * (rad + dRy);
      }
    }
    const double Phi0 = 3.1415926 * rad * rad * nPores * nPores / (dX * (nX - 1) * dY * (nY - 1));
    const double Phi = 3.1415926 * HoleAreaPi / (dX * (nX - 1) * dY * (nY - 1));
    const double PhiPer = nPores > 2 ?
        3.1415926 * InternalHoleAreaPi / (dX * (nX - 1) * dY * (nY - 1) * (nPores - 2) * (nPores - 2) / nPores / nPores) : 0.0;
    r->hole_area_pi = HoleAreaPi;
    r->internal_hole_area_pi = InternalHoleAreaPi;
    r->phi0 = Phi0;
    r->phi = Phi;
    r->phi_per = PhiPer;
    r->dphi = 3.1415926 * fabs(HoleAreaPi - rad * rad * nPores * nPores) / (dX * (nX - 1) * dY * (nY - 1));
    r->dphi_per = fabs(PhiPer - Phi0);

    /* analytic moduli, EffPlast2D.cu:643-696 */
    const double G0 = s->G0, K0 = s->K0, Y = s->Y;
    const double phi = 3.1415926 * rad * rad / (dX * (nX - 1) * dY * (nY - 1));
    r->kphi_exact_elast = r->kd_exact_elast = NAN;
    r->kphi_exact_plast = r->kd_exact_plast = r->kphi_exact_plast_per = r->kd_exact_plast_per = NAN;
    r->g_exact_elast = r->g_exact_plast = r->g_exact_plast_per = NAN;
    if (s->nl <= 1) {
      const double KphiExactElast = G0 / Phi0;
      r->kphi_exact_elast = KphiExactElast;
      s->an.kphi = G0 / Phi0;
      r->kd_exact_elast = (1.0 - phi) / (1.0 / K0 + 1.0 / KphiExactElast);
      s->an.kd = G0 / Phi0;
    } else if (step == 0) {
      const double KphiExactPlast = G0 / Phi / exp(fabs(r->delta_p) / Y - 1.0) / (1.0 + r->tau_infty * r->tau_infty / Y / Y);
      r->kphi_exact_plast = KphiExactPlast;
      s->an.kphi = KphiExactPlast;
      r->kd_exact_plast = (1.0 - phi) / (1.0 / K0 + 1.0 / KphiExactPlast);
      s->an.kd = r->kd_exact_plast;
      const double KphiExactPlastPer = G0 / Phi0 / exp(fabs(r->delta_p_per) / Y - 1.0) / (1.0 + r->tau_infty * r->tau_infty / Y / Y);
      r->kphi_exact_plast_per = KphiExactPlastPer;
      s->an_per.kphi = KphiExactPlastPer;
      r->kd_exact_plast_per = (1.0 - phi) / (1.0 / K0 + 1.0 / KphiExactPlastPer);
      s->an_per.kd = r->kd_exact_plast_per;
    }
    if (s->nl == 3 && step == 0) {
      r->g_exact_elast = G0 / (1.0 + Phi0);
      r->g_exact_plast = G0 / (1.0 + Phi * exp(fabs(r->delta_p) / Y - 1.0));
      s->an.g = r->g_exact_plast;
      r->g_exact_plast_per = G0 / (1.0 + Phi0 * exp(fabs(r->delta_p_per) / Y - 1.0));
      s->an_per.g = r->g_exact_plast_per;
    }
    if (out) out[it] = *r;
  }
  return EP2D_OK;
}

int orc_get_record(orc_state* s, int32_t step, int32_t t, ep2d_step_record* out) {
  if (!s || !out || step < 0 || step >= NSTEP_MAX || t < 0 || t >= s->nts[step]) return EP2D_ERR_ARG;
  *out = s->rec[step][t];
  return EP2D_OK;
}

int orc_get_check_errors(orc_state* s, int32_t step, int32_t t, double* errors, int32_t max_n, int32_t* n_out) {
  if (!s || step < 0 || step >= NSTEP_MAX || t < 0 || t >= NT_MAX) return EP2D_ERR_ARG;
  const int n = s->nchecks[step][t];
  if (n_out) *n_out = n;
  for (int a = 0; a < n && a < max_n; a++) errors[a] = s->checks[step][t][a];
  return EP2D_OK;
}

/* ComputeEffDamping, EffPlast2D.cu:230-243: the preload over nTimeSteps, then NL-1
   increments of one time step each along the same load type, of loadValue times the
   difference of sin(i 2 pi' / (NL-1)) between consecutive steps (pi' = 3.1415926 as
   written there).  The printed tensors (:245-297) are the records. */
int orc_compute_eff_damping(orc_state* s, double initLoadValue, const double loadType[3], int32_t nTimeSteps,
                            double loadValue, int64_t* total_iterations) {
  if (!s || !loadType || nTimeSteps < 1) return EP2D_ERR_ARG;
  if (s->nl < 4) return EP2D_ERR_ARG; /* :233-235 */
  memcpy(s->loadType_, loadType, sizeof(s->loadType_));
  s->an.kphi = s->an.kd = s->an.g = 0.0;
  s->an_per = s->num = s->num_per = s->an;
  int rc = orc_solve_step(s, 0, initLoadValue, loadType, nTimeSteps, NULL);
  if (rc) return rc;
  for (int i = 1; i < s->nl; i++) {
    const double v = loadValue * (sin(i * 2.0 * 3.1415926 / (s->nl - 1)) - sin((i - 1) * 2.0 * 3.1415926 / (s->nl - 1)));
    rc = orc_solve_step(s, i, v, loadType, 1, NULL);
    if (rc) return rc;
  }
  if (total_iterations) {
    int64_t tot = 0;
    for (int a = 0; a < s->nl; a++)
      for (int t = 0; t < s->nts[a]; t++) tot += s->rec[a][t].iterations;
    *total_iterations = tot;
  }
  return EP2D_OK;
}

/* ComputeEffModuli, EffPlast2D.cu:179-229, and the calc and get functions, :1412-1539 */
int orc_compute_eff_moduli(orc_state* s, double initLoadValue, const double loadType[3], int32_t nTimeSteps,
                           ep2d_result* out) {
  if (!s || !loadType || nTimeSteps < 1) return EP2D_ERR_ARG;
  if (s->nl > EP2D_MAX_NL) return EP2D_ERR_ARG; /* EffPlast2D.cu:182-184 */
  const double incPercent = 0.005;
  memcpy(s->loadType_, loadType, sizeof(s->loadType_));
  const double sph[3] = {0.5 * (loadType[0] + loadType[1]), 0.5 * (loadType[0] + loadType[1]), 0.0};
  const double dev[3] = {loadType[0] - sph[0], loadType[1] - sph[1], loadType[2]};
  s->an.kphi = s->an.kd = s->an.g = 0.0;
  s->an_per = s->num = s->num_per = s->an;
  int rc = orc_solve_step(s, 0, initLoadValue, loadType, nTimeSteps, NULL);
  if (rc) return rc;
  const int T = nTimeSteps - 1;
  if (s->nl == 1) {
    /* calcBulkModuli_PureElast, :1412-1428 */
    const ep2d_step_record* r0 = &s->rec[0][T];
    s->num.kphi = r0->delta_p / r0->dphi;
    s->num_per.kphi = r0->delta_p_per / r0->dphi_per;
    {
      const double pInc = -0.33333333 * (r0->sigma[0] + r0->sigma[1] + r0->sigma[2]);
      const double epsInc = r0->macro_strain[0] + r0->macro_strain[1];
      s->num.kd = -pInc / epsInc;
    }
    {
      const double pIncPer = -0.33333333 * (r0->sigma_per[0] + r0->sigma_per[1] + r0->sigma_per[2]);
      const double epsIncPer = r0->eps_per[0] + r0->eps_per[1];
      s->num_per.kd = -pIncPer / epsIncPer;
    }
  } else {
    rc = orc_solve_step(s, 1, initLoadValue * incPercent, sph, 1, NULL);
    if (rc) return rc;
    /* calcBulkModuli_ElastPlast, :1429-1445 */
    const ep2d_step_record* r0 = &s->rec[0][T];
    const ep2d_step_record* r1 = &s->rec[1][0];
    s->num.kphi = (r1->delta_p - r0->delta_p) / (r1->dphi - r0->dphi);
    s->num_per.kphi = (r1->delta_p_per - r0->delta_p_per) / (r1->dphi_per - r0->dphi_per);
    {
      const double pInc = -0.33333333 * (r1->sigma[0] + r1->sigma[1] + r1->sigma[2] - r0->sigma[0] - r0->sigma[1] - r0->sigma[2]);
      const double epsInc = r1->macro_strain[0] + r1->macro_strain[1] - r0->macro_strain[0] - r0->macro_strain[1];
      s->num.kd = -pInc / epsInc;
    }
    {
      const double pInc = -0.33333333 * (r1->sigma_per[0] + r1->sigma_per[1] + r1->sigma_per[2] - r0->sigma_per[0] - r0->sigma_per[1] - r0->sigma_per[2]);
      const double epsInc = r1->eps_per[0] + r1->eps_per[1] - r0->eps_per[0] - r0->eps_per[1];
      s->num_per.kd = -pInc / epsInc;
    }
  }
  if (s->nl == 3) {
    rc = orc_solve_step(s, 2, initLoadValue * incPercent, dev, 1, NULL);
    if (rc) return rc;
    /* calcShearModulus / getG / getGper, :1446-1454, :1516-1539 */
    const ep2d_step_record* r1 = &s->rec[1][0];
    const ep2d_step_record* r2 = &s->rec[2][0];
    s->num.g = 0.5 * (r2->sigma[0] - r1->sigma[0] - r2->sigma[1] + r1->sigma[1]) /
               (r2->macro_strain[0] - r1->macro_strain[0] - r2->macro_strain[1] + r1->macro_strain[1]);
    s->num_per.g = 0.5 * (r2->sigma_per[0] - r1->sigma_per[0] - r2->sigma_per[1] + r1->sigma_per[1]) /
                   (r2->eps_per[0] - r1->eps_per[0] - r2->eps_per[1] + r1->eps_per[1]);
  }
  if (out) {
    memset(out, 0, sizeof(*out));
    out->an = s->an;
    out->an_per = s->an_per;
    out->num = s->num;
    out->num_per = s->num_per;
    out->nl = s->nl;
    out->n_time_steps = nTimeSteps;
    int allc = 1;
    int64_t tot = 0;
    for (int a = 0; a < s->nl; a++)
      for (int t = 0; t < s->nts[a]; t++) {
        tot += s->rec[a][t].iterations;
        allc &= s->rec[a][t].converged;
      }
    out->total_iterations = tot;
    out->all_converged = allc;
  }
  return EP2D_OK;
}

/* ---- analytic static solution, EffPlast2D.cu:989-1292 -------------------------- */

typedef struct {
  double Y, rad, G0, K0;
} an_ctx;

/* getAnalytic, EffPlast2D.cu:989-1012 */
static void get_analytic(const an_ctx* c, double x, double y, double xi, double kappa, double c0,
                         double complex* zeta, double complex* w, double complex* dw, double complex* wv,
                         double complex* Phi, double complex* Psi) {
  const double complex z = CMPLX(x, y);
  double signx = x > 0.0 ? 1.0 : -1.0;
  if (fabs(x) < DBL_EPSILON) signx = 1.0;
  *zeta = (z + signx * csqrt(z * z + 4.0 * c0 * c0 * kappa)) / 2.0 / c0;
  *w = c0 * (*zeta - kappa / *zeta);
  *dw = c0 * (1.0 + kappa / (*zeta * *zeta));
  *wv = c0 * (1.0 / *zeta - kappa * *zeta);
  *Phi = -c->Y * xi / 2.0 - c->Y * xi * clog(*w / *zeta / c->rad);
  *Psi = -c->Y * xi / *zeta * *wv / *dw;
}
/* getAnalyticUelast, EffPlast2D.cu:1014-1026 */
static double complex get_u_elast(const an_ctx* c, double x, double y, double tauInfty, double xi, double kappa, double c0) {
  double complex zeta, w, dw, wv, Phi, Psi;
  get_analytic(c, x, y, xi, kappa, c0, &zeta, &w, &dw, &wv, &Phi, &Psi);
  const double complex phi = -c->Y * xi * w * (clog(w / zeta / c->rad) + 0.5) - 2.0 * c0 * tauInfty / zeta;
  const double complex psi = c0 * c->Y * xi * (1.0 / zeta + kappa * zeta);
  const double complex dphi = Phi * dw;
  return ((1.0 + 6.0 * c->G0 / (c->G0 + 3.0 * c->K0)) * phi - w / conj(dw) * conj(dphi) - conj(psi)) / 2.0 / c->G0;
}
/* getAnalyticUrHydro, EffPlast2D.cu:1027-1029 */
static double get_ur_hydro(const an_ctx* c, double r, double deltaP) {
  return -0.5 * c->Y * c->rad * c->rad * exp((deltaP - c->Y) / c->Y) / (c->G0 * r);
}
static double getJ1(double S11, double S22) { return 0.5 * (S11 + S22); }
static double getJ2(double S11, double S22, double S12) { return 0.5 * ((S11 - S22) * (S11 - S22) + 4.0 * S12 * S12); }
/* getAnalyticJelast, EffPlast2D.cu:1036-1051 */
static void get_j_elast(const an_ctx* c, double x, double y, double xi, double kappa, double c0, double* J1, double* J2) {
  double complex zeta, w, dw, wv, Phi, Psi;
  get_analytic(c, x, y, xi, kappa, c0, &zeta, &w, &dw, &wv, &Phi, &Psi);
  const double complex z = CMPLX(x, y);
  const double complex dPhi = -2.0 * xi * c->Y * kappa / zeta / (zeta * zeta - kappa);
  const double complex F = 2.0 * (conj(w) / dw * dPhi + Psi) / cexp(-2.0 * carg(z) * CMPLX(0.0, 1.0));
  const double Srr = 2.0 * creal(Phi) - creal(F) / 2.0;
  const double Sff = 2.0 * creal(Phi) + creal(F) / 2.0;
  const double Srf = cimag(F) / 2.0;
  *J1 = getJ1(Srr, Sff);
  *J2 = getJ2(Srr, Sff, Srf);
}
/* getAnalyticJplast, EffPlast2D.cu:1052-1059 */
static void get_j_plast(const an_ctx* c, double r, double xi, double* J1, double* J2) {
  const double Srr = -2.0 * xi * c->Y * log(r / c->rad);
  const double Sff = -2.0 * xi * c->Y * (1.0 + log(r / c->rad));
  *J1 = getJ1(Srr, Sff);
  *J2 = getJ2(Srr, Sff, 0.0);
}

/* SaveAnStatic2D, EffPlast2D.cu:1060-1292 (the file writes are the caller's) */
int orc_static_fields(orc_state* s, double deltaP, double tauInfty, double* UnuAbs, double* J1nu, double* J2nu,
                      double* UanAbs, double* errorUabs, double* J1an, double* J2an, double* errorJ1, double* errorJ2,
                      double stats[6]) {
  if (!s || !UnuAbs || !J1nu || !J2nu) return EP2D_ERR_ARG;
  const long nX = s->nX, nY = s->nY;
  const double dX = s->dX, dY = s->dY, rad = s->rad, Y = s->Y;
  const an_ctx c = {Y, rad, s->G0, s->K0};
  const int one = (s->nPores == 1);
  if (one && (!UanAbs || !errorUabs || !J1an || !J2an || !errorJ1 || !errorJ2)) return EP2D_ERR_ARG;
  const int isHydroStatic = (fabs(s->loadType_[0] - s->loadType_[1]) < DBL_EPSILON) && fabs(s->loadType_[2]) < DBL_EPSILON;
  const double Rmin = rad;
  const double Rmax = 0.5 * dX * (nX - 1) - dX * 20.0;
  const double eps = 1.0e-18;
  const double xi = (deltaP > 0.0) ? 1.0 : -1.0;
  const double kappa = tauInfty / Y * xi;
  const double c0 = rad * exp(fabs(deltaP) / 2.0 / Y - 0.5);
  const double rx = rad + get_ur_hydro(&c, rad, deltaP);
  const double ry = rx;
  const double Rx = c0 * (1.0 - kappa);
  const double Ry = c0 * (1.0 + kappa);
  double eUmax = 0.0, eUavg = 0.0, eJ1max = 0.0, eJ1avg = 0.0, eJ2max = 0.0, eJ2avg = 0.0;
  size_t eUn = 0, eJn = 0;
  const double *Ux = s->hUx, *Uy = s->hUy, *P = s->hP, *txx = s->htauXX, *tyy = s->htauYY, *txy = s->htauXY;
  for (int i = 0; i < nX; i++) {
    for (int j = 0; j < nY; j++) {
      const double ux = 0.5 * (Ux[(nX + 1) * j + i] + Ux[(nX + 1) * j + (i + 1)]);
      const double uy = 0.5 * (Uy[nX * j + i] + Uy[nX * (j + 1) + i]);
      UnuAbs[j * nX + i] = sqrt(ux * ux + uy * uy);
      if (i < nX - 1 && j < nY - 1) {
        const double Sxx = 0.25 * (-P[j * nX + i] + txx[j * nX + i] + -P[j * nX + (i + 1)] + txx[j * nX + (i + 1)] +
                                   -P[(j + 1) * nX + i] + txx[(j + 1) * nX + i] + -P[(j + 1) * nX + (i + 1)] + txx[(j + 1) * nX + (i + 1)]);
        const double Syy = 0.25 * (-P[j * nX + i] + tyy[j * nX + i] + -P[j * nX + (i + 1)] + tyy[j * nX + (i + 1)] +
                                   -P[(j + 1) * nX + i] + tyy[(j + 1) * nX + i] + -P[(j + 1) * nX + (i + 1)] + tyy[(j + 1) * nX + (i + 1)]);
        const double Sxy = txy[j * (nX - 1) + i];
        J1nu[j * (nX - 1) + i] = getJ1(Sxx, Syy);
        J2nu[j * (nX - 1) + i] = getJ2(Sxx, Syy, Sxy);
      }
      if (one) {
        const double x = -0.5 * dX * (nX - 1) + dX * i;
        const double y = -0.5 * dY * (nY - 1) + dY * j;
        const double r = sqrt(x * x + y * y);
        if (x * x / (Rx * Rx) + y * y / (Ry * Ry) > 1.0) {
          if (isHydroStatic) UanAbs[j * nX + i] = fabs(get_ur_hydro(&c, r, deltaP));
          else UanAbs[j * nX + i] = cabs(get_u_elast(&c, x, y, tauInfty, xi, kappa, c0));
        } else if (x * x / (rx * rx) + y * y / (ry * ry) > 1.0) {
          UanAbs[j * nX + i] = fabs(get_ur_hydro(&c, r, deltaP));
        } else {
          UanAbs[j * nX + i] = 0.0;
        }
        errorUabs[j * nX + i] = 0.0;
        if (x * x + y * y > Rmin * Rmin && x * x + y * y < Rmax * Rmax && fabs(UnuAbs[j * nX + i]) > eps) {
          errorUabs[j * nX + i] = fabs((UanAbs[j * nX + i] - UnuAbs[j * nX + i]) / UanAbs[j * nX + i]);
          eUmax = std_max(eUmax, errorUabs[j * nX + i]);
          eUavg += errorUabs[j * nX + i];
          eUn++;
          if (fabs(errorUabs[j * nX + i]) > 0.5) errorUabs[j * nX + i] = -0.5;
        }
        if (i < nX - 1 && j < nY - 1) {
          const double xs = -0.5 * dX * (nX - 1) + dX * i + 0.5 * dX;
          const double ys = -0.5 * dY * (nY - 1) + dY * j + 0.5 * dY;
          const double rs = sqrt(xs * xs + ys * ys);
          const long q = j * (nX - 1) + i;
          if (xs * xs / (Rx * Rx) + ys * ys / (Ry * Ry) > 1.0) {
            if (isHydroStatic) {
              const double relR = rad / rs;
              const double Srr = -deltaP + relR * relR * Y * exp(deltaP / Y - 1);
              const double Sff = -deltaP - relR * relR * Y * exp(deltaP / Y - 1);
              J1an[q] = getJ1(Srr, Sff);
              J2an[q] = getJ2(Srr, Sff, 0.0);
            } else {
              get_j_elast(&c, xs, ys, xi, kappa, c0, &J1an[q], &J2an[q]);
            }
          } else if (xs * xs / (rx * rx) + ys * ys / (ry * ry) > 1.0) {
            get_j_plast(&c, rs, xi, &J1an[q], &J2an[q]);
          } else {
            J1an[q] = 0.0;
            J2an[q] = 0.0;
          }
          errorJ1[q] = 0.0;
          errorJ2[q] = 0.0;
          if (xs * xs + ys * ys > Rmin * Rmin && xs * xs + ys * ys < Rmax * Rmax) {
            if (fabs(J1nu[q]) > eps) {
              errorJ1[q] = fabs((J1an[q] - J1nu[q]) / J1an[q]);
              eJ1max = std_max(eJ1max, errorJ1[q]);
              eJ1avg += errorJ1[q];
              if (fabs(errorJ1[q]) > 0.5) errorJ1[q] = -0.5;
            }
            if (fabs(J2nu[q]) > eps) {
              errorJ2[q] = fabs((J2an[q] - J2nu[q]) / J2an[q]);
              eJ2max = std_max(eJ2max, errorJ2[q]);
              eJ2avg += errorJ2[q];
              if (fabs(errorJ2[q]) > 0.5) errorJ2[q] = -0.5;
            }
            eJn++;
          }
        }
      }
    }
  }
  if (stats) {
    if (one) {
      stats[0] = eUmax; stats[1] = eUavg / eUn;
      stats[2] = eJ1max; stats[3] = eJ1avg / eJn;
      stats[4] = eJ2max; stats[5] = eJ2avg / eJn;
    } else {
      for (int a = 0; a < 6; a++) stats[a] = NAN;
    }
  }
  return EP2D_OK;
}

/* ---- plastic zone and polar stresses (get_sigma_2D.m) ------------------------ */

int orc_track_plastic_zone(orc_state* s, int32_t on) {
  if (!s) return EP2D_ERR_ARG;
  s->track = on ? 1 : 0;
  if (on) {
    memset(s->plast, 0, (size_t)s->nX * s->nY);
    memset(s->plast_xy, 0, (size_t)(s->nX - 1) * (s->nY - 1));
  }
  return EP2D_OK;
}

/* get_sigma_2D.m:170-194 on the current state, with the zone accumulated since
 * orc_track_plastic_zone(s, 1): Plast(node) + PlastXY of the (up to) four corners around
 * it (:170-173), then, where that count is > 0, the numerical stresses rotated to polar
 * axes about the grid centre (:185-194; sinsin = y/r, coscos = x/r, :74-75) and the
 * analytic ones (:176-179, P0 = 0 as at :7); every map is 0 inside the centred pore
 * radius and where the count is 0.  x, y: the node coordinates -L/2 + d i (:18-21),
 * here -0.5 d (n - 1) + d i.  Outputs nX*nY, row-major with x fastest. */
int orc_polar_fields(orc_state* s, double load_value, double* snrr, double* snff, double* sarr, double* saff,
                     uint8_t* count_out) {
  if (!s || !snrr || !snff || !sarr || !saff || !count_out) return EP2D_ERR_ARG;
  const long nX = s->nX, nY = s->nY;
  const double coh = s->pa[8], rad = s->pa[9];
  const double sgn = (load_value > 0.0) ? 1.0 : (load_value < 0.0 ? -1.0 : 0.0);
  const double P0 = 0.0; /* get_sigma_2D.m:7 */
  for (long j = 0; j < nY; j++) {
    for (long i = 0; i < nX; i++) {
      const long q = j * nX + i;
      int count = s->plast[q];
      for (int dj = -1; dj <= 0; dj++)
        for (int di = -1; di <= 0; di++) {
          const long ci = i + di, cj = j + dj;
          if (ci >= 0 && ci < nX - 1 && cj >= 0 && cj < nY - 1) count += s->plast_xy[cj * (nX - 1) + ci];
        }
      const double x = -0.5 * s->dX * (nX - 1) + s->dX * i;
      const double y = -0.5 * s->dY * (nY - 1) + s->dY * j;
      const double r = sqrt(x * x + y * y);
      const double sn = y / r, cs = x / r;
      double a = 0.0, b = 0.0, ar = 0.0, af = 0.0;
      if (count > 0) {
        const double sxx = s->tauXX[q] - s->P[q], syy = s->tauYY[q] - s->P[q], sxy = s->tauXYav[q];
        a = sxx * cs * cs + 2.0 * sxy * sn * cs + syy * sn * sn;
        b = sxx * sn * sn - 2.0 * sxy * sn * cs + syy * cs * cs;
        ar = -P0 + sgn * 2.0 * coh * log(sqrt(r)) / sqrt(2.0);
        af = -P0 + sgn * 2.0 * coh * (log(sqrt(r)) + 1.0) / sqrt(2.0);
      }
      if (r < rad) a = b = ar = af = 0.0;
      snrr[q] = a;
      snff[q] = b;
      sarr[q] = ar;
      saff[q] = af;
      count_out[q] = (uint8_t)count;
    }
  }
  return EP2D_OK;
}
