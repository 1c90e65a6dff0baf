/*
 * mdbas_oracle.c -- CPU restatement of MDBas's real-space nonbonded hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see mdbas_oracle.h).  Each routine names the
 * MDBas source lines it restates.  Expressions are written with MDBas's
 * association order and the file is compiled with -ffp-contract=off, so the
 * FP64 results match MDBas's own build bit for bit; tests/test_oracle_ref.py
 * checks exactly that against oracle/_ref/libmdbas_ref.so.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "mdbas_oracle.h"
#include "../mdbas_b200/csrc/link_stencil.h"

#define SQRTPI_ (1.772453850905516) /* global.h:62 */
#define TYPE_CUBIC 1
#define TYPE_ORBIC 2
#define TYPE_TCLIN 3

/* nint: round half away from zero, then truncate (src/utils.c:606-609). */
int orc_nint(double x)
{
  return (x >= 0.) ? (int)(x + 0.5) : (int)(x - 0.5);
}

/* init_box (src/init.c:840-908): reciprocal (Wigner-Seitz) vectors scaled by
 * 1/det, widths pa/pb/pc of the enclosing orthorhombic cell, volume. */
void orc_init_box(int type, const double cell[9], double box[ORC_BOX_LEN])
{
  double a1 = cell[0], a2 = cell[1], a3 = cell[2];
  double b1 = cell[3], b2 = cell[4], b3 = cell[5];
  double c1 = cell[6], c2 = cell[7], c3 = cell[8];
  double u1, u2, u3, v1, v2, v3, w1, w2, w3, det, vol;
  (void)type;
  u1 = b2 * c3 - c2 * b3;
  u2 = c1 * b3 - b1 * c3;
  u3 = b1 * c2 - c1 * b2;
  v1 = c2 * a3 - a2 * c3;
  v2 = a1 * c3 - c1 * a3;
  v3 = c1 * a2 - a1 * c2;
  w1 = a2 * b3 - b2 * a3;
  w2 = b1 * a3 - a1 * b3;
  w3 = a1 * b2 - b1 * a2;
  det = a1 * u1 + a2 * u2 + a3 * u3;
  vol = fabs(det);
  box[ORC_PA] = vol / sqrt(u1 * u1 + u2 * u2 + u3 * u3);
  box[ORC_PB] = vol / sqrt(v1 * v1 + v2 * v2 + v3 * v3);
  box[ORC_PC] = vol / sqrt(w1 * w1 + w2 * w2 + w3 * w3);
  if (fabs(det) > 0.) {
    u1 /= det; u2 /= det; u3 /= det;
    v1 /= det; v2 /= det; v3 /= det;
    w1 /= det; w2 /= det; w3 /= det;
  } else {
    u1 = u2 = u3 = v1 = v2 = v3 = w1 = w2 = w3 = 0.0;
  }
  box[ORC_A1] = a1; box[ORC_A2] = a2; box[ORC_A3] = a3;
  box[ORC_B1] = b1; box[ORC_B2] = b2; box[ORC_B3] = b3;
  box[ORC_C1] = c1; box[ORC_C2] = c2; box[ORC_C3] = c3;
  box[ORC_U1] = u1; box[ORC_U2] = u2; box[ORC_U3] = u3;
  box[ORC_V1] = v1; box[ORC_V2] = v2; box[ORC_V3] = v3;
  box[ORC_W1] = w1; box[ORC_W2] = w2; box[ORC_W3] = w3;
  box[ORC_VOL] = vol;
  box[ORC_DET] = det;
}

/* Derived cut-off terms as read_SIMU leaves them (src/io.c:714-723). */
void orc_fill_param(double cutOff, double cutOn, double alpha, double chargeConst,
                    int vdwSwitch, int elecType, orc_param *p)
{
  p->chargeConst = chargeConst;
  p->alpha = alpha;
  p->cutOff = cutOff;
  p->cutOn = cutOn;
  p->rcutOff = 1. / cutOff;
  p->cutOff2 = cutOff * cutOff;
  p->rcutOff2 = 1. / p->cutOff2;
  p->cutOn2 = cutOn * cutOn;
  p->switch2 = 1. / ((p->cutOff2 - p->cutOn2) * (p->cutOff2 - p->cutOn2) *
                     (p->cutOff2 - p->cutOn2));
  p->vdwSwitch = vdwSwitch;
  p->elecType = elecType;
}

/* dist (src/utils.c:38-80): minimum image by nint per box type, returns r^2. */
double orc_dist(int type, const double b[ORC_BOX_LEN], double d[3])
{
  double xt, yt, zt;
  switch (type) {
  case TYPE_CUBIC:
    d[0] -= b[ORC_A1] * orc_nint(d[0] * b[ORC_U1]);
    d[1] -= b[ORC_A1] * orc_nint(d[1] * b[ORC_U1]);
    d[2] -= b[ORC_A1] * orc_nint(d[2] * b[ORC_U1]);
    break;
  case TYPE_ORBIC:
    d[0] -= b[ORC_A1] * orc_nint(d[0] * b[ORC_U1]);
    d[1] -= b[ORC_B2] * orc_nint(d[1] * b[ORC_V2]);
    d[2] -= b[ORC_C3] * orc_nint(d[2] * b[ORC_W3]);
    break;
  case TYPE_TCLIN:
    xt = d[0] * b[ORC_U1] + d[1] * b[ORC_U2] + d[2] * b[ORC_U3];
    yt = d[0] * b[ORC_V1] + d[1] * b[ORC_V2] + d[2] * b[ORC_V3];
    zt = d[0] * b[ORC_W1] + d[1] * b[ORC_W2] + d[2] * b[ORC_W3];
    xt -= orc_nint(xt);
    yt -= orc_nint(yt);
    zt -= orc_nint(zt);
    d[0] = xt * b[ORC_A1] + yt * b[ORC_B1] + zt * b[ORC_C1];
    d[1] = xt * b[ORC_A2] + yt * b[ORC_B2] + zt * b[ORC_C2];
    d[2] = xt * b[ORC_A3] + yt * b[ORC_B3] + zt * b[ORC_C3];
    break;
  default:
    break;
  }
  return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
}

/* image_update (src/utils.c:162-218): wrap positions into the primary cell. */
void orc_image_update(int type, const double b[ORC_BOX_LEN], int n, double *x, double *y,
                      double *z)
{
  int i;
  double xt, yt, zt;
  for (i = 0; i < n; i++) {
    switch (type) {
    case TYPE_CUBIC:
      x[i] = x[i] - b[ORC_A1] * orc_nint(x[i] * b[ORC_U1]);
      y[i] = y[i] - b[ORC_A1] * orc_nint(y[i] * b[ORC_U1]);
      z[i] = z[i] - b[ORC_A1] * orc_nint(z[i] * b[ORC_U1]);
      break;
    case TYPE_ORBIC:
      x[i] = x[i] - b[ORC_A1] * orc_nint(x[i] * b[ORC_U1]);
      y[i] = y[i] - b[ORC_B2] * orc_nint(y[i] * b[ORC_V2]);
      z[i] = z[i] - b[ORC_C3] * orc_nint(z[i] * b[ORC_W3]);
      break;
    case TYPE_TCLIN:
      xt = x[i] * b[ORC_U1] + y[i] * b[ORC_U2] + z[i] * b[ORC_U3];
      yt = x[i] * b[ORC_V1] + y[i] * b[ORC_V2] + z[i] * b[ORC_V3];
      zt = x[i] * b[ORC_W1] + y[i] * b[ORC_W2] + z[i] * b[ORC_W3];
      xt -= orc_nint(xt);
      yt -= orc_nint(yt);
      zt -= orc_nint(zt);
      x[i] = xt * b[ORC_A1] + yt * b[ORC_B1] + zt * b[ORC_C1];
      y[i] = xt * b[ORC_A2] + yt * b[ORC_B2] + zt * b[ORC_C2];
      z[i] = xt * b[ORC_A3] + yt * b[ORC_B3] + zt * b[ORC_C3];
      break;
    default:
      break;
    }
  }
}

static int excluded(int i, int j, const int *frozen, const int *exclStart, const int *exclFlat)
{
  int k;
  if (frozen && (frozen[i] * frozen[j]) != 0) return 1;
  for (k = exclStart[i]; k < exclStart[i + 1]; k++)
    if (exclFlat[k] == j) return 1;
  return 0;
}

/* verlet_list / verlet_list_update (src/list.c:896-1123): all pairs i<j by
 * dist(), kept iff r^2 <= (rc+delr)^2, not a frozen pair, not in exclList[i];
 * neighOrder is the identity.  Returns the number of entries (the list is
 * written only while it fits in capacity). */
long orc_verlet_list(int n, int type, const double box[ORC_BOX_LEN], double cutOff, double delr,
                     const double *x, const double *y, const double *z, const int *frozen,
                     const int *exclStart, const int *exclFlat, int *neighPair,
                     int *neighOrder, int *neighList, long capacity)
{
  long offset = 0;
  int i, j;
  double cutnb2 = cutOff + delr, d[3], r2;
  cutnb2 = cutnb2 * cutnb2;
  for (i = 0; i < n; i++) {
    neighPair[i] = 0;
    neighOrder[i] = i;
  }
  for (i = 0; i < n - 1; i++) {
    for (j = i + 1; j < n; j++) {
      d[0] = x[j] - x[i];
      d[1] = y[j] - y[i];
      d[2] = z[j] - z[i];
      r2 = orc_dist(type, box, d);
      if (r2 <= cutnb2 && !excluded(i, j, frozen, exclStart, exclFlat)) {
        if (offset < capacity) neighList[offset] = j;
        neighPair[i]++;
        offset++;
      }
    }
  }
  return offset;
}

/* Link-cell grid size (src/list.c:1888-1890) and makelist's choice
 * (src/list.c:42-57).  Returns 1 when makelist would take the link-cell
 * path (noLink aside). */
int orc_link_cell_counts(int type, const double box[ORC_BOX_LEN], double cutOff, double delr,
                         int linkRatio, int nlc[3])
{
  double cutnb = cutOff + delr;
  (void)type;
  if (linkRatio < 1) linkRatio = 1;
  if (linkRatio > 5) linkRatio = 5;
  nlc[0] = (int)(box[ORC_PA] * (double)linkRatio / cutnb);
  nlc[1] = (int)(box[ORC_PB] * (double)linkRatio / cutnb);
  nlc[2] = (int)(box[ORC_PC] * (double)linkRatio / cutnb);
  if (nlc[0] < 3 || nlc[1] < 3 || nlc[2] < 3) return 0;
  if (nlc[0] * nlc[1] * nlc[2] <= 27) return 0;
  return 1;
}

/* link_cell_verlet_list_update (src/list.c:2276-2619), which is also the
 * fill pass of link_cell_verlet_list (src/list.c:2130-2261); the caller wraps
 * positions first when restating the first build (src/list.c:1927).
 * Cells are filled as LIFO chains (head/link, src/list.c:1943-1966), so each
 * cell lists its atoms in descending index; neighOrder is that cell-major
 * order; each atom i scans the stencil cells in table order, and its own cell
 * only after i in the chain (src/list.c:2043).  Returns entries, or -1 when
 * the grid has fewer than 2*linkRatio+1 cells per side. */
long orc_link_cell_list(int n, int type, const double box[ORC_BOX_LEN], double cutOff,
                        double delr, int linkRatio, const double *x, const double *y,
                        const double *z, const int *frozen, const int *exclStart,
                        const int *exclFlat, int *neighPair, int *neighOrder, int *neighList,
                        long capacity, int *nCells)
{
  int nlcx, nlcy, nlcz, cellCheck, i, j, k, l, ll, ix, iy, iz, jx, jy, jz, iorder, ncell;
  long offset = 0;
  double cutnb = cutOff + delr, cutnb2, dnlcx, dnlcy, dnlcz;
  double cx, cy, cz, xt, yt, zt, xd, yd, zd, r2;
  double *xu, *yu, *zu;
  int *head, *link;
  (void)type;

  cutnb2 = cutnb * cutnb;
  if (linkRatio < 1) linkRatio = 1;
  if (linkRatio > 5) linkRatio = 5;
  cellCheck = LINK_STENCIL_COUNT[linkRatio - 1];
  nlcx = (int)(box[ORC_PA] * (double)linkRatio / cutnb);
  nlcy = (int)(box[ORC_PB] * (double)linkRatio / cutnb);
  nlcz = (int)(box[ORC_PC] * (double)linkRatio / cutnb);
  if (nlcx < 2 * linkRatio + 1 || nlcy < 2 * linkRatio + 1 || nlcz < 2 * linkRatio + 1)
    return -1;
  dnlcx = (double)nlcx;
  dnlcy = (double)nlcy;
  dnlcz = (double)nlcz;
  ncell = nlcx * nlcy * nlcz;
  if (nCells) *nCells = ncell;

  xu = (double *)malloc((size_t)n * sizeof(double));
  yu = (double *)malloc((size_t)n * sizeof(double));
  zu = (double *)malloc((size_t)n * sizeof(double));
  link = (int *)malloc((size_t)n * sizeof(int));
  head = (int *)malloc((size_t)ncell * sizeof(int));
  for (i = 0; i < ncell; i++) head[i] = -1;
  for (i = 0; i < n; i++) {
    link[i] = -1;
    neighPair[i] = 0;
  }

  for (i = 0; i < n; i++) {
    xu[i] = (x[i] * box[ORC_U1] + y[i] * box[ORC_U2] + z[i] * box[ORC_U3]) + 0.5;
    yu[i] = (x[i] * box[ORC_V1] + y[i] * box[ORC_V2] + z[i] * box[ORC_V3]) + 0.5;
    zu[i] = (x[i] * box[ORC_W1] + y[i] * box[ORC_W2] + z[i] * box[ORC_W3]) + 0.5;
  }
  for (i = 0; i < n; i++) {
    int icell;
    ix = (int)(dnlcx * xu[i]);
    if (ix > nlcx - 1) ix = nlcx - 1;
    iy = (int)(dnlcy * yu[i]);
    if (iy > nlcy - 1) iy = nlcy - 1;
    iz = (int)(dnlcz * zu[i]);
    if (iz > nlcz - 1) iz = nlcz - 1;
    icell = ix + nlcx * (iy + nlcy * iz);
    link[i] = head[icell];
    head[icell] = i;
  }
  iorder = 0;
  for (k = 0; k < ncell; k++)
    for (i = head[k]; i != -1; i = link[i]) neighOrder[iorder++] = i;

  ix = iy = iz = 0;
  for (k = 0; k < ncell; k++) {
    for (i = head[k]; i != -1; i = link[i]) {
      for (l = 0; l < cellCheck; l++) {
        cx = cy = cz = 0.;
        jx = ix + LINK_STENCIL[l][0];
        jy = iy + LINK_STENCIL[l][1];
        jz = iz + LINK_STENCIL[l][2];
        if (jx > nlcx - 1) { jx -= nlcx; cx = 1.; } else if (jx < 0) { jx += nlcx; cx = -1.; }
        if (jy > nlcy - 1) { jy -= nlcy; cy = 1.; } else if (jy < 0) { jy += nlcy; cy = -1.; }
        if (jz > nlcz - 1) { jz -= nlcz; cz = 1.; } else if (jz < 0) { jz += nlcz; cz = -1.; }
        ll = jx + nlcx * (jy + nlcy * jz);
        j = (k == ll) ? link[i] : head[ll];
        for (; j != -1; j = link[j]) {
          xt = xu[j] - xu[i] + cx;
          yt = yu[j] - yu[i] + cy;
          zt = zu[j] - zu[i] + cz;
          xd = xt * box[ORC_A1] + yt * box[ORC_B1] + zt * box[ORC_C1];
          yd = xt * box[ORC_A2] + yt * box[ORC_B2] + zt * box[ORC_C2];
          zd = xt * box[ORC_A3] + yt * box[ORC_B3] + zt * box[ORC_C3];
          r2 = xd * xd + yd * yd + zd * zd;
          if (r2 <= cutnb2 && !excluded(i, j, frozen, exclStart, exclFlat)) {
            if (offset < capacity) neighList[offset] = j;
            neighPair[i]++;
            offset++;
          }
        }
      }
    }
    ix = ix + 1;
    if (ix > nlcx - 1) {
      ix = 0;
      iy = iy + 1;
      if (iy > nlcy - 1) {
        iy = 0;
        iz = iz + 1;
      }
    }
  }
  free(xu); free(yu); free(zu); free(link); free(head);
  return offset;
}

/* ewald_dir (src/ewald.c:356-369). */
static double ewald_dir_(const orc_param *p, double *dE, double qel, double r, double rt)
{
  double e, alphar = p->alpha * r;
  e = qel * erfc(alphar) * rt;
  *dE = 2.0 * qel * p->alpha * exp(-(alphar * alphar)) / SQRTPI_;
  *dE = -(e + *dE) * rt;
  return e;
}

/* ewald_corr (src/ewald.c:371-384). */
static double ewald_corr_(const orc_param *p, double *dE, double qel, double r, double rt)
{
  double e, alphar = p->alpha * r;
  e = -qel * erf(alphar) * rt;
  *dE = 2.0 * qel * p->alpha * exp(-(alphar * alphar)) / SQRTPI_;
  *dE = -(e + *dE) * rt;
  return e;
}

/* vdw_switch (src/vdw.c:144-184) / vdw_none (dvdw = 0). */
static double vdw_(const orc_param *p, double *dvdw, double veps, double vsig, double r2,
                   double rt)
{
  double v6, v12, pvdw, dpvdw, s1, sf, dsf, t;
  if (!p->vdwSwitch) {
    *dvdw = 0.;
    return 0.;
  }
  t = vsig * rt;
  v6 = (t * t * t) * (t * t * t);
  v12 = v6 * v6;
  if (r2 <= p->cutOn2) {
    pvdw = 4. * veps * (v12 - v6);
    *dvdw = 24. * veps * rt * (v6 - 2. * v12);
    return pvdw;
  }
  s1 = p->cutOff2 - r2;
  sf = (s1 * s1) * (p->cutOff2 + 2. * r2 - 3. * p->cutOn2) * p->switch2;
  dsf = 12. * r2 * s1 * (p->cutOn2 - r2) * p->switch2;
  pvdw = 4. * veps * (v12 - v6);
  dpvdw = 24. * veps * (v6 - 2. * v12);
  *dvdw = pvdw * dsf + dpvdw * sf;
  *dvdw *= rt;
  return pvdw * sf;
}

/* ewald_energy with keyEwald=3 (src/energy.c:450-643): the pair loop over the
 * half list (:480-561) and the erf correction over excluded pairs j>i with no
 * cut-off (:567-621).  Forces accumulate (+=) like MDBas. */
void orc_ewald_energy(int n, int type, const double box[ORC_BOX_LEN], const orc_param *p,
                      const double *x, const double *y, const double *z, const double *q,
                      const double *eps, const double *sig, const int *neighList,
                      const int *neighPair, const int *neighOrder, const int *exclStart,
                      const int *exclFlat, double *fx, double *fy, double *fz, double out[8])
{
  int i, j, k, l;
  long offset = 0, npair = 0;
  double eDir = 0., dDir = 0., virDir = 0., eCorr = 0., dCorr = 0., virCorr = 0.;
  double evdw = 0., dvdw = 0., virvdw = 0.;
  double r, r2, rt, fxj, fyj, fzj, fxi, fyi, fzi, qel, d[3];

  for (l = 0; l < n; l++) {
    i = neighOrder[l];
    fxi = fyi = fzi = 0.;
    for (k = 0; k < neighPair[i]; k++) {
      j = neighList[offset++];
      d[0] = x[j] - x[i];
      d[1] = y[j] - y[i];
      d[2] = z[j] - z[i];
      r2 = orc_dist(type, box, d);
      r = sqrt(r2);
      rt = 1. / r;
      if (r2 <= p->cutOff2) {
        npair++;
        qel = p->chargeConst * q[i] * q[j];
        eDir += ewald_dir_(p, &dDir, qel, r, rt);
        evdw += vdw_(p, &dvdw, eps[i] * eps[j], sig[i] + sig[j], r2, rt);
        virDir += dDir * r;
        virvdw += dvdw * r;
        fxj = (dDir + dvdw) * d[0] * rt;
        fyj = (dDir + dvdw) * d[1] * rt;
        fzj = (dDir + dvdw) * d[2] * rt;
        fxi += fxj;
        fyi += fyj;
        fzi += fzj;
        fx[j] += -fxj;
        fy[j] += -fyj;
        fz[j] += -fzj;
      }
    }
    fx[i] += fxi;
    fy[i] += fyi;
    fz[i] += fzi;
  }

  for (i = 0; i < n; i++) {
    fxi = fyi = fzi = 0.;
    for (k = exclStart[i]; k < exclStart[i + 1]; k++) {
      j = exclFlat[k];
      if (j > i) {
        d[0] = x[j] - x[i];
        d[1] = y[j] - y[i];
        d[2] = z[j] - z[i];
        r2 = orc_dist(type, box, d);
        r = sqrt(r2);
        rt = 1. / r;
        qel = p->chargeConst * q[i] * q[j];
        eCorr += ewald_corr_(p, &dCorr, qel, r, rt);
        virCorr += dCorr * r;
        fxj = dCorr * d[0] * rt;
        fyj = dCorr * d[1] * rt;
        fzj = dCorr * d[2] * rt;
        fxi += fxj;
        fyi += fyj;
        fzi += fzj;
        fx[j] += -fxj;
        fy[j] += -fyj;
        fz[j] += -fzj;
      }
    }
    fx[i] += fxi;
    fy[i] += fyi;
    fz[i] += fzi;
  }
  out[0] = eDir;
  out[1] = eCorr;
  out[2] = evdw;
  out[3] = virDir;
  out[4] = virCorr;
  out[5] = virvdw;
  out[6] = (double)npair;
  out[7] = 0.;
}

/* coulomb_shift1 / shift2 / switch / none (src/elec.c:137-263, :25-36). */
static double coulomb_(const orc_param *p, double *delec, double qel, double r2, double rt)
{
  double s1, s2, sf, dsf, pelec;
  switch (p->elecType) {
  case 2: /* SHIFT1 */
    s1 = rt * r2 * p->rcutOff;
    s2 = r2 * p->rcutOff2;
    sf = 1. - 2. * s1 + s2;
    dsf = 2. * (s2 - s1);
    pelec = p->chargeConst * qel * rt;
    *delec = pelec * rt * (dsf - sf);
    return pelec * sf;
  case 3: /* SHIFT2 */
    s1 = r2 * p->rcutOff2;
    s2 = s1 * s1;
    sf = 1. - 2. * s1 + s2;
    dsf = 4. * (s2 - s1);
    pelec = p->chargeConst * qel * rt;
    *delec = pelec * rt * (dsf - sf);
    return pelec * sf;
  case 4: /* SWITCH */
    if (r2 <= p->cutOn2) {
      pelec = p->chargeConst * qel * rt;
      *delec = -pelec * rt;
      return pelec;
    }
    s1 = p->cutOff2 - r2;
    sf = (s1 * s1) * (p->cutOff2 + 2. * r2 - 3. * p->cutOn2) * p->switch2;
    dsf = 12. * r2 * s1 * (p->cutOn2 - r2) * p->switch2;
    pelec = p->chargeConst * qel * rt;
    *delec = pelec * rt * (dsf - sf);
    return pelec * sf;
  default: /* NOELEC, FULL -> coulomb_none (src/energy.c:40-48) */
    *delec = 0.;
    return 0.;
  }
}

/* nonbond_energy (src/energy.c:216-345): same loop as ewald_energy with the
 * cut-off Coulomb kernel and qel = q_i q_j. */
void orc_nonbond_energy(int n, int type, const double box[ORC_BOX_LEN], const orc_param *p,
                        const double *x, const double *y, const double *z, const double *q,
                        const double *eps, const double *sig, const int *neighList,
                        const int *neighPair, const int *neighOrder, double *fx, double *fy,
                        double *fz, double out[5])
{
  int i, j, k, l;
  long offset = 0, npair = 0;
  double elec = 0., evdw = 0., delec = 0., dvdw = 0., virelec = 0., virvdw = 0.;
  double r, r2, rt, fxj, fyj, fzj, fxi, fyi, fzi, d[3];
  for (l = 0; l < n; l++) {
    i = neighOrder[l];
    fxi = fyi = fzi = 0.;
    for (k = 0; k < neighPair[i]; k++) {
      j = neighList[offset++];
      d[0] = x[j] - x[i];
      d[1] = y[j] - y[i];
      d[2] = z[j] - z[i];
      r2 = orc_dist(type, box, d);
      r = sqrt(r2);
      rt = 1. / r;
      if (r2 <= p->cutOff2) {
        npair++;
        elec += coulomb_(p, &delec, q[i] * q[j], r2, rt);
        evdw += vdw_(p, &dvdw, eps[i] * eps[j], sig[i] + sig[j], r2, rt);
        virelec += delec * r;
        virvdw += dvdw * r;
        fxj = (delec + dvdw) * d[0] * rt;
        fyj = (delec + dvdw) * d[1] * rt;
        fzj = (delec + dvdw) * d[2] * rt;
        fxi += fxj;
        fyi += fyj;
        fzi += fzj;
        fx[j] += -fxj;
        fy[j] += -fyj;
        fz[j] += -fzj;
      }
    }
    fx[i] += fxi;
    fy[i] += fyi;
    fz[i] += fzi;
  }
  out[0] = elec;
  out[1] = evdw;
  out[2] = virelec;
  out[3] = virvdw;
  out[4] = (double)npair;
}

/* Ewald self energy inside ewald_rec (src/ewald.c:165-171). */
double orc_self_energy(int n, const double *q, double chargeConst, double alpha)
{
  double e = 0.;
  int i;
  for (i = 0; i < n; i++) e += q[i] * q[i];
  return -chargeConst * alpha * e / SQRTPI_;
}

/* Helper grid for the searches below: cells of width >= rcut on an
 * orthorhombic/cubic box (triclinic falls back to all pairs). */
typedef struct {
  int nc[3], ncell, *head, *next;
} grid_t;

static int grid_build(grid_t *g, int n, int type, const double *b, double rcut, const double *x,
                      const double *y, const double *z)
{
  int i, d;
  double w[3];
  if (type != TYPE_CUBIC && type != TYPE_ORBIC) return 0;
  w[0] = b[ORC_A1]; w[1] = b[ORC_B2]; w[2] = b[ORC_C3];
  for (d = 0; d < 3; d++) {
    g->nc[d] = (int)(w[d] / rcut);
    if (g->nc[d] < 3) return 0;
  }
  g->ncell = g->nc[0] * g->nc[1] * g->nc[2];
  g->head = (int *)malloc((size_t)g->ncell * sizeof(int));
  g->next = (int *)malloc((size_t)n * sizeof(int));
  for (i = 0; i < g->ncell; i++) g->head[i] = -1;
  for (i = 0; i < n; i++) {
    int c[3];
    double s[3];
    s[0] = x[i] / w[0] + 0.5; s[1] = y[i] / w[1] + 0.5; s[2] = z[i] / w[2] + 0.5;
    for (d = 0; d < 3; d++) {
      s[d] -= floor(s[d]);
      c[d] = (int)(s[d] * g->nc[d]);
      if (c[d] >= g->nc[d]) c[d] = g->nc[d] - 1;
      if (c[d] < 0) c[d] = 0;
    }
    {
      int cell = c[0] + g->nc[0] * (c[1] + g->nc[1] * c[2]);
      g->next[i] = g->head[cell];
      g->head[cell] = i;
    }
  }
  return 1;
}

static void grid_free(grid_t *g)
{
  free(g->head);
  free(g->next);
}

static int grid_cell_of(const grid_t *g, const double *b, double x, double y, double z, int c[3])
{
  double s[3] = {x / b[ORC_A1] + 0.5, y / b[ORC_B2] + 0.5, z / b[ORC_C3] + 0.5};
  int d;
  for (d = 0; d < 3; d++) {
    s[d] -= floor(s[d]);
    c[d] = (int)(s[d] * g->nc[d]);
    if (c[d] >= g->nc[d]) c[d] = g->nc[d] - 1;
    if (c[d] < 0) c[d] = 0;
  }
  return c[0] + g->nc[0] * (c[1] + g->nc[1] * c[2]);
}

/* The pair set MDBas's pair loop evaluates on a current list: unordered
 * pairs i<j with dist() r^2 <= r2max, not frozen pairs, not excluded.
 * Pairs are written as (i, j) while they fit; returns the count. */
long orc_pairs_within(int n, int type, const double box[ORC_BOX_LEN], double r2max,
                      const double *x, const double *y, const double *z, const int *frozen,
                      const int *exclStart, const int *exclFlat, int *pairs, long capacity)
{
  long cnt = 0;
  int i, j;
  double d[3], r2;
  grid_t g;
  if (!grid_build(&g, n, type, box, sqrt(r2max), x, y, z)) {
    for (i = 0; i < n - 1; i++)
      for (j = i + 1; j < n; j++) {
        d[0] = x[j] - x[i]; d[1] = y[j] - y[i]; d[2] = z[j] - z[i];
        r2 = orc_dist(type, box, d);
        if (r2 <= r2max && !excluded(i, j, frozen, exclStart, exclFlat)) {
          if (cnt < capacity) { pairs[2 * cnt] = i; pairs[2 * cnt + 1] = j; }
          cnt++;
        }
      }
    return cnt;
  }
  for (i = 0; i < n; i++) {
    int c[3], dx, dy, dz;
    grid_cell_of(&g, box, x[i], y[i], z[i], c);
    for (dz = -1; dz <= 1; dz++)
      for (dy = -1; dy <= 1; dy++)
        for (dx = -1; dx <= 1; dx++) {
          int cx = (c[0] + dx + g.nc[0]) % g.nc[0];
          int cy = (c[1] + dy + g.nc[1]) % g.nc[1];
          int cz = (c[2] + dz + g.nc[2]) % g.nc[2];
          for (j = g.head[cx + g.nc[0] * (cy + g.nc[1] * cz)]; j != -1; j = g.next[j]) {
            if (j <= i) continue;
            d[0] = x[j] - x[i]; d[1] = y[j] - y[i]; d[2] = z[j] - z[i];
            r2 = orc_dist(type, box, d);
            if (r2 <= r2max && !excluded(i, j, frozen, exclStart, exclFlat)) {
              if (cnt < capacity) { pairs[2 * cnt] = i; pairs[2 * cnt + 1] = j; }
              cnt++;
            }
          }
        }
  }
  grid_free(&g);
  return cnt;
}

/* Total real-space force (direct + switched LJ over every non-excluded
 * partner within rc, erf correction over every excluded partner) on each
 * atom of a subset, from the same pair formulas.  Exclusion rows must be
 * symmetric.  Returns 0 when the box is too small for the cell search. */
int orc_forces_subset(int n, int type, const double box[ORC_BOX_LEN], const orc_param *p,
                      const double *x, const double *y, const double *z, const double *q,
                      const double *eps, const double *sig, const int *exclStart,
                      const int *exclFlat, int nsub, const int *subset, double *fx, double *fy,
                      double *fz)
{
  int s, j, k;
  double d[3], r2, r, rt, dE, dvdw, f;
  grid_t g;
  if (!grid_build(&g, n, type, box, p->cutOff, x, y, z)) return 0;
  for (s = 0; s < nsub; s++) {
    int i = subset[s], c[3], dx, dy, dz;
    double sx = 0., sy = 0., sz = 0.;
    grid_cell_of(&g, box, x[i], y[i], z[i], c);
    for (dz = -1; dz <= 1; dz++)
      for (dy = -1; dy <= 1; dy++)
        for (dx = -1; dx <= 1; dx++) {
          int cx = (c[0] + dx + g.nc[0]) % g.nc[0];
          int cy = (c[1] + dy + g.nc[1]) % g.nc[1];
          int cz = (c[2] + dz + g.nc[2]) % g.nc[2];
          for (j = g.head[cx + g.nc[0] * (cy + g.nc[1] * cz)]; j != -1; j = g.next[j]) {
            if (j == i) continue;
            d[0] = x[j] - x[i]; d[1] = y[j] - y[i]; d[2] = z[j] - z[i];
            r2 = orc_dist(type, box, d);
            if (r2 > p->cutOff2) continue;
            {
              int ex = 0;
              for (k = exclStart[i]; k < exclStart[i + 1]; k++)
                if (exclFlat[k] == j) ex = 1;
              if (ex) continue;
            }
            r = sqrt(r2);
            rt = 1. / r;
            ewald_dir_(p, &dE, p->chargeConst * q[i] * q[j], r, rt);
            vdw_(p, &dvdw, eps[i] * eps[j], sig[i] + sig[j], r2, rt);
            f = (dE + dvdw) * rt;
            sx += f * d[0]; sy += f * d[1]; sz += f * d[2];
          }
        }
    for (k = exclStart[i]; k < exclStart[i + 1]; k++) {
      j = exclFlat[k];
      d[0] = x[j] - x[i]; d[1] = y[j] - y[i]; d[2] = z[j] - z[i];
      r2 = orc_dist(type, box, d);
      r = sqrt(r2);
      rt = 1. / r;
      ewald_corr_(p, &dE, p->chargeConst * q[i] * q[j], r, rt);
      f = dE * rt;
      sx += f * d[0]; sy += f * d[1]; sz += f * d[2];
    }
    fx[s] = sx;
    fy[s] = sy;
    fz[s] = sz;
  }
  grid_free(&g);
  return 1;
}
