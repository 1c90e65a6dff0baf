/*
 * ref_harness.c -- flat C entry points around the UNMODIFIED MDBas sources.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled by oracle/Makefile together
 * with MDBas's own src/*.c (read in place, never copied) into
 * oracle/_ref/libmdbas_ref.so.  Only tests/, the smoke check and the CPU
 * baseline leg of bench.py load that library, always as the checker.
 *
 * The harness replaces MDBas's driver (src/mdbas.c:51 main) for the hot path:
 *   - it fills the CTRL/PARAM/PBC/NEIGH/EWALD structs the way read_SIMU
 *     (src/io.c:47-111 defaults, src/io.c:714-723 derived cut-off terms) and
 *     init_system (src/init.c:102-103 CHARMM charge constant, src/init.c:840
 *     init_box) leave them, without reading SIMU/CONF/FORF files;
 *   - it calls the reference's own makelist (src/list.c:29), which selects the
 *     link-cell or O(N^2) builder and the matching exclusion builder;
 *   - it calls the reference's own energy() (src/energy.c:103) with
 *     keyEwald=3, so ewald_energy (src/energy.c:450) skips both k-space
 *     branches (src/energy.c:469-472) and returns exactly the real-space direct
 *     term, the exclusion correction and the switched LJ term.
 * The FP64 Ewald self term lives inside ewald_rec (src/ewald.c:165-171), which
 * keyEwald=3 skips; ref_self_energy restates that one formula.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <stddef.h>

#include "global.h"
#include "energy.h"
#include "list.h"
#include "utils.h"
#include "init.h"
#include "spme.h"
#include "ewald.h"
#include "integrate.h"
#include "shake.h"

/* MDBas's driver owns this global (src/mdbas.c:43). */
FILE *outFile = NULL;

/* src/spme.c needs FFTW3, which is absent here; energy.c references these
 * three symbols but keyEwald=3 never reaches them. */
void init_spme(CTRL *ctrl, PARAM *param, EWALD *ewald, PBC *box)
{ (void)ctrl; (void)param; (void)ewald; (void)box; }
void spme_free(PARAM *param) { (void)param; }
double spme_energy(PARAM *param, EWALD *ewald, PBC *box, const double x[], const double y[],
                   const double z[], double fx[], double fy[], double fz[], const double q[],
                   double stress[6], double *virEwaldRec)
{
  (void)param; (void)ewald; (void)box; (void)x; (void)y; (void)z; (void)fx; (void)fy;
  (void)fz; (void)q; (void)stress; (void)virEwaldRec;
  return 0.0;
}

typedef struct {
  CTRL ctrl;
  PARAM param;
  PBC box;
  NEIGH neigh;
  EWALD ewald;
  ENERGY ener;
  BOND *bond, *ub;
  ANGLE *angle;
  int bondedOn; /* ref_set_bonded: energy() evaluates the bonded terms */
  int kspaceKey; /* ref_set_kspace: energy()'s keyEwald (0: real space only, 3) */
  int nonbondOn; /* ref_set_nonbond: energy() with keyEwald = 0 (nonbond_energy) */
  CONSTRAINT *constList;
  DIHE *dihe, *impr;
  double *x, *y, *z, *q, *eps, *sig, *fx, *fy, *fz, *vx, *vy, *vz;
  int *frozen;
  int *neighList, *neighPair, *neighOrder, *neighList14, **exclList, *exclPair;
  int listBuilt;
  /* dynamics (ref_md_init) */
  double *mass, *rmass;
  int *nAtConst;
  BATH bath;
  int mdInit;
} RefSys;

static double *dup_d(const double *src, int n)
{
  double *p = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  if (src) memcpy(p, src, (size_t)n * sizeof(double));
  return p;
}

/*
 * Create a system.  cell[9] holds the box rows a1 a2 a3 b1 b2 b3 c1 c2 c3
 * (the CONF box lines); boxType follows enum BOX_TYPE (global.h:75-80).
 * eps/sig are the per-atom FORF values after read_FORF's conversion
 * (eps_i = sqrt(eps*418.4), src/io.c:1174; sig_i = FORF sigma, src/io.c:1175).
 * bonds: 2*nBond atom indices; angles: 3*nAngle atom indices.
 */
RefSys *ref_create(int nAtom, int boxType, const double cell[9], double cutOff, double cutOn,
                   double delr, int linkRatio, int noLink, double alpha,
                   const double *x, const double *y, const double *z, const double *q,
                   const double *eps, const double *sig, const int *frozen,
                   int nBond, const int *bonds, int nAngle, const int *angles)
{
  RefSys *s = (RefSys *)calloc(1, sizeof(RefSys));
  int i;
  if (outFile == NULL) outFile = stderr;

  s->ctrl.newjob = 1;
  s->ctrl.mdType = 1;
  s->ctrl.keyEwald = 3;
  s->ctrl.noLink = noLink;
  s->ctrl.elecType = FULL;
  s->ctrl.vdwType = VSWITCH;

  s->param.nAtom = nAtom;
  s->param.nBond = nBond;
  s->param.nAngle = nAngle;
  s->param.cutOff = cutOff;
  s->param.cutOn = cutOn;
  s->param.delr = delr;
  s->param.scal14 = 1.0;
  s->param.chargeConst = chgcharmm * kcaltoiu;          /* src/init.c:102-103 */
  s->param.rcutOff = 1. / s->param.cutOff;               /* src/io.c:714-721 */
  s->param.cutOff2 = X2(s->param.cutOff);
  s->param.rcutOff2 = 1. / s->param.cutOff2;
  s->param.cutOn2 = X2(s->param.cutOn);
  s->param.switch2 = 1. / X3(s->param.cutOff2 - s->param.cutOn2);

  s->box.type = (enum BOX_TYPE)boxType;
  s->box.a1 = cell[0]; s->box.a2 = cell[1]; s->box.a3 = cell[2];
  s->box.b1 = cell[3]; s->box.b2 = cell[4]; s->box.b3 = cell[5];
  s->box.c1 = cell[6]; s->box.c2 = cell[7]; s->box.c3 = cell[8];
  init_box(&s->box);

  s->neigh.update = 1;
  s->neigh.linkRatio = linkRatio;

  s->ewald.alpha = alpha;

  s->x = dup_d(x, nAtom); s->y = dup_d(y, nAtom); s->z = dup_d(z, nAtom);
  s->q = dup_d(q, nAtom); s->eps = dup_d(eps, nAtom); s->sig = dup_d(sig, nAtom);
  s->fx = dup_d(NULL, nAtom); s->fy = dup_d(NULL, nAtom); s->fz = dup_d(NULL, nAtom);
  s->vx = dup_d(NULL, nAtom); s->vy = dup_d(NULL, nAtom); s->vz = dup_d(NULL, nAtom);
  s->frozen = (int *)calloc((size_t)nAtom, sizeof(int));
  if (frozen) memcpy(s->frozen, frozen, (size_t)nAtom * sizeof(int));

  s->bond = (BOND *)calloc((size_t)(nBond > 0 ? nBond : 1), sizeof(BOND));
  for (i = 0; i < nBond; i++) { s->bond[i].a = bonds[2 * i]; s->bond[i].b = bonds[2 * i + 1]; }
  s->angle = (ANGLE *)calloc((size_t)(nAngle > 0 ? nAngle : 1), sizeof(ANGLE));
  for (i = 0; i < nAngle; i++) {
    s->angle[i].a = angles[3 * i]; s->angle[i].b = angles[3 * i + 1]; s->angle[i].c = angles[3 * i + 2];
  }
  s->constList = (CONSTRAINT *)calloc(1, sizeof(CONSTRAINT));
  s->dihe = (DIHE *)calloc(1, sizeof(DIHE));
  s->impr = (DIHE *)calloc(1, sizeof(DIHE));
  return s;
}

/* Dihedrals and impropers (4 atom indices each) for the exclusion builders;
 * call before ref_makelist. */
void ref_set_torsions(RefSys *s, int nDihedral, const int *dihe, int nImproper, const int *impr)
{
  int i;
  free(s->dihe);
  free(s->impr);
  s->dihe = (DIHE *)calloc((size_t)(nDihedral > 0 ? nDihedral : 1), sizeof(DIHE));
  s->impr = (DIHE *)calloc((size_t)(nImproper > 0 ? nImproper : 1), sizeof(DIHE));
  for (i = 0; i < nDihedral; i++) {
    s->dihe[i].a = dihe[4 * i]; s->dihe[i].b = dihe[4 * i + 1];
    s->dihe[i].c = dihe[4 * i + 2]; s->dihe[i].d = dihe[4 * i + 3];
  }
  for (i = 0; i < nImproper; i++) {
    s->impr[i].a = impr[4 * i]; s->impr[i].b = impr[4 * i + 1];
    s->impr[i].c = impr[4 * i + 2]; s->impr[i].d = impr[4 * i + 3];
  }
  s->param.nDihedral = nDihedral;
  s->param.nImproper = nImproper;
}

/*
 * Bonded terms with their parameters (MDBas structs, copied): bonds,
 * angles, Urey-Bradley, dihedrals, impropers.  They replace the topology of
 * ref_create / ref_set_torsions (so they also feed the exclusion builders)
 * and from now on energy() evaluates them (src/energy.c:167-190).
 */
static void *dup_terms(const void *src, int n, size_t size)
{
  void *p = calloc((size_t)(n > 0 ? n : 1), size);
  if (n > 0) memcpy(p, src, (size_t)n * size);
  return p;
}

void ref_set_bonded(RefSys *s, int nBond, const BOND *bond, int nAngle, const ANGLE *angle,
                    int nUb, const BOND *ub, int nDihedral, const DIHE *dihe, int nImproper,
                    const DIHE *impr)
{
  free(s->bond);
  free(s->angle);
  free(s->ub);
  free(s->dihe);
  free(s->impr);
  s->bond = (BOND *)dup_terms(bond, nBond, sizeof(BOND));
  s->angle = (ANGLE *)dup_terms(angle, nAngle, sizeof(ANGLE));
  s->ub = (BOND *)dup_terms(ub, nUb, sizeof(BOND));
  s->dihe = (DIHE *)dup_terms(dihe, nDihedral, sizeof(DIHE));
  s->impr = (DIHE *)dup_terms(impr, nImproper, sizeof(DIHE));
  s->param.nBond = nBond;
  s->param.nAngle = nAngle;
  s->param.nUb = nUb;
  s->param.nDihedral = nDihedral;
  s->param.nImproper = nImproper;
  s->bondedOn = 1;
}

/* Bonded energies of the last energy(): bond, angle, Urey-Bradley,
 * dihedral, improper, bond virial, Urey-Bradley virial. */
void ref_bonded_energies(const RefSys *s, double out[7])
{
  out[0] = s->ener.bond;
  out[1] = s->ener.ang;
  out[2] = s->ener.ub;
  out[3] = s->ener.dihe;
  out[4] = s->ener.impr;
  out[5] = s->ener.virbond;
  out[6] = s->ener.virub;
}

/* energy()'s parameters: the bonded counts only once ref_set_bonded gave
 * the terms' parameters (before that the terms feed the exclusions only). */
static PARAM energy_param(const RefSys *s)
{
  PARAM p = s->param;
  if (!s->bondedOn) {
    p.nBond = 0;
    p.nAngle = 0;
    p.nUb = 0;
    p.nDihedral = 0;
    p.nImproper = 0;
  }
  return p;
}

/*
 * Explicit Ewald k-space in energy() (keyEwald = 1, src/energy.c:469-470)
 * with the harness alpha and the m-range m1..m3: MDBas's init_ewald sets the
 * k count and allocates its tables (kept until ref_destroy).  Energies then
 * include the reciprocal, self and non-neutral terms.  Returns mmax.
 */
int ref_set_kspace(RefSys *s, double prec, int m1, int m2, int m3)
{
  CTRL c = s->ctrl;
  if (s->kspaceKey == 1) return -1;
  c.keyAlpha = 1;
  c.keyMmax = 1;
  s->ewald.prec = prec;
  s->ewald.m1max = m1;
  s->ewald.m2max = m2;
  s->ewald.m3max = m3;
  init_ewald(&c, &s->param, &s->ewald, &s->box);
  s->kspaceKey = 1;
  return s->ewald.mmax;
}

/*
 * 1-4 pairs: with keyNb14 set, energy() adds ewald14_energy (keyEwald != 0)
 * or nonbond14_energy (keyEwald = 0) over the 1-4 list (src/energy.c:
 * 152-164), scaled by scal14.  The exclusion builders make that list from
 * these dihedrals at the next makelist (src/list.c:439-441, :851-853); the
 * dihedral energy terms themselves stay off unless ref_set_bonded is called.
 * Call before the first makelist.
 */
void ref_set_nb14(RefSys *s, double scal14, int nDihedral, const DIHE *dihe)
{
  if (!s->bondedOn) {
    free(s->dihe);
    s->dihe = (DIHE *)dup_terms(dihe, nDihedral, sizeof(DIHE));
    s->param.nDihedral = nDihedral;
  }
  s->param.scal14 = scal14;
  s->ctrl.keyNb14 = 1;
}

/*
 * Cut-off electrostatics instead of Ewald: energy() with keyEwald = 0 calls
 * nonbond_energy (src/energy.c:158-161), whose pair functions come from
 * init_energy_ptrs (src/energy.c:35-92) for these elecType / vdwType values.
 * Returns -1 for values MDBas would stop on (UNKNOWN_ELEC_ERROR and the like).
 */
int ref_set_nonbond(RefSys *s, int elecType, int vdwType)
{
  if (elecType < NOELEC || elecType > SWITCH || vdwType < NOVDW || vdwType > VSWITCH)
    return -1;
  s->ctrl.elecType = elecType;
  s->ctrl.vdwType = vdwType;
  s->nonbondOn = 1;
  return 0;
}

int ref_n_pair14(const RefSys *s) { return s->neigh.nPair14; }

void ref_get_list14(const RefSys *s, int *out)
{
  memcpy(out, s->neighList14, (size_t)(2 * s->neigh.nPair14) * sizeof(int));
}

/* sizeof and field offsets of MDBas's structs, for the ABI layout check:
 * "NAME size off0 off1 ...;" for each struct, written into buf. */
#define OFF(T, f) (int)offsetof(T, f)
int ref_layout(char *buf, int len)
{
  int n = 0;
  n += snprintf(buf + n, len - n, "PBC %d %d %d %d %d %d %d;", (int)sizeof(PBC), OFF(PBC, type),
                OFF(PBC, a1), OFF(PBC, u1), OFF(PBC, pa), OFF(PBC, vol0), OFF(PBC, stress9));
  n += snprintf(buf + n, len - n, "CTRL %d %d %d %d %d %d;", (int)sizeof(CTRL), OFF(CTRL, newjob),
                OFF(CTRL, keyLink), OFF(CTRL, keyEwald), OFF(CTRL, elecType), OFF(CTRL, ens));
  n += snprintf(buf + n, len - n, "PARAM %d %d %d %d %d %d %d %d;", (int)sizeof(PARAM),
                OFF(PARAM, timeStep), OFF(PARAM, nAtom), OFF(PARAM, tolShake),
                OFF(PARAM, chargeConst), OFF(PARAM, cutOff2), OFF(PARAM, switch2),
                OFF(PARAM, maxminst));
  n += snprintf(buf + n, len - n, "BOND %d %d %d %d;", (int)sizeof(BOND), OFF(BOND, a),
                OFF(BOND, k), OFF(BOND, beta));
  n += snprintf(buf + n, len - n, "ANGLE %d %d %d %d;", (int)sizeof(ANGLE), OFF(ANGLE, a),
                OFF(ANGLE, c), OFF(ANGLE, theta0));
  n += snprintf(buf + n, len - n, "DIHE %d %d %d %d;", (int)sizeof(DIHE), OFF(DIHE, order),
                OFF(DIHE, d), OFF(DIHE, mult));
  n += snprintf(buf + n, len - n, "NEIGH %d %d %d;", (int)sizeof(NEIGH), OFF(NEIGH, linkRatio),
                OFF(NEIGH, nPair14));
  n += snprintf(buf + n, len - n, "ENERGY %d %d %d %d;", (int)sizeof(ENERGY), OFF(ENERGY, elec),
                OFF(ENERGY, virelec), OFF(ENERGY, virtot));
  n += snprintf(buf + n, len - n, "CONSTRAINT %d %d;", (int)sizeof(CONSTRAINT),
                OFF(CONSTRAINT, rc2));
  n += snprintf(buf + n, len - n, "EWALD %d %d %d;", (int)sizeof(EWALD), OFF(EWALD, m3max),
                OFF(EWALD, alpha));
  return n;
}

/* Box quantities after init_box, in PBC field order a..vol (for host checks). */
void ref_box(const RefSys *s, double out[30])
{
  const PBC *b = &s->box;
  double v[30] = {b->a, b->a1, b->a2, b->a3, b->b, b->b1, b->b2, b->b3, b->c, b->c1, b->c2, b->c3,
                  b->u, b->u1, b->u2, b->u3, b->v, b->v1, b->v2, b->v3, b->w, b->w1, b->w2, b->w3,
                  b->pa, b->pb, b->pc, b->det, b->vol, b->vol0};
  memcpy(out, v, sizeof(v));
}

/* First list build through makelist(newjob=1) (src/list.c:36-85). */
int ref_makelist(RefSys *s)
{
  s->ctrl.newjob = 1;
  makelist(&s->ctrl, &s->param, &s->box, &s->neigh, s->constList, s->bond, s->angle, s->dihe,
           s->impr, s->x, s->y, s->z, s->frozen, &s->neighList, &s->neighPair, &s->neighOrder,
           &s->neighList14, &s->exclList, &s->exclPair);
  s->listBuilt = 1;
  return s->ctrl.keyLink;
}

/* Rebuild with new coordinates through makelist(newjob=0) (src/list.c:87-105). */
void ref_update_list(RefSys *s, const double *x, const double *y, const double *z)
{
  if (x) memcpy(s->x, x, (size_t)s->param.nAtom * sizeof(double));
  if (y) memcpy(s->y, y, (size_t)s->param.nAtom * sizeof(double));
  if (z) memcpy(s->z, z, (size_t)s->param.nAtom * sizeof(double));
  s->param.step = 0; /* step % update == 0 */
  makelist(&s->ctrl, &s->param, &s->box, &s->neigh, s->constList, s->bond, s->angle, s->dihe,
           s->impr, s->x, s->y, s->z, s->frozen, &s->neighList, &s->neighPair, &s->neighOrder,
           &s->neighList14, &s->exclList, &s->exclPair);
}

int ref_key_link(const RefSys *s) { return s->ctrl.keyLink; }
int ref_n_cells(const RefSys *s) { return s->neigh.nCells; }
int ref_size_list(const RefSys *s) { return s->neigh.sizeList; }

/* Number of list entries actually filled (sum of neighPair). */
long ref_list_entries(const RefSys *s)
{
  long t = 0;
  int i;
  for (i = 0; i < s->param.nAtom; i++) t += s->neighPair[i];
  return t;
}

void ref_get_list(const RefSys *s, int *neighList, int *neighPair, int *neighOrder)
{
  long t = ref_list_entries(s);
  memcpy(neighList, s->neighList, (size_t)t * sizeof(int));
  memcpy(neighPair, s->neighPair, (size_t)s->param.nAtom * sizeof(int));
  memcpy(neighOrder, s->neighOrder, (size_t)s->param.nAtom * sizeof(int));
}

/* The reference's own list arrays (not copies), for callers that hand them
 * to another routine the way MDBas's driver does. */
void ref_list_ptrs(const RefSys *s, int **neighList, int **neighPair, int **neighOrder)
{
  *neighList = s->neighList;
  *neighPair = s->neighPair;
  *neighOrder = s->neighOrder;
}

/* Exclusions as built by the reference: count per atom and flattened rows. */
long ref_excl_entries(const RefSys *s)
{
  long t = 0;
  int i;
  for (i = 0; i < s->param.nAtom; i++) t += s->exclPair[i];
  return t;
}

void ref_get_excl(const RefSys *s, int *exclPair, int *exclFlat)
{
  long o = 0;
  int i, k;
  memcpy(exclPair, s->exclPair, (size_t)s->param.nAtom * sizeof(int));
  for (i = 0; i < s->param.nAtom; i++)
    for (k = 0; k < s->exclPair[i]; k++) exclFlat[o++] = s->exclList[i][k];
}

/* Positions as the reference holds them (the link-cell build wraps them). */
void ref_get_positions(const RefSys *s, double *x, double *y, double *z)
{
  memcpy(x, s->x, (size_t)s->param.nAtom * sizeof(double));
  memcpy(y, s->y, (size_t)s->param.nAtom * sizeof(double));
  memcpy(z, s->z, (size_t)s->param.nAtom * sizeof(double));
}

void ref_set_positions(RefSys *s, const double *x, const double *y, const double *z)
{
  memcpy(s->x, x, (size_t)s->param.nAtom * sizeof(double));
  memcpy(s->y, y, (size_t)s->param.nAtom * sizeof(double));
  memcpy(s->z, z, (size_t)s->param.nAtom * sizeof(double));
}

/*
 * One energy() call (src/energy.c:103) on the current list.  Bonded terms
 * count only after ref_set_bonded (else energy() sees nBond = nAngle = 0).
 * out[0..5] = elec, vdw, virelec, virvdw, pot, virpot (internal units).
 */
void ref_energy(RefSys *s, double *fx, double *fy, double *fz, double out[6])
{
  PARAM p = energy_param(s);
  s->ctrl.keyEwald = s->nonbondOn ? 0 : (s->kspaceKey ? s->kspaceKey : 3);
  init_energy_ptrs(&s->ctrl);
  energy(&s->ctrl, &p, &s->ener, &s->ewald, &s->box, &s->neigh, s->bond, s->ub, s->angle,
         s->dihe, s->impr, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->q,
         s->eps, s->sig, s->eps, s->sig, s->frozen, s->neighList, s->neighPair, s->neighOrder,
         s->neighList14, s->exclList, s->exclPair);
  if (fx) memcpy(fx, s->fx, (size_t)s->param.nAtom * sizeof(double));
  if (fy) memcpy(fy, s->fy, (size_t)s->param.nAtom * sizeof(double));
  if (fz) memcpy(fz, s->fz, (size_t)s->param.nAtom * sizeof(double));
  out[0] = s->ener.elec;
  out[1] = s->ener.vdw;
  out[2] = s->ener.virelec;
  out[3] = s->ener.virvdw;
  out[4] = s->ener.pot;
  out[5] = s->ener.virpot;
}

/* Ewald self energy, the formula of src/ewald.c:165-171 restated. */
double ref_self_energy(const RefSys *s)
{
  double e = 0.;
  int i;
  for (i = 0; i < s->param.nAtom; i++) e += X2(s->q[i]);
  return -s->param.chargeConst * s->ewald.alpha * e / SQRTPI;
}

/* Wall-clock seconds from CLOCK_MONOTONIC, for the CPU baseline. */
double ref_now(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

void ref_destroy(RefSys *s)
{
  int i;
  if (!s) return;
  if (s->kspaceKey == 1) ewald_free(&s->ewald);
  free(s->x); free(s->y); free(s->z); free(s->q); free(s->eps); free(s->sig);
  free(s->fx); free(s->fy); free(s->fz); free(s->vx); free(s->vy); free(s->vz);
  free(s->frozen); free(s->bond); free(s->ub); free(s->angle); free(s->constList); free(s->dihe);
  free(s->impr);
  free(s->mass); free(s->rmass); free(s->nAtConst);
  if (s->mdInit) {
    integrators_free_arrays(&s->ctrl, &s->param);
    if (s->param.nConst > 0) shake_free_arrays();
  }
  if (s->listBuilt) {
    free(s->neighList); free(s->neighPair); free(s->neighOrder); free(s->neighList14);
    if (s->exclList) {
      int rows = s->ctrl.keyLink ? s->param.nAtom : s->param.nAtom - 1;
      for (i = 0; i < rows; i++) free(s->exclList[i]);
      free(s->exclList);
    }
    free(s->exclPair);
  }
  free(s);
}

/*
 * Velocity-Verlet dynamics through MDBas's own integrator, as the MD loop of
 * src/mdbas.c:244-300 drives it: vv_integrate stage 1 (src/integrate.c:1479,
 * vv_nve/vv_nvt_b with vv_shake_r), makelist on the neigh.update cadence,
 * energy(), vv_integrate stage 2 (vv_shake_v, kinetic, image_update).
 * Bonded terms count as in ref_energy (only after ref_set_bonded).
 * constAtoms holds 2*nConst atom indices, constLen2 the squared lengths.
 * tauT > 0 selects NVT_B (Berendsen) toward temp0, else NVE.
 * Requires ref_makelist first.  MDBas keeps its integrator and SHAKE work
 * arrays in file-scope statics, so one RefSys at a time may run dynamics.
 */
int ref_md_init(RefSys *s, const double *mass, const double *vx, const double *vy,
                const double *vz, double timeStep, int listUpdate, int nConst,
                const int *constAtoms, const double *constLen2, double tolShake, int maxCycle,
                double temp0, double tauT)
{
  int i, n = s->param.nAtom;
  if (!s->listBuilt || s->mdInit) return -1;
  s->mass = dup_d(mass, n);
  s->rmass = dup_d(NULL, n);
  for (i = 0; i < n; i++) s->rmass[i] = 1.0 / mass[i];
  if (vx) memcpy(s->vx, vx, (size_t)n * sizeof(double));
  if (vy) memcpy(s->vy, vy, (size_t)n * sizeof(double));
  if (vz) memcpy(s->vz, vz, (size_t)n * sizeof(double));
  free(s->constList);
  s->constList = (CONSTRAINT *)calloc((size_t)(nConst > 0 ? nConst : 1), sizeof(CONSTRAINT));
  s->nAtConst = (int *)calloc((size_t)n, sizeof(int));
  for (i = 0; i < nConst; i++) {
    s->constList[i].a = constAtoms[2 * i];
    s->constList[i].b = constAtoms[2 * i + 1];
    s->constList[i].rc2 = constLen2[i];
    s->nAtConst[constAtoms[2 * i]]++;
    s->nAtConst[constAtoms[2 * i + 1]]++;
  }
  s->param.nConst = nConst;
  s->param.tolShake = tolShake;
  s->param.maxCycle = maxCycle;
  s->param.timeStep = timeStep;
  s->param.rTimeStep = 1. / timeStep;
  s->param.step = 0;
  s->param.nFrozen = 0;
  for (i = 0; i < n; i++) s->param.nFrozen += s->frozen[i] != 0;
  get_degfree(&s->param, &s->box);
  s->param.temp0 = temp0;
  s->param.kinTemp0 = 0.5 * temp0 * (double)s->param.nDegFree * rboltzui;
  s->bath.tauT = tauT;
  s->ctrl.integrator = VELOCITY;
  s->ctrl.ens = tauT > 0. ? NVT_B : NVE;
  s->neigh.update = listUpdate > 0 ? listUpdate : 1;
  integrators_allocate_arrays(&s->ctrl, &s->param);
  if (nConst > 0) shake_allocate_arrays(&s->param);
  s->mdInit = 1;
  /* forces and energies at time 0 (src/mdbas.c:166-176) */
  {
    double out[6];
    ref_energy(s, NULL, NULL, NULL, out);
  }
  s->ener.kin = kinetic(&s->param, s->vx, s->vy, s->vz, s->mass);
  return s->param.nDegFree;
}

/* nSteps MD steps; rows[4*k] = {step, pot, kin, pot+kin} after each step
 * (pot = energy()'s real-space elec + vdw, internal units). */
void ref_md_run(RefSys *s, int nSteps, double *rows)
{
  int k;
  PARAM p;
  for (k = 0; k < nSteps; k++) {
    s->param.step++;
    vv_integrate(&s->ctrl, &s->param, &s->ener, &s->box, &s->bath, s->constList, s->x, s->y,
                 s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->mass, s->rmass,
                 s->nAtConst, 1);
    makelist(&s->ctrl, &s->param, &s->box, &s->neigh, s->constList, s->bond, s->angle, s->dihe,
             s->impr, s->x, s->y, s->z, s->frozen, &s->neighList, &s->neighPair,
             &s->neighOrder, &s->neighList14, &s->exclList, &s->exclPair);
    p = energy_param(s);
    energy(&s->ctrl, &p, &s->ener, &s->ewald, &s->box, &s->neigh, s->bond, s->ub, s->angle,
           s->dihe, s->impr, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->q,
           s->eps, s->sig, s->eps, s->sig, s->frozen, s->neighList, s->neighPair, s->neighOrder,
           s->neighList14, s->exclList, s->exclPair);
    vv_integrate(&s->ctrl, &s->param, &s->ener, &s->box, &s->bath, s->constList, s->x, s->y,
                 s->z, s->vx, s->vy, s->vz, s->fx, s->fy, s->fz, s->mass, s->rmass,
                 s->nAtConst, 2);
    if (rows) {
      rows[4 * k + 0] = (double)s->param.step;
      rows[4 * k + 1] = s->ener.pot;
      rows[4 * k + 2] = s->ener.kin;
      rows[4 * k + 3] = s->ener.pot + s->ener.kin;
    }
  }
}

void ref_get_velocities(const RefSys *s, double *vx, double *vy, double *vz)
{
  memcpy(vx, s->vx, (size_t)s->param.nAtom * sizeof(double));
  memcpy(vy, s->vy, (size_t)s->param.nAtom * sizeof(double));
  memcpy(vz, s->vz, (size_t)s->param.nAtom * sizeof(double));
}

/*
 * MDBas's explicit Ewald reciprocal sum: init_ewald (src/ewald.c:7-72) with
 * the harness's alpha (keyAlpha) and, when mmax[0] > 0, the given k ranges
 * (keyMmax), then ewald_rec (src/ewald.c:131-354) on zeroed force arrays
 * (it rescales them), then ewald_free.  out[0] = energy (reciprocal + self +
 * non-neutral terms), out[1] = virial, out[2..4] = m1max, m2max, m3max,
 * out[5] = number of k vectors.
 */
void ref_ewald_rec(RefSys *s, double prec, const int mmax[3], double *fx, double *fy,
                   double *fz, double out[6])
{
  double stress[6], vir = 0.;
  int n = s->param.nAtom;
  CTRL c = s->ctrl;
  EWALD ew = s->ewald;
  c.keyAlpha = 1;
  c.keyMmax = mmax && mmax[0] > 0;
  ew.prec = prec;
  if (c.keyMmax) {
    ew.m1max = mmax[0];
    ew.m2max = mmax[1];
    ew.m3max = mmax[2];
  }
  init_ewald(&c, &s->param, &ew, &s->box);
  memset(fx, 0, (size_t)n * sizeof(double));
  memset(fy, 0, (size_t)n * sizeof(double));
  memset(fz, 0, (size_t)n * sizeof(double));
  out[0] = ewald_rec(&s->param, &ew, &s->box, s->x, s->y, s->z, fx, fy, fz, s->q, stress, &vir);
  out[1] = vir;
  out[2] = ew.m1max;
  out[3] = ew.m2max;
  out[4] = ew.m3max;
  out[5] = ew.mmax;
  ewald_free(&ew);
}
