/*
 * mdbas_nb.h -- C ABI of libmdbas_nb.so, the B200 (sm_100a) implementation of
 * MDBas's real-space nonbonded hot path.
 *
 * Three groups of entry points:
 *
 *  1. Drop-in replacements with MDBas's own prototypes.  A MDBas build links
 *     libmdbas_nb.so in place of obj/energy.o and obj/list.o; everything else
 *     (integrators, bonded terms, k-space, I/O) stays MDBas's own code, which
 *     these routines reach through weak references.  Errors go through
 *     my_error-style reporting (message on stderr/outFile, exit) exactly as in
 *     MDBas; the *_status API below returns codes instead.
 *
 *  2. A UserEnergyPtr plugin (include/user.h:29-33 of MDBas) plus the init call
 *     the plugin ABI lacks (charges, LJ parameters, exclusions) and a getter for
 *     the energy/virial the plugin ABI cannot return.
 *
 *  3. A device-resident engine (mdbas_nb_engine_*) that keeps positions,
 *     topology, the cluster-pair list and the fixed-point accumulators in HBM
 *     between calls; it is what the drop-in's mixed-precision mode and the
 *     benchmarks drive.  Every engine call returns an mdbas_nb_status.
 *
 * Units are MDBas internal units throughout: lengths in Angstrom, energies in
 * 10 J/mol (kcal/mol x 418.4), charges in e.
 */
#ifndef MDBAS_NB_H
#define MDBAS_NB_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* MDBas data model.  Field order and types match MDBas include/global.h    */
/* (enums :79-153, PBC :175-184, CTRL :195-217, PARAM :219-238, BOND         */
/* :247-252, ANGLE :254-259, DIHE :261-267, NEIGH :269-276, ENERGY :282-290, */
/* CONSTRAINT :296-300, EWALD :311-316) so that the same struct pointers can */
/* be passed across the ABI.  When MDBas's global.h is already included its  */
/* definitions are used instead.                                              */
/* ------------------------------------------------------------------------ */
#ifndef GLOBALH_INCLUDED
#ifndef MDBAS_NB_MIRROR_TYPES
#define MDBAS_NB_MIRROR_TYPES

enum ELEC_TYPE { NOELEC = 0, FULL = 1, SHIFT1 = 2, SHIFT2 = 3, SWITCH = 4 };
enum VDW_TYPE { NOVDW = 0, VFULL = 1, VSWITCH = 2 };
enum BOX_TYPE { NOBOX = 0, CUBIC = 1, ORBIC = 2, TCLIN = 3 };
enum INTEGRATOR_TYPE { LEAPFROG = 0, VELOCITY = 1 };
enum ENSEMBLE_TYPE { NVE = 0, NVT_B = 1, NPT_B = 2, NVT_H = 3, NPT_H = 4 };
enum BOND_TYPE { BHARM = 0, BMORSE = 1 };
enum ANGLE_TYPE { AHARM = 0 };
enum DIHE_TYPE { DCOS = 1, DHARM = 2 };

typedef struct {
  enum BOX_TYPE type;
  double a, a1, a2, a3, b, b1, b2, b3, c, c1, c2, c3;
  double u, u1, u2, u3, v, v1, v2, v3, w, w1, w2, w3;
  double pa, pb, pc, det, vol, vol0;
  double stress1, stress2, stress3;
  double stress4, stress5, stress6;
  double stress7, stress8, stress9;
} PBC;

typedef struct {
  int newjob;
  int keyRand, keyTraj, keyProp, keyForF, keyRest;
  int printOut, printProp, printTraj, printRest;
  int keyMd, mdType;
  int seed;
  int keyMinim;
  int keyLink, noLink;
  int keyConstH;
  int keyNb14, keyNumForce;
  int keyEwald, keyAlpha, keyMmax;
  enum ELEC_TYPE elecType;
  enum VDW_TYPE vdwType;
  enum INTEGRATOR_TYPE integrator;
  enum ENSEMBLE_TYPE ens;
} CTRL;

typedef struct {
  int step, nSteps;
  double timeStep, rTimeStep;
  int nAtom, nDegFree, nFrozen;
  int nBond, nAngle, nDihedral, nImproper, nUb;
  int nConst, maxCycle;
  double tolShake;
  double chargeConst, delr, scal14;
  double cutOff, rcutOff, cutOff2, rcutOff2;
  double cutOn, cutOn2, switch2;
  double temp0, press0, kinTemp0;
  double tolMinim, maxminsiz, maxminst;
} PARAM;

typedef struct {
  enum BOND_TYPE type;
  int a, b;
  double k, r0, beta;
} BOND;

typedef struct {
  enum ANGLE_TYPE type;
  int a, b, c;
  double k, theta0;
} ANGLE;

typedef struct {
  enum DIHE_TYPE type;
  int order;
  int a, b, c, d;
  double k, phi0, mult;
} DIHE;

typedef struct {
  int update;
  int linkRatio;
  int nCells;
  int sizeList;
  int nPair14;
} NEIGH;

typedef struct {
  double tot, pot, kin;
  double elec, vdw;
  double bond, ang, ub, dihe, impr;
  double conint, consv;
  double virelec, virvdw, virbond, virub;
  double virshake, virpot, virtot;
} ENERGY;

typedef struct {
  int a, b;
  double rc2;
} CONSTRAINT;

typedef struct {
  int nbsp;
  int mmax, m1max, m2max, m3max;
  double prec, tol, tol1, alpha;
} EWALD;

#endif /* MDBAS_NB_MIRROR_TYPES */
#endif /* GLOBALH_INCLUDED */

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum {
  MDBAS_NB_OK = 0,
  MDBAS_NB_ERR_ARG = 1,          /* invalid argument (null pointer, bad size)   */
  MDBAS_NB_ERR_CUDA = 2,         /* a CUDA runtime call failed                  */
  MDBAS_NB_ERR_NO_DEVICE = 3,    /* no usable sm_100 device                     */
  MDBAS_NB_ERR_ALLOC = 4,        /* device or host allocation failed            */
  MDBAS_NB_ERR_CAPACITY = 5,     /* a device list outgrew its capacity; the
                                    engine grows it and rebuilds, callers see
                                    this only when growing failed               */
  MDBAS_NB_ERR_BOX = 6,          /* box too small or unsupported for the path  */
  MDBAS_NB_ERR_LINKCELL = 7,     /* fewer than 2*linkRatio+1 cells per side
                                    (MDBas LNKCELL_NCELLS_ERROR)                */
  MDBAS_NB_ERR_EXCL = 8,         /* exclusion topology invalid (MDBas
                                    EXCLLIST_LASTATOM_ERROR / DIHE_NONPARAM)    */
  MDBAS_NB_ERR_UNSUPPORTED = 9,  /* option not implemented on this path        */
  MDBAS_NB_ERR_OVERFLOW = 10,    /* a fixed-point accumulator would overflow   */
  MDBAS_NB_ERR_NONFINITE = 11,   /* NaN/Inf coordinates                         */
  MDBAS_NB_ERR_MISSING = 12,     /* a MDBas routine this call delegates to
                                    (bonded terms, k-space) is not linked       */
  MDBAS_NB_ERR_STATE = 13        /* call out of order (e.g. compute before
                                    positions were set)                         */
} mdbas_nb_status;

const char *mdbas_nb_status_string(int status);
/* Last status recorded by any call in this process (drop-in routines record
 * their status here before reporting it the MDBas way). */
int mdbas_nb_last_status(void);
/* Text of the last CUDA or validation failure (empty when none). */
const char *mdbas_nb_last_message(void);
/* Library version and the compute capability it was built for (1000 = sm_100a). */
int mdbas_nb_version(void);
int mdbas_nb_build_arch(void);

/* Drop-in precision mode, read by energy()/ewald_energy()/nonbond_energy().
 *   0 (default): plain FP64 GPU form over the caller's Verlet list, the same
 *                pair set and operation order as MDBas's CPU loop.
 *   1          : FP32 pair arithmetic + 64-bit fixed-point accumulation over
 *                the library's own cluster-pair list (built on the device from
 *                the same coordinates; equal to MDBas's pair set whenever the
 *                caller's list is current, i.e. no atom moved more than half
 *                the skin since it was built).
 * The environment variable MDBAS_NB_MODE=fp64|mixed sets the initial value. */
int mdbas_nb_set_mode(int mode);
int mdbas_nb_get_mode(void);

/* ------------------------------------------------------------------------ */
/* 1. Drop-in replacements (MDBas include/energy.h, include/list.h)          */
/* ------------------------------------------------------------------------ */

/* Replaces init_energy_ptrs (energy.c:35-92): records ctrl->elecType and
 * ctrl->vdwType; unknown values report UNKNOWN_ELEC/VDW errors like MDBas. */
void init_energy_ptrs(CTRL *ctrl);

/* Replaces energy() (include/energy.h:30-37, src/energy.c:103-205): zeroes
 * forces, energies and the stress tensor, evaluates the nonbonded terms on the
 * GPU, then the bonded terms on the GPU (section 8) and MDBas's freeze_atoms
 * (weak reference). */
void energy(CTRL *ctrl, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box, NEIGH *neigh,
            BOND bond[], BOND ub[], ANGLE angle[], DIHE dihe[], DIHE impr[],
            const double x[], const double y[], const double z[],
            double vx[], double vy[], double vz[], double fx[], double fy[],
            double fz[], const double q[], const double eps[], const double sig[],
            const double eps14[], const double sig14[], const int frozen[],
            const int neighList[], const int neighPair[], const int neighOrder[],
            const int neighList14[], int **exclList, const int exclPair[]);

/* Replaces nonbond_energy (include/energy.h:39-42, src/energy.c:216-345):
 * cut-off Coulomb (shift1/shift2/switch per init_energy_ptrs) + switched LJ
 * over the caller's list; accumulates into fx/fy/fz and ener. */
void nonbond_energy(PARAM *param, ENERGY *ener, PBC *box,
                    const double x[], const double y[], const double z[], double fx[], double fy[],
                    double fz[], const double q[], const double eps[], const double sig[],
                    const int neighList[], const int neighPair[], const int neighOrder[]);

/* Replaces nonbond14_energy (include/energy.h:44-47, src/energy.c:356-439). */
void nonbond14_energy(PARAM *param, ENERGY *ener, PBC *box, NEIGH *neigh,
                      const double x[], const double y[], const double z[], double fx[], double fy[],
                      double fz[], const double q[], const double eps[], const double sig[],
                      const int neighList14[]);

/* Replaces ewald_energy (include/energy.h:49-53, src/energy.c:450-643):
 * real-space Ewald direct term + switched LJ over the caller's list and the
 * erf exclusion correction on the GPU; keyEwald==1/2 k-space by ewald_rec
 * (section 9) / spme_energy (section 7), also on the GPU. */
void ewald_energy(CTRL *ctrl, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box, const double x[],
                  const double y[], const double z[], double fx[], double fy[],
                  double fz[], const double q[], const double eps[], const double sig[],
                  const int neighList[], const int neighPair[], const int neighOrder[],
                  int **exclList, const int exclPair[]);

/* Replaces ewald14_energy (include/energy.h:55-58, src/energy.c:654-742). */
void ewald14_energy(PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box, NEIGH *neigh,
                    const double x[], const double y[], const double z[], double fx[], double fy[],
                    double fz[], const double q[], const double eps[], const double sig[],
                    const int neighList14[]);

/* Replaces makelist (include/list.h:28-31, src/list.c:29-106). */
void makelist(CTRL *ctrl, PARAM *param, PBC *box, NEIGH *neigh, CONSTRAINT constList[],
              BOND bond[], ANGLE angle[], DIHE dihe[], DIHE impr[], double x[], double y[],
              double z[], int frozen[], int **neighList, int **neighPair, int **neighOrder,
              int **neighList14, int ***exclList, int **exclPair);

/* Replaces exclude_list (include/list.h:33-35, src/list.c:108-894): half
 * (j>i) exclusion rows, 1-4 pair list; host code (one-off topology walk). */
void exclude_list(CTRL *ctrl, PARAM *param, NEIGH *neigh, CONSTRAINT constList[],
                  BOND bond[], ANGLE angle[], DIHE dihe[], DIHE impr[],
                  int **neighList14, int ***exclList, int **exclPair);

/* Replaces verlet_list (include/list.h:37-39, src/list.c:896-1040): O(N^2)
 * half list built on the GPU, same entries in the same order as MDBas. */
void verlet_list(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[], double z[],
                 int frozen[], int **neighList, int **neighPair, int **neighOrder,
                 int **exclList, int exclPair[]);

/* Replaces verlet_list_update (include/list.h:41-43, src/list.c:1042-1123). */
void verlet_list_update(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[], double z[],
                        int frozen[], int **neighList, int neighPair[], int **exclList,
                        int exclPair[]);

/* Replaces link_cell_exclude_list (include/list.h:45-47, src/list.c:1125-1791):
 * symmetric exclusion rows; host code. */
void link_cell_exclude_list(CTRL *ctrl, PARAM *param, NEIGH *neigh, CONSTRAINT constList[],
                            BOND bond[], ANGLE angle[], DIHE dihe[], DIHE impr[],
                            int **neighList14, int ***exclList, int **exclPair);

/* Replaces link_cell_verlet_list (include/list.h:49-51, src/list.c:1793-2274):
 * wraps x/y/z in place (image_update), bins into link cells and builds the
 * half list on the GPU, same entries in the same order as MDBas. */
void link_cell_verlet_list(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[], double z[],
                           int frozen[], int **neighList, int **neighPair, int **neighOrder,
                           int **exclList, int exclPair[]);

/* Replaces link_cell_verlet_list_update (include/list.h:53-55,
 * src/list.c:2276-2619): no wrap, list storage reused and grown by 1% steps. */
void link_cell_verlet_list_update(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                                  double z[], int frozen[], int **neighList, int neighPair[],
                                  int neighOrder[], int **exclList, int exclPair[]);

/* ------------------------------------------------------------------------ */
/* Status-returning forms of the drop-in list and energy routines.           */
/* They take the same arguments and never exit the process.                  */
/* ------------------------------------------------------------------------ */
int mdbas_nb_verlet_list_status(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                                double z[], int frozen[], int **neighList, int **neighPair,
                                int **neighOrder, int **exclList, int exclPair[], int update);
int mdbas_nb_link_cell_list_status(PARAM *param, PBC *box, NEIGH *neigh, double x[], double y[],
                                   double z[], int frozen[], int **neighList, int **neighPair,
                                   int **neighOrder, int **exclList, int exclPair[], int update);
int mdbas_nb_ewald_energy_status(CTRL *ctrl, PARAM *param, ENERGY *ener, EWALD *ewald, PBC *box,
                                 const double x[], const double y[], const double z[], double fx[],
                                 double fy[], double fz[], const double q[], const double eps[],
                                 const double sig[], const int neighList[], const int neighPair[],
                                 const int neighOrder[], int **exclList, const int exclPair[]);

/* ------------------------------------------------------------------------ */
/* 2. UserEnergyPtr plugin (MDBas include/user.h:29-33, plugins/custom_nb.c) */
/* ------------------------------------------------------------------------ */

/* The plugin ABI carries neither charges, LJ parameters nor exclusions:
 * register them once.  eps/sig are MDBas per-atom values (eps_i =
 * sqrt(eps*418.4), sig_i = FORF sigma).  exclPair/exclList use MDBas's
 * layout (rows may be half or symmetric; only j>i entries are used).
 * alpha is the Ewald splitting parameter; vdwSwitch selects vdw_switch (1)
 * or no LJ (0). */
int mdbas_nb_plugin_init(int nAtom, const double q[], const double eps[], const double sig[],
                         const int exclPair[], int **exclList, double alpha, int vdwSwitch);

/* UserEnergyPtr-compatible entry: real-space Ewald + switched LJ over the
 * given half list, exclusion correction included; ADDS forces into fx/fy/fz
 * and returns elec+vdw (internal units).  neighList14 is unused (water-style
 * systems have no 1-4 pairs; ewald14_energy covers them in the drop-in). */
double mdbas_nb_user_energy(const PARAM *param, const PBC *box,
                            const double x[], const double y[], const double z[],
                            double fx[], double fy[], double fz[],
                            const int neighList[], const int neighPair[], const int neighOrder[],
                            const int neighList14[]);

/* Energy and virial terms of the last mdbas_nb_user_energy call:
 * out[0..3] = elec, vdw, virelec, virvdw. */
int mdbas_nb_plugin_last_energy(double out[4]);
void mdbas_nb_plugin_release(void);

/* ------------------------------------------------------------------------ */
/* 3. Device-resident engine                                                 */
/* ------------------------------------------------------------------------ */
typedef struct mdbas_nb_engine mdbas_nb_engine;

typedef struct {
  int nAtom;
  int device;             /* CUDA device ordinal                             */
  double cutOff;          /* rc (A)                                          */
  double cutOn;           /* LJ switch start (A)                             */
  double delr;            /* Verlet skin (A)                                 */
  double alpha;           /* Ewald splitting parameter (1/A)                 */
  double chargeConst;     /* Coulomb constant in internal units              */
  int vdwSwitch;          /* 1: vdw_switch, 0: no LJ                         */
  int precision;          /* 0: plain FP64 pair kernel, 1: FP32 + fixed point */
  int linkRatio;          /* precision 0: MDBas link ratio (1..5)            */
  int noLink;             /* precision 0: force the all-pairs builder        */
} mdbas_nb_engine_config;

/* Energy/virial terms (internal units) filled by mdbas_nb_engine_energies. */
typedef struct {
  double elec_direct;     /* sum qel*erfc(a r)/r over in-cut-off pairs       */
  double elec_corr;       /* -sum qel*erf(a r)/r over excluded pairs         */
  double elec_self;       /* -C a/sqrt(pi) sum q^2                           */
  double vdw;             /* switched LJ                                     */
  double vir_direct;      /* sum r dE/dr, MDBas's virial convention          */
  double vir_corr;
  double vir_vdw;
  double n_pairs;         /* in-cut-off pair interactions evaluated          */
} mdbas_nb_energies;

int mdbas_nb_engine_create(mdbas_nb_engine **out, const mdbas_nb_engine_config *cfg,
                           const PBC *box);
int mdbas_nb_engine_destroy(mdbas_nb_engine *e);
/* Work on this CUDA stream (cudaStream_t passed as void*; NULL = default). */
int mdbas_nb_engine_set_stream(mdbas_nb_engine *e, void *stream);
int mdbas_nb_engine_set_box(mdbas_nb_engine *e, const PBC *box);
/* Per-atom topology.  eps/sig as MDBas per-atom values; frozen may be NULL;
 * exclusions in MDBas row layout flattened: exclPair[i] entries of exclFlat
 * per atom in order (half or symmetric rows; duplicates are harmless). */
int mdbas_nb_engine_set_topology(mdbas_nb_engine *e, const double *q, const double *eps,
                                 const double *sig, const int *frozen, const int *exclPair,
                                 const int *exclFlat);
/* Positions: host pointers (copied H2D on the engine stream) or device
 * pointers (device != 0), FP64, original atom order. */
int mdbas_nb_engine_set_positions(mdbas_nb_engine *e, const double *x, const double *y,
                                  const double *z, int device_ptrs);
/* Sort atoms into cells/clusters and build the cluster-pair list (precision 1)
 * or the MDBas-format half list (precision 0).  A precision-1 rebuild on the
 * grid and list room of the previous build returns without waiting for the
 * list counts; its outcome is settled by the next call that returns results
 * (get_forces, energies, list_stats, export_pairs, autotune, set_positions,
 * md_init, md_run): a list that outgrew its room is built again with more
 * room and the evaluation redone, and non-finite positions return
 * MDBAS_NB_ERR_NONFINITE there. */
int mdbas_nb_engine_build(mdbas_nb_engine *e);
/* Refresh the per-atom float4 layout from the current FP64 positions without
 * rebuilding the list (between rebuilds during dynamics). */
int mdbas_nb_engine_refresh(mdbas_nb_engine *e);
/* Evaluate forces, energies and virial into the device accumulators. */
int mdbas_nb_engine_compute(mdbas_nb_engine *e);
/* Forces in original atom order, FP64; host or device destination. */
int mdbas_nb_engine_get_forces(mdbas_nb_engine *e, double *fx, double *fy, double *fz,
                               int device_ptrs);
int mdbas_nb_engine_energies(mdbas_nb_engine *e, mdbas_nb_energies *out);
/* One evaluation on host arrays in a single call: set_positions (host), then
 * build (rebuild != 0) or refresh (rebuild == 0: the atoms are within half
 * the skin of the last build), compute, get_forces into fx/fy/fz and, when
 * out is not NULL, energies; one wait.  The same results as those calls made
 * one by one. */
int mdbas_nb_engine_evaluate(mdbas_nb_engine *e, const double *x, const double *y,
                             const double *z, int rebuild, double *fx, double *fy, double *fz,
                             mdbas_nb_energies *out);
/* Statistics of the current list: out[0] = clusters (or atoms), out[1] =
 * list entries (cluster pairs or atom pairs), out[2] = candidate atom pairs
 * evaluated per compute, out[3] = list capacity. */
int mdbas_nb_engine_list_stats(mdbas_nb_engine *e, long long out[4]);
/* Export the atom-pair set the current list evaluates within distance
 * sqrt(r2max) (original indices, i<j), for parity checks.  *count receives
 * the number of pairs; pairs (2*capacity ints) may be NULL to query it. */
int mdbas_nb_engine_export_pairs(mdbas_nb_engine *e, double r2max, int *pairs, long long capacity,
                                 long long *count);
/* Pair kernel variant of the mixed-precision path: 7 (default) is variant 4
 * in a lean form (pairs outside the mask placed at r^2 = 1e30 instead of
 * zeroed products, fewer registers; the same forces bit for bit); 4 takes two
 * 4-atom halves of j clusters per warp step against an 8-atom i cluster, a
 * lane's two pairs in packed f32x2 arithmetic, over the inner list (the
 * halves holding a pair within the cut-off, written by the list build for
 * the build's positions, or within the pruning radius during dynamics) and
 * over the full list once positions have changed since the build; 2 computes
 * every pair of each 8x8 cluster pair in one warp step, a lane's two pairs in
 * packed f32x2 arithmetic, with each chunk of 8 cluster pairs staged in
 * shared memory; 0 is the same in scalar FP32 without staging; 1 filters the
 * pairs first and computes only in-cut-off pairs from per-atom queues; 3 is
 * variant 2 with each chunk's j data brought into shared memory by
 * asynchronous bulk copies (cp.async.bulk with an mbarrier, double buffered)
 * instead of per-lane loads -- the same results as 2 bit for bit.  Variants
 * 0-3 always walk the full list.  5 is variant 4 at up to 80 registers.
 * 6 splits each inner-list half into its two 4-atom i halves and computes
 * 4 x 4 units, four per warp step (i clusters of 4 atoms: fewer pairs beyond
 * the cut-off); without a current inner list it runs as variant 4. */
int mdbas_nb_engine_set_variant(mdbas_nb_engine *e, int variant);
/* Autotuner of the mixed-precision pair kernel: times each variant and
 * launch shape (threads per block x blocks per SM) on the current list with
 * CUDA events and keeps the fastest for later computes.  out = {variant,
 * block, blocks per SM, candidates tried}.  Call after build; the
 * accumulators are left dirty, so compute again before reading forces. */
int mdbas_nb_engine_autotune(mdbas_nb_engine *e, int out[4]);
/* Mixed precision: one synchronising list build with CUDA events between its
 * stages (no counterpart in MDBas; measurement of the build).  ms[0..5] =
 * binning into columns, the columns' scans and padding, scatter into
 * columns, in-column z sort, cluster layout, cluster-pair search. */
int mdbas_nb_engine_build_stages(mdbas_nb_engine *e, double ms[6]);
/* Kernels this engine launched since creation. */
long long mdbas_nb_engine_launch_count(mdbas_nb_engine *e);
/* Average duration (ms) of the pair kernel over the launches recorded since
 * the last call with reset != 0, measured with CUDA events on the engine
 * stream when timing is enabled. */
int mdbas_nb_engine_set_timing(mdbas_nb_engine *e, int enable);
int mdbas_nb_engine_kernel_time(mdbas_nb_engine *e, int which, double *avg_ms, long long *count,
                                int reset);

/* ------------------------------------------------------------------------ */
/* 4. Device-resident velocity-Verlet dynamics                               */
/*    (replaces the loop src/mdbas.c:244-300 over vv_integrate,               */
/*    src/integrate.c:1518-1634 vv_nve / 1636-1750 vv_nvt_b, with SHAKE and   */
/*    RATTLE of src/shake.c:209-456, makelist and energy)                    */
/* ------------------------------------------------------------------------ */
/* Start dynamics from the engine's current positions.  mass in MDBas units
 * (amu); velocities in A/ps (NULL = zero); timeStep in ps.  listUpdate > 0
 * rebuilds the list every listUpdate steps (MDBas's "list" keyword);
 * listUpdate = 0 rebuilds when an atom has moved more than delr/2 since the
 * last build.  Constraints: nConst pairs (constAtoms[2k], constAtoms[2k+1])
 * at squared length constLen2[k] (A^2), solved per molecule with MDBas's
 * SHAKE/RATTLE iteration (tolShake <= 0 -> 1e-8, maxCycle <= 0 -> 150);
 * a constrained molecule holds at most 16 atoms and 32 constraints.
 * Evaluates the forces at the start positions. */
int mdbas_nb_engine_md_init(mdbas_nb_engine *e, const double *mass, const double *vx,
                            const double *vy, const double *vz, double timeStep, int listUpdate,
                            int nConst, const int *constAtoms, const double *constLen2,
                            double tolShake, int maxCycle);
/* Advance nSteps steps.  tauT > 0 applies MDBas's Berendsen scaling toward
 * targetTemp (K) after the second half kick (vv_nvt_b); tauT <= 0 is NVE.
 * Every energyEvery steps (if energies != NULL) a row {step, potential,
 * kinetic, total} (internal units; potential = the nonbonded real-space
 * terms plus the Ewald self term plus the bonded terms of
 * mdbas_nb_engine_set_bonded) is appended to energies.  Returns
 * MDBAS_NB_ERR_UNSUPPORTED if SHAKE did not converge (CONVERG_SHAKE_ERROR). */
int mdbas_nb_engine_md_run(mdbas_nb_engine *e, int nSteps, int energyEvery, double targetTemp,
                           double tauT, double *energies);
/* Mixed precision (precision 1) runs whole steps as CUDA graphs of
 * stepsPerLaunch steps (default 20): the rebuild test is made on the device
 * and the list build is a conditional graph node, so the host synchronises
 * once per launch.  A launch whose rebuild outgrows the pair list is redone
 * from a snapshot with a larger list.  0 runs every step from the host.
 * Both forms give bit-identical trajectories (fixed-point sums). */
int mdbas_nb_engine_md_set_graph(mdbas_nb_engine *e, int stepsPerLaunch);
/* Dynamic pruning of the mixed form (off by default; buffer > 0 enables): the pair
 * kernel walks an inner copy of the list holding only the pairs found within
 * cutOff + buffer, re-pruned from the full list whenever an atom has moved
 * more than buffer/2 since the last prune (and after every rebuild), so no
 * pair inside the cut-off is ever missed.  0 <= buffer <= delr; call before
 * md_init.  Results are bit-identical with and without it.  With the 2 A skin
 * of the 96k water benchmark a 0.5 A buffer removes only 11% of the pair
 * kernel's time and the prune pass costs as much, so it is off by default. */
int mdbas_nb_engine_md_set_prune(mdbas_nb_engine *e, double buffer);
/* out[0] steps taken, out[1] list builds, out[2] largest SHAKE iteration
 * count of the last md_run, out[3] constrained molecules, out[4] prunes,
 * out[5] 1 while the pair kernel walks the pruned list. */
int mdbas_nb_engine_md_stats(mdbas_nb_engine *e, long long out[6]);
/* Current positions / velocities (original atom order). */
int mdbas_nb_engine_get_positions(mdbas_nb_engine *e, double *x, double *y, double *z,
                                  int device_ptrs);
int mdbas_nb_engine_get_velocities(mdbas_nb_engine *e, double *vx, double *vy, double *vz,
                                   int device_ptrs);

/* ------------------------------------------------------------------------ */
/* 7. Reciprocal space: smooth particle-mesh Ewald on the GPU                 */
/*    (replaces src/spme.c, which needs FFTW3; include/spme.h:28-40)          */
/* ------------------------------------------------------------------------ */
/* MDBas prototypes: init_spme sets ewald->m1max..m3max, mmax (and alpha/tol
 * as MDBas does); spme_energy adds the reciprocal forces to the caller's
 * arrays, removes the mean force, fills stress[6] and the virial and returns
 * the reciprocal energy plus the self and non-neutral terms; spme_free is a
 * no-op (the device context is per process). */
void init_spme(CTRL *ctrl, PARAM *param, EWALD *ewald, PBC *box);
void spme_free(PARAM *param);
double spme_energy(PARAM *param, EWALD *ewald, PBC *box, const double x[], const double y[],
                   const double z[], double fx[], double fy[], double fz[], const double q[],
                   double stress[6], double *virEwaldRec);
/* Status form on host or device arrays: grid m1 x m2 x m3, B-spline order
 * nbsp (2..16).  Forces minus their mean are added to fx/fy/fz.  out[0] =
 * energy (reciprocal + self + non-neutral), out[1] = virial, out[2..7] =
 * stress.  stream: cudaStream_t (NULL = default). */
int mdbas_nb_spme(int nAtom, const PBC *box, double alpha, double chargeConst, int m1, int m2,
                  int m3, int nbsp, const double *x, const double *y, const double *z,
                  const double *q, double *fx, double *fy, double *fz, double out[8],
                  int device_ptrs, void *stream);

/* ------------------------------------------------------------------------ */
/* 9. Explicit reciprocal-space Ewald sum on the GPU (replaces src/ewald.c:   */
/*    10-354, include/ewald.h)                                               */
/* ------------------------------------------------------------------------ */
/* MDBas prototypes: init_ewald sets prec, tol, alpha (unless keyAlpha), tol1,
 * m1max..m3max (unless keyMmax) and mmax = the number of k-vectors, as MDBas
 * does (without MDBas's per-atom table allocation); ewald_free is a no-op;
 * ewald_rec adds the reciprocal forces to fx/fy/fz and then multiplies the
 * whole arrays by 4 pi C / V as MDBas does (energy() calls it on zeroed
 * arrays), fills stress[6] and the virial and returns the reciprocal energy
 * plus the self and non-neutral terms. */
void init_ewald(CTRL *ctrl, PARAM *param, EWALD *ewald, PBC *box);
void ewald_free(EWALD *ewald);
double ewald_rec(PARAM *param, EWALD *ewald, PBC *box, const double x[], const double y[],
                 const double z[], double fx[], double fy[], double fz[], const double q[],
                 double stress[6], double *virEwaldRec);
/* Status form on host or device arrays: every k = 2 pi (m1 u + m2 v + m3 w)
 * with |m_d| <= m{d}max inside MDBas's reciprocal cut-off.  The reciprocal
 * forces are added to fx/fy/fz.  out[0] = energy (reciprocal + self +
 * non-neutral), out[1] = virial, out[2..7] = stress.  stream: cudaStream_t
 * (NULL = default). */
int mdbas_nb_ewald_rec(int nAtom, const PBC *box, double alpha, double chargeConst, int m1max,
                       int m2max, int m3max, const double *x, const double *y, const double *z,
                       const double *q, double *fx, double *fy, double *fz, double out[8],
                       int device_ptrs, void *stream);

/* ------------------------------------------------------------------------ */
/* 8. Bonded terms on the GPU (replace src/internal.c:21-620,                 */
/*    include/internal.h:28-42)                                              */
/* ------------------------------------------------------------------------ */
/* MDBas prototypes: add the terms' forces to fx/fy/fz (host arrays) and their
 * energies (and the bond / Urey-Bradley virials) to ener, as MDBas does:
 * harmonic or Morse bonds (BHARM, BMORSE), harmonic Urey-Bradley terms,
 * harmonic angles, cosine or harmonic dihedrals and impropers (DCOS, DHARM).
 * FP64 with MDBas's operation order; each force component receives the
 * terms' contributions in MDBas's order (harmonic bonds and Urey-Bradley
 * terms are bit-identical; terms with exp, acos, atan2, cos or sin agree to
 * the last place of those functions).  Errors terminate like MDBas. */
void bond_energy(const PARAM *param, ENERGY *ener, const PBC *box, const BOND bond[],
                 const double *x, const double *y, const double *z, double *fx, double *fy,
                 double *fz);
void ub_energy(const PARAM *param, ENERGY *ener, const PBC *box, const BOND ub[], const double *x,
               const double *y, const double *z, double *fx, double *fy, double *fz);
void angle_energy(const PARAM *param, ENERGY *ener, const PBC *box, const ANGLE angle[],
                  const double *x, const double *y, const double *z, double *fx, double *fy,
                  double *fz);
void dihedral_energy(const PARAM *param, ENERGY *ener, const PBC *box, const DIHE dihe[],
                     const double *x, const double *y, const double *z, double *fx, double *fy,
                     double *fz);
void improper_energy(const PARAM *param, ENERGY *ener, const PBC *box, const DIHE impr[],
                     const double *x, const double *y, const double *z, double *fx, double *fy,
                     double *fz);
/* Status form of one routine: kind 0 bonds, 1 angles, 2 Urey-Bradley,
 * 3 dihedrals, 4 impropers (the order of energy(), src/energy.c:167-190);
 * terms points to nTerms MDBas structs (BOND, ANGLE, BOND, DIHE, DIHE).
 * Host arrays; forces are added to fx/fy/fz; out[0] = energy, out[1] =
 * virial (bonds and Urey-Bradley; 0 otherwise).  An atom index outside
 * [0, nAtom) returns MDBAS_NB_ERR_ARG. */
int mdbas_nb_bonded(int kind, int nAtom, const PBC *box, int nTerms, const void *terms,
                    const double *x, const double *y, const double *z, double *fx, double *fy,
                    double *fz, double out[2]);
/* Bonded terms of an engine (atom indices in the engine's order; for a batch
 * the concatenated indices, each term inside one replica).  Dynamics
 * (section 4) then adds their forces after the nonbonded ones and their
 * energy to the potential of the energy rows.  Counts of 0 clear a kind. */
int mdbas_nb_engine_set_bonded(mdbas_nb_engine *e, int nBond, const BOND *bond, int nAngle,
                               const ANGLE *angle, int nUb, const BOND *ub, int nDihedral,
                               const DIHE *dihe, int nImproper, const DIHE *impr);
/* Evaluate the engine's bonded terms at its current positions: forces are
 * added to fx/fy/fz (host or device; NULL = energies only); out = {bond,
 * angle, Urey-Bradley, dihedral, improper energies, bond virial, Urey-Bradley
 * virial}. */
int mdbas_nb_engine_bonded(mdbas_nb_engine *e, double *fx, double *fy, double *fz,
                           int device_ptrs, double out[7]);

/* Reciprocal space in the dynamics, as MDBas's energy() with keyEwald 1
 * (ewald_rec) or 2 (spme_energy) adds it: kind 0 off (default: real space
 * only, the benchmark's potential), 1 explicit Ewald sum over |m_d| <=
 * m{d} (section 9), 2 SPME on an m1 x m2 x m3 grid with B-splines of order
 * nbsp (section 7); the engine's alpha and charge constant.  Single boxes
 * only (MDBAS_NB_ERR_UNSUPPORTED for a batch); call after the topology.
 * Dynamics then add the reciprocal forces every step (inside the step's
 * CUDA graph) and the energy rows' potential holds the reciprocal and
 * non-neutral terms as well.  Explicit Ewald is deterministic, and so is
 * SPME when every grid dimension is a multiple of 8 (other grids spread
 * charges with FP64 atomics and agree run to run only to rounding). */
int mdbas_nb_engine_set_kspace(mdbas_nb_engine *e, int kind, int m1, int m2, int m3, int nbsp);
/* The engine's reciprocal term at its current positions: forces added to
 * fx/fy/fz (host arrays, NULL = energy only); out[0] = energy (reciprocal +
 * self + non-neutral, MDBas's ewald_rec / spme_energy value), out[1] =
 * virial. */
int mdbas_nb_engine_kspace(mdbas_nb_engine *e, double *fx, double *fy, double *fz, double out[2]);

/* ------------------------------------------------------------------------ */
/* 6. Adjoint of the real-space energy (no counterpart in MDBas, whose        */
/*    numderiv.c gives only finite differences)                              */
/* ------------------------------------------------------------------------ */
/* On an FP64-form engine (precision 0) after build: gq/geps/gsig receive
 * dE/d(q_i, eps_i, sig_i) per atom (eps_i, sig_i the per-atom MDBas values;
 * E = real-space direct + exclusion correction + switched LJ + self term).
 * With upstream weights v = (vx, vy, vz) on the forces F = -dE/dx, also
 * hx/hy/hz = d(v.F)/dx (= -H v, a Hessian-vector product along positions)
 * and pq/peps/psig = d(v.F)/d(q_i, eps_i, sig_i); pass vx = NULL to skip.
 * Arrays of nAtom doubles, host (device_ptrs = 0) or device. */
int mdbas_nb_engine_adjoint(mdbas_nb_engine *e, const double *vx, const double *vy,
                            const double *vz, double *gq, double *geps, double *gsig,
                            double *hx, double *hy, double *hz, double *pq, double *peps,
                            double *psig, int device_ptrs);

/* ------------------------------------------------------------------------ */
/* 5. Batches of independent boxes (no counterpart in MDBas, which runs one   */
/*    system per process)                                                    */
/* ------------------------------------------------------------------------ */
/* An engine over nRep independent periodic boxes (orthorhombic) whose atoms
 * are concatenated: replica r owns repAtoms[r] consecutive atoms, in order.
 * cfg->nAtom = sum of repAtoms; mixed precision only (cfg->precision = 1).
 * Every engine call above then works on the concatenated arrays: topology
 * with global atom indices in the exclusions, positions, forces, energies
 * (summed over replicas) and dynamics.  The list build, the pair kernel, the
 * exclusion correction and each integration stage run as one launch over
 * all replicas, each pair with its own replica's box. */
int mdbas_nb_batch_create(mdbas_nb_engine **out, const mdbas_nb_engine_config *cfg, int nRep,
                          const PBC *boxes, const int *repAtoms);
/* Number of replicas of an engine (1 for a single system). */
int mdbas_nb_batch_count(mdbas_nb_engine *e);


/* ------------------------------------------------------------------------ */
/* Evaluation without device allocation (no counterpart in MDBas).           */
/* ------------------------------------------------------------------------ */
/* For callers that cannot let the library call cudaMalloc -- programs that
 * own all device memory through their own allocator, or loops that must not
 * hit the device-wide synchronisation cudaMalloc/cudaFree imply.  Same work
 * as the plain FP64 form of ewald_energy (direct Ewald term + switched LJ
 * over a MDBas half list, erf exclusion correction for every excluded pair
 * j>i), but every array is a DEVICE pointer owned by the caller and the only
 * scratch is a fixed area compiled into the library:
 * MDBAS_NB_NOALLOC_SCRATCH_BYTES per GPU that loads it, held until exit,
 * enough for MDBAS_NB_NOALLOC_MAX_ATOMS atoms; larger systems are rejected
 * with MDBAS_NB_ERR_CAPACITY.  The function calls no cudaMalloc/cudaFree.
 *   x..sig, neighList/neighPair/neighOrder (MDBas layout), exclStart
 *   (nAtom+1 offsets) + exclFlat (rows as in MDBas's exclList): inputs;
 *   fx/fy/fz: forces are ADDED into them; energies (host, 6 doubles):
 *   eDir, eCorr, eVdw, virDir, virCorr, virVdw.
 * The first call on each device resolves the scratch area's device address
 * (cudaGetSymbolAddress) with that device current: make it before any stream
 * capture.  All calls share the scratch area, so calls that overlap on the
 * GPU (unordered streams) race; order them on one stream or serialise them.
 * Runs on `stream` (cudaStream_t as void*, NULL = default) and returns after
 * the energies are copied back. */
#define MDBAS_NB_NOALLOC_MAX_ATOMS 131072
#define MDBAS_NB_NOALLOC_SCRATCH_BYTES 1574656
int mdbas_nb_ewald_fp64_noalloc(int nAtom, const PBC *box, double cutOff, double cutOn,
                                double alpha, double chargeConst, int vdwSwitch,
                                const double *x, const double *y, const double *z,
                                const double *q, const double *eps, const double *sig,
                                const int *neighList, const int *neighPair,
                                const int *neighOrder, const int *exclStart,
                                const int *exclFlat, double *fx, double *fy, double *fz,
                                double energies[6], void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MDBAS_NB_H */
