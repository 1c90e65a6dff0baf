/*
 * mdbas_oracle.h -- CPU restatement of MDBas's real-space nonbonded hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU library.  Only tests/,
 * the smoke check and bench.py's CPU-baseline leg load it; the product never
 * links, loads or calls it.  Every routine keeps MDBas's FP64 operation order
 * (compiled with -ffp-contract=off) so that its results are bit-identical to
 * the reference C built by oracle/Makefile, which the CPU tests check.
 *
 * Box layout (ORC_BOX_*): the PBC fields MDBas's hot path reads.
 * Exclusions: CSR rows (exclStart[n+1], exclFlat), either MDBas's half rows
 * (exclude_list, j>i) or its symmetric rows (link_cell_exclude_list).
 */
#ifndef MDBAS_ORACLE_H
#define MDBAS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_A1 = 0, ORC_A2, ORC_A3, ORC_B1, ORC_B2, ORC_B3, ORC_C1, ORC_C2, ORC_C3,
  ORC_U1, ORC_U2, ORC_U3, ORC_V1, ORC_V2, ORC_V3, ORC_W1, ORC_W2, ORC_W3,
  ORC_PA, ORC_PB, ORC_PC, ORC_VOL, ORC_DET, ORC_BOX_LEN
};

/* Pair-potential parameters of one evaluation (PARAM/EWALD fields). */
typedef struct {
  double chargeConst, alpha;
  double cutOff, cutOn, cutOff2, cutOn2, rcutOff, rcutOff2, switch2;
  int vdwSwitch; /* 1: vdw_switch, 0: vdw_none */
  int elecType;  /* enum ELEC_TYPE, used by orc_nonbond_energy only */
} orc_param;

int orc_nint(double x);
void orc_init_box(int type, const double cell[9], double box[ORC_BOX_LEN]);
void orc_fill_param(double cutOff, double cutOn, double alpha, double chargeConst,
                    int vdwSwitch, int elecType, orc_param *p);
double orc_dist(int type, const double box[ORC_BOX_LEN], double delta[3]);
void orc_image_update(int type, const double box[ORC_BOX_LEN], int n, double *x, double *y,
                      double *z);

long orc_verlet_list(int n, int type, const double box[ORC_BOX_LEN], double cutOff, double delr,
                     const double *x, const double *y, const double *z, const int *frozen,
                     const int *exclStart, const int *exclFlat, int *neighPair,
                     int *neighOrder, int *neighList, long capacity);

long orc_link_cell_list(int n, int type, const double box[ORC_BOX_LEN], double cutOff,
                        double delr, int linkRatio, const double *x, const double *y,
                        const double *z, const int *frozen, const int *exclStart,
                        const int *exclFlat, int *neighPair, int *neighOrder, int *neighList,
                        long capacity, int *nCells);

int orc_link_cell_counts(int type, const double box[ORC_BOX_LEN], double cutOff, double delr,
                         int linkRatio, int nlc[3]);

/* out[0..7] = eDir, eCorr, evdw, virDir, virCorr, virvdw, nPairsInCut, 0 */
void orc_ewald_energy(int n, int type, const double box[ORC_BOX_LEN], const orc_param *p,
                      const double *x, const double *y, const double *z, const double *q,
                      const double *eps, const double *sig, const int *neighList,
                      const int *neighPair, const int *neighOrder, const int *exclStart,
                      const int *exclFlat, double *fx, double *fy, double *fz, double out[8]);

/* out[0..4] = elec, vdw, virelec, virvdw, nPairsInCut */
void orc_nonbond_energy(int n, int type, const double box[ORC_BOX_LEN], const orc_param *p,
                        const double *x, const double *y, const double *z, const double *q,
                        const double *eps, const double *sig, const int *neighList,
                        const int *neighPair, const int *neighOrder, double *fx, double *fy,
                        double *fz, double out[5]);

double orc_self_energy(int n, const double *q, double chargeConst, double alpha);

long orc_pairs_within(int n, int type, const double box[ORC_BOX_LEN], double r2max,
                      const double *x, const double *y, const double *z, const int *frozen,
                      const int *exclStart, const int *exclFlat, int *pairs, long capacity);

int orc_forces_subset(int n, int type, const double box[ORC_BOX_LEN], const orc_param *p,
                      const double *x, const double *y, const double *z, const double *q,
                      const double *eps, const double *sig, const int *exclStart,
                      const int *exclFlat, int nsub, const int *subset, double *fx, double *fy,
                      double *fz);

#ifdef __cplusplus
}
#endif

#endif
