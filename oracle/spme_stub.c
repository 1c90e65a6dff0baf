/* TEST INFRASTRUCTURE.  MDBas's src/spme.c needs FFTW3, which is absent
 * here; the stock MDBas driver built for the link test gets these stand-ins
 * (include/spme.h:28-40).  A run that asks for SPME stops with a message:
 * the link test uses the explicit Ewald sum. */
#include <stdio.h>
#include <stdlib.h>

#include "global.h"

void init_spme(CTRL *ctrl, PARAM *param, EWALD *ewald, PBC *box)
{
  (void)ctrl; (void)param; (void)ewald; (void)box;
  fprintf(stderr, "this MDBas build has no SPME (FFTW3 is absent)\n");
  exit(3);
}

void spme_free(PARAM *param) { (void)param; }

double spme_energy(PARAM *param, EWALD *ewald, PBC *box, const double x[], const double y[],
                   const double z[], double fx[], double fy[], double fz[], const double q[],
                   double stress[6], double *virEwaldRec)
{
  (void)param; (void)ewald; (void)box; (void)x; (void)y; (void)z; (void)fx; (void)fy;
  (void)fz; (void)q; (void)stress; (void)virEwaldRec;
  fprintf(stderr, "this MDBas build has no SPME (FFTW3 is absent)\n");
  exit(3);
  return 0.0;
}
