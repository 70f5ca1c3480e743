// Entry points whose GPU implementation is not built yet: they return
// INVALID_PARAMETERS without touching their arguments.
#include "../../include/bksp.h"
extern "C" {
int dblcg(dspmat*, dmat*, double, int, dmat*) { return INVALID_PARAMETERS; }
int dblbicgstab(dspmat*, dmat*, double, int, dmat*) { return INVALID_PARAMETERS; }
int dblbicgstabl(dspmat*, dmat*, int, double, int, dmat*) { return INVALID_PARAMETERS; }
int myqr(int, int, double*, double*) { return INVALID_PARAMETERS; }
}
