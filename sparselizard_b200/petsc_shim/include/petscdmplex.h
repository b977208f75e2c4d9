// Stand-in header: see slshim_petsc.h.
#include "slshim_petsc.h"
