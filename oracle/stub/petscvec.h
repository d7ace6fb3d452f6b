/* Stand-in: see petsc.h in this folder. */
#include "petsc.h"
