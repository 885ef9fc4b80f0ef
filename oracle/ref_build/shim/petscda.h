/* oracle build stand-in: see petsc.h */
#include "petsc.h"
