/* oracle build stand-in: PC internals used by src/omg/omg.C (setupcalled) */
#include "petsc.h"
