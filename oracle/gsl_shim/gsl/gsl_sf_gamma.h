/* TEST INFRASTRUCTURE ONLY: the GSL stand-in (gsl_shim.h). */
#include "gsl_shim.h"
