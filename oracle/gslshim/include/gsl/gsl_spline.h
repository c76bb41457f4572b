/* forwards to the project-written GSL subset shim (test infrastructure) */
#include "gslshim.h"
