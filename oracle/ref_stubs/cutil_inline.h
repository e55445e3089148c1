/* Project-written empty stand-in for a retired CUDA SDK header (test oracle build only). */
#include "cutil.h"
