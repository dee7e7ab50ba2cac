/* Oracle shim: forwards to the single-rank stand-ins. */
#include "shim_trilinos.h"
