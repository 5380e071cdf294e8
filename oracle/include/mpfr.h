/* Stand-in for <mpfr.h>: the image has the MPFR runtime but no headers. */
#include "../mpfr_decls.h"
