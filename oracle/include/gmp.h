/* Stand-in for <gmp.h>: the image has the GMP runtime but no headers. */
#include "../mpfr_decls.h"
