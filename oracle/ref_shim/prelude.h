/*
 * Forced-include prelude for compiling the reference's own hot-path C
 * functions (oracle/Makefile, target "ref") without Chameleon, StarPU,
 * NLopt or GSL, none of which are installed here.
 *
 * The Makefile defines the include guards of the reference's Chameleon /
 * StarPU glue headers (include/common.h, include/descriptor.h,
 * include/chameleon_starpu.h) and of src/include/MLE.h, so their bodies are
 * skipped; the third-party system headers resolve to the empty files in
 * oracle/ref_shim/include.  What the remaining declarations in
 * misc/include/MLE_misc.h still need is declared here.
 */
#ifndef ORACLE_REF_PRELUDE_H
#define ORACLE_REF_PRELUDE_H
#include <stdint.h>
#include <time.h>

/* NLopt's optimizer handle, only named in prototypes of MLE_misc.h */
typedef void *nlopt_opt;

#endif
