/* Empty stand-in for <cblas.h>: the reference functions compiled into oracle/_ref
 * use none of its declarations (see oracle/ref_shim/prelude.h). */
