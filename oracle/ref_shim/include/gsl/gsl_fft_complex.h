/* Empty stand-in for <gsl/gsl_fft_complex.h>: the reference functions compiled into oracle/_ref
 * use none of its declarations (see oracle/ref_shim/prelude.h). */
