/* Empty stand-in for MATLAB's blas.h: the reference mex files on the
 * layer-builder path include it but call no BLAS routine. */
