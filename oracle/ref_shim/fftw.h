/* Empty stand-in for the FFTW2 header.
 * The reference includes <fftw.h> through ifftw.h but calls no FFTW routine
 * on the operator / solver / contraction path, so nothing is declared here. */
#ifndef ORACLE_SHIM_FFTW_H
#define ORACLE_SHIM_FFTW_H
#endif
