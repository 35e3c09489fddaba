/* Empty stand-in for the FFTW2 threads header (see fftw.h). */
#ifndef ORACLE_SHIM_FFTW_THREADS_H
#define ORACLE_SHIM_FFTW_THREADS_H
#endif
