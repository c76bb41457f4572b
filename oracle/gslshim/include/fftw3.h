/* FFTW is included by the reference headers but not called on the AAK waveform path; empty stand-in. */
#ifndef FFTW3_SHIM_H
#define FFTW3_SHIM_H
#endif
