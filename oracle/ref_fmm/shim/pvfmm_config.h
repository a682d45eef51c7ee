/* Configuration of the reference build that pins the oracle (single rank, no
 * CUDA, no FFTW: the reference's own matrix DFT in include/fft_wrapper.hpp
 * runs; BLAS/LAPACK come through the SCTL stand-in).  PVFMM_EXTENDED_BC as
 * in the reference's CMakeLists.txt default. */
#ifndef PVFMM_REF_CONFIG_H
#define PVFMM_REF_CONFIG_H
#define PVFMM_HAVE_SYS_STAT_H
#define PVFMM_EXTENDED_BC
#define PVFMM_PRECOMP_DATA_PATH ""
#endif
