/* Configuration of the reference build that pins the oracle (single rank, no
 * CUDA, no FFTW: the reference's own matrix DFT in include/fft_wrapper.hpp
 * runs; BLAS/LAPACK come through the SCTL stand-in).  PVFMM_EXTENDED_BC as
 * in the reference's CMakeLists.txt default; off (PVFMM_REF_LATTICE_BC) in the
 * second library that pins the periodic lattice sum. */
#ifndef PVFMM_REF_CONFIG_H
#define PVFMM_REF_CONFIG_H
#define PVFMM_HAVE_SYS_STAT_H
#ifndef PVFMM_REF_LATTICE_BC  /* the periodic lattice-sum variant, built as a separate library */
#define PVFMM_EXTENDED_BC
#endif
#define PVFMM_PRECOMP_DATA_PATH ""
#endif
