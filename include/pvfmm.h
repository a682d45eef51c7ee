/*
 * pvfmm.h -- C interface of the B200 particle-FMM library (libpvfmm_b200.so).
 *
 * The particle entry points keep the names, argument meaning and layouts of
 * the reference C interface (dmalhotra/pvfmm include/pvfmm.h:238-303), so a
 * caller of the reference links against this library unchanged:
 *
 *   positions  AoS [x1 y1 z1 x2 y2 z2 ...]
 *   densities  [q1 ... qn] (k0 values per point: 1 for Laplace, 3 for Stokes)
 *   outputs    n_trg x k1 values, overwritten (not accumulated)
 *
 * Boundaries: box_size <= 0 is free space: the points are mapped into the
 * unit box with the reference's bounding-box rule and densities and outputs
 * are rescaled by the kernel's scale exponents (src/pvfmm-wrapper.cpp:458-541,
 * 800-808).  box_size > 0 is periodic with period box_size in x, y and z
 * (src/pvfmm-wrapper.cpp:397-404, 512-517): the points are scaled by
 * 1/box_size and wrapped into the unit cube, the interaction lists wrap
 * around it, and the images beyond the root's 3x3x3 block enter through the
 * boundary operator of the reference's default build (PVFMM_EXTENDED_BC: the
 * images of the 5x5x5 block; PVFMMSetPeriodicBC selects the lattice sum over
 * all images or adds a user operator).
 *
 * Errors: the reference signatures return void.  On failure an evaluation
 * fills trg_val with NaN and records a message for PVFMMGetLastError().
 *
 * Threading: one CUDA stream per context; contexts are independent; calls on
 * one context must not overlap.
 */
#ifndef PVFMM_B200_PVFMM_H_
#define PVFMM_B200_PVFMM_H_

#include <stdint.h>

#include "pvfmm_mpi_stub.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel functions; values 0-5 as in the reference (include/pvfmm.h:21-28),
 * all implemented, plus the extension LaplacePotGrad (potential and -grad in
 * one pass, 4 outputs). */
enum PVFMMKernel {
  PVFMMLaplacePotential    = 0,
  PVFMMLaplaceGradient     = 1,
  PVFMMStokesPressure      = 2,
  PVFMMStokesVelocity      = 3,
  PVFMMStokesVelocityGrad  = 4,
  PVFMMBiotSavartPotential = 5,
  PVFMMLaplacePotGrad      = 6   /* extension: no reference counterpart */
};

/* ---------------------------------------------------------------------------
 * Reference entry points (include/pvfmm.h:254-301 of the reference).
 * ------------------------------------------------------------------------- */

/* Replaces PVFMMCreateContextD/F (reference include/pvfmm.h:254-255,
 * src/pvfmm-wrapper.cpp:385-443): builds the translation operators (FP64 on
 * the host) for kernel `kernel`, multipole order `m` (even, 2..16) and at most
 * `n` points per leaf.  `comm` must be a single-rank communicator.  The D
 * context evaluates in FP64 ("plain" form); the F context evaluates in the
 * mixed form (see PVFMMPrecisionMixed). */
void* PVFMMCreateContextD(double box_size, int n, int m, enum PVFMMKernel kernel, MPI_Comm comm);
void* PVFMMCreateContextF(float box_size, int n, int m, enum PVFMMKernel kernel, MPI_Comm comm);

/* Replaces PVFMMCreateContextDWorld/FWorld (reference include/pvfmm.h:256-257). */
void* PVFMMCreateContextDWorld(double box_size, int n, int m, enum PVFMMKernel kernel);
void* PVFMMCreateContextFWorld(float box_size, int n, int m, enum PVFMMKernel kernel);

/* Replaces PVFMMEvalD/F (reference include/pvfmm.h:290-291,
 * src/pvfmm-wrapper.cpp:445-811).  Host pointers.  setup=1 rebuilds the tree
 * for new positions; setup=0 reuses it (same positions, new densities, the
 * same of sl_den / dl_den passed as at setup).
 *
 * sl_den: single-layer densities (k0 per source) or NULL.
 * dl_den: double-layer values (k0 + 3 per source) or NULL; only the
 * LaplacePotential and StokesVelocity kernels have double-layer kernels (any
 * other kernel with dl_den is an error).  The values are used as the
 * reference uses them: the first k0 are scaled like densities (times scale_x
 * of the bounding-box map), the last three are not, and the kernels read
 * them in the reference's order -- Laplace (kernel.txx:1299-1311) takes
 * values 0-2 as the normal and value 3 as the density; Stokes
 * (kernel.txx:1437-1456) takes values 0-2 as the density f and 3-5 as the
 * normal n, with n.f formed as v0 v3 + v1 v1 + v2 v2.  Passing both
 * densities counts every source twice in the leaf-size rule, as the
 * reference does (fmm_node.txx:81-92). */
void PVFMMEvalD(const double* src_pos, const double* sl_den, const double* dl_den, long n_src,
                const double* trg_pos, double* trg_val, long n_trg, const void* ctx, int setup);
void PVFMMEvalF(const float* src_pos, const float* sl_den, const float* dl_den, long n_src,
                const float* trg_pos, float* trg_val, long n_trg, const void* ctx, int setup);

/* Replaces PVFMMDestroyContextD/F (reference include/pvfmm.h:299-300):
 * releases the context and sets *ctx to NULL. */
void PVFMMDestroyContextD(void** ctx);
void PVFMMDestroyContextF(void** ctx);

/* Replace the Fortran bindings pvfmmcreatecontextd_/f_, pvfmmevald_/f_ and
 * pvfmmdestroycontextd_/f_ (reference src/pvfmm-wrapper.cpp:831-875): the same
 * functions with every argument passed by reference, 32-bit integers for the
 * leaf size, order, kernel and setup flag, 64-bit point counts, and the
 * communicator as a Fortran handle, which must denote a single rank. */
void pvfmmcreatecontextd_(void** ctx, double* box_size, int32_t* n, int32_t* m, int32_t* kernel, int32_t* fcomm);
void pvfmmcreatecontextf_(void** ctx, float* box_size, int32_t* n, int32_t* m, int32_t* kernel, int32_t* fcomm);
void pvfmmevald_(const double* src_pos, const double* sl_den, int64_t* n_src, const double* trg_pos, double* trg_val,
                 int64_t* n_trg, void** ctx, int32_t* setup);
void pvfmmevalf_(const float* src_pos, const float* sl_den, int64_t* n_src, const float* trg_pos, float* trg_val,
                 int64_t* n_trg, void** ctx, int32_t* setup);
void pvfmmdestroycontextd_(void** ctx);
void pvfmmdestroycontextf_(void** ctx);

/* ---------------------------------------------------------------------------
 * Extensions (no counterpart in the reference).
 * ------------------------------------------------------------------------- */

enum PVFMMPrecision {
  PVFMMPrecisionPlain = 0,   /* FP64 everywhere */
  PVFMMPrecisionMixed = 1    /* FP32 near field (U and W lists: rsqrt + one
                                Newton step, hi+lo coordinates, partial sums
                                promoted to FP64 every 16 sources), FP32
                                V-list DFTs, V-list products on the tensor
                                cores as 3-term split TF32; FP64 for the
                                check-to-equivalent chain (S2U and X check
                                potentials, pseudo-inverse GEMMs, U2U, D2D,
                                D2T evaluation) */
};

/* Context on double-precision inputs with an explicit precision form, so the
 * plain and the mixed form can run on the same FP64 inputs. */
void* PVFMMCreateContextExD(double box_size, int n, int m, enum PVFMMKernel kernel, int precision);

/* Boundary operator of a periodic context (box_size > 0), replacing
 * FMM_Pts::SetM2C and the reference's build option PVFMM_EXTENDED_BC
 * (include/fmm_pts.txx:790-1232, 2642-2686):
 *   lattice 0 (the default): the images in the 5x5x5 block around the root
 *     outside its 3x3x3 block (the reference built with PVFMM_EXTENDED_BC, its
 *     CMake default), plus m2c when not NULL: an (ns*k0) x (ns*k1) row-major
 *     operator from the root's upward equivalent density to its downward
 *     check potential, ns = 6(m-1)^2+2, added as SetM2C's operator is;
 *   lattice 1: the lattice sum over all images (the reference built without
 *     that option: zero-average projections, the unit volume potential's far
 *     field and the corner correction; for LaplacePotential and
 *     StokesVelocity the potential of the mean density is taken out of the
 *     outputs); LaplacePotential, LaplaceGradient and StokesVelocity only,
 *     m2c must be NULL.  With PVFMM_DIR set, the lattice operator is kept in
 *     PVFMM_DIR/Precomp_<kernel name>_m<m>_lattice_bc.data (int rows, int
 *     cols, FP64 values) and read back by later contexts.
 * Returns 0, or -1 (message in PVFMMGetLastError()) for a free-space context,
 * an unsupported kernel or bad arguments. */
int PVFMMSetPeriodicBC(void* ctx, int lattice, const double* m2c);

/* Periodic axes of a periodic context (the reference's BoundaryType PX, PXY
 * and PXYZ == Periodic, include/mpi_tree.hpp:23-30, which its C++ interface
 * selects in PtFMM_CreateTree): 1 = x, 3 = x and y, 7 = x, y and z (the
 * default, the only one the C interface's box_size gives).  Along the other
 * axes the unit cube is free space.  The next evaluation rebuilds the tree.
 * Returns 0, or -1 (message in PVFMMGetLastError()) for a free-space context
 * or another mask. */
int PVFMMSetPeriodicAxes(void* ctx, int axes);

/* Evaluation on device pointers (CUDA global memory).  The work is ordered
 * after the work already queued on `stream` (a cudaStream_t) and `stream`
 * waits for its completion; with NULL it is ordered after the legacy default
 * stream and the call returns when the values are written.  Returns 0 on
 * success, nonzero on error (message in PVFMMGetLastError()). */
int PVFMMEvalDeviceD(const void* ctx, const double* src_pos, const double* sl_den, long n_src,
                     const double* trg_pos, double* trg_val, long n_trg, int setup, void* stream);
int PVFMMEvalDeviceF(const void* ctx, const float* src_pos, const float* sl_den, long n_src,
                     const float* trg_pos, float* trg_val, long n_trg, int setup, void* stream);

/* PVFMMEvalDeviceD/F with double-layer values as well (dl_den as in
 * PVFMMEvalD; either density may be NULL). */
int PVFMMEvalLayersDeviceD(const void* ctx, const double* src_pos, const double* sl_den, const double* dl_den,
                           long n_src, const double* trg_pos, double* trg_val, long n_trg, int setup, void* stream);
int PVFMMEvalLayersDeviceF(const void* ctx, const float* src_pos, const float* sl_den, const float* dl_den,
                           long n_src, const float* trg_pos, float* trg_val, long n_trg, int setup, void* stream);

/* Evaluation with the roles of sources and targets exchanged (for adjoints and
 * gradients; no counterpart in the reference):
 *   src_val[j*k1+k] = sum_i K_k(src_j - trg_i) trg_den[i*k0 ...],
 * i.e. densities at the targets, values at the sources, with ctx's kernel.
 * For LaplacePotential (a symmetric kernel) this is the transpose of the
 * forward map; with LaplacePotGrad the last three values are the -gradient
 * that position derivatives need.  When src_pos == trg_pos (same array and
 * count) ctx's own tree is used, and setup=0 reuses the tree of the last
 * forward evaluation; otherwise a companion context with the same kernel,
 * order, leaf size and precision holds the exchanged tree (setup=0 reuses
 * it).  Device pointers, ordered after `stream`.  Returns 0 on success. */
int PVFMMEvalAdjointDeviceD(const void* ctx, const double* src_pos, long n_src, const double* trg_pos,
                            const double* trg_den, long n_trg, double* src_val, int setup, void* stream);
int PVFMMEvalAdjointDeviceF(const void* ctx, const float* src_pos, long n_src, const float* trg_pos,
                            const float* trg_den, long n_trg, float* src_val, int setup, void* stream);

/* Replaces Kernel<T>::ker_poten (reference include/kernel.hpp:40-41,
 * include/kernel.txx:1137-1265): FP64 direct evaluation on the device of the
 * kernel function, trg_val[t*k1+k] += sum_s K_k(trg_t - src_s) den_s, r == 0
 * excluded, for every source.  Device pointers, on `stream` (NULL: legacy
 * default stream).  Uses stream-ordered scratch of n_chunks*n_trg*k1 doubles.
 * Returns 0 on success. */
int PVFMMKernelEvalDeviceD(enum PVFMMKernel kernel, const double* src_pos, const double* den, long n_src,
                           const double* trg_pos, double* trg_val, long n_trg, void* stream);

/* Host-pointer form of PVFMMKernelEvalDeviceD with the calling convention of
 * Kernel<T>::ker_poten (reference include/kernel.hpp:40-41): copies the
 * arrays to the current device, evaluates there and adds the result into
 * trg_val.  Returns 0 on success. */
int PVFMMKernelEvalD(enum PVFMMKernel kernel, const double* src_pos, const double* den, long n_src,
                     const double* trg_pos, double* trg_val, long n_trg);

/* Allocation-free form of PVFMMKernelEvalDeviceD, for callers that cannot
 * allocate device memory at the call (a host framework that owns the device
 * memory pool, or a loop that must not pay for an allocation).  No
 * counterpart in the reference.  The partial sums use a fixed 8 MiB array in
 * the library's device image instead of allocated scratch, so
 * n_trg * k1 <= 1048576 (larger requests return an error).  The first call on
 * a device looks up the array's address and keeps it for the life of the
 * process (it is stale after cudaDeviceReset); make that call before any
 * stream capture.
 * All calls share the array: calls that overlap on the GPU race, and the
 * caller must serialise them.  Returns 0 on success. */
int PVFMMKernelEvalDeviceNoAllocD(enum PVFMMKernel kernel, const double* src_pos, const double* den, long n_src,
                                  const double* trg_pos, double* trg_val, long n_trg, void* stream);

/* Unit-box mode (on != 0), the tree rule of the reference C++ interface
 * (include/pvfmm.txx:216-244, PtFMM_CreateTree): coordinates are used as given
 * and must lie in [0,1)^3 (no bounding-box rescale), and the tree's point set
 * is the targets instead of the seed grid of PVFMMCreateContext
 * (src/pvfmm-wrapper.cpp:416-432).  The next evaluation rebuilds the tree.
 * Returns 0 on success. */
int PVFMMSetUnitBox(void* ctx, int on);

/* Layer-points mode (on != 0), for the reference C++ interface's separate
 * single- and double-layer point sets (include/pvfmm.txx:216-244: src_coord
 * and surf_coord both count in the leaf-size rule): the source points passed
 * are the two sets concatenated, each carrying its own layer's values and
 * zeros for the other, and every source point counts once in the tree.  The
 * next evaluation rebuilds the tree.  Returns 0 on success. */
int PVFMMSetLayerPoints(void* ctx, int on);

/* Last error message of the calling thread ("" if none). */
const char* PVFMMGetLastError(void);

/* Device time in milliseconds of the stages of the last evaluation on ctx, in
 * the order of the reference profile tags: 0 setup (tree + lists),
 * 1 S2U, 2 U2U, 3 V-list FFT, 4 V-list Hadamard, 5 V-list IFFT, 6 X-list,
 * 7 D2D, 8 D2T+W+U (D2T pseudo-inverse GEMMs and the fused near field),
 * 9 total, 10 the near-field kernel alone, 11 the D2T GEMMs alone.  Returns
 * the number written. */
int PVFMMGetStageTimes(const void* ctx, double* ms, int n);

/* Number of this library's own CUDA kernels launched on ctx since its
 * creation (library calls such as cuBLAS GEMMs and CUB sorts not counted). */
long PVFMMGetLaunchCount(const void* ctx);

/* Tree and evaluation introspection for parity tests.  `what`:
 *   0: number of nodes            1: tree depth
 *   2: node Morton coordinates (x, y, z, depth) as 4 x int64 per node
 *   3: node flags (is_leaf) as int64     4: src ranges (lo, hi) x int64
 *   5: trg ranges (lo, hi) x int64        6: parent index x int64
 *   7: upward equivalent densities (n_nodes x ns*k0, double)
 *   8: downward check potentials   (n_nodes x ns*k1, double)
 *   9: source permutation (sorted -> input index) x int64
 *  10: target permutation x int64
 *  11: 19 doubles of tree/list statistics: n_nodes, depth, n_sleaf, n_tleaf,
 *      n_vsrc, n_vtrg, n_xtrg, list entries (p2p, x, w), pair counts (p2p,
 *      x, w, d2t, s2u), n_leaves, n_src, n_trg, V-list (target parent,
 *      offset) pairs
 * Copies at most `n` elements into out and returns the element count needed. */
long PVFMMGetTreeData(const void* ctx, int what, void* out, long n);

/* Host precompute of one operator (FP64 row-major), for tests; every
 * PVFMMKernel value, including Stokes pressure, Stokes velocity gradient and
 * Biot-Savart, whose evaluation is not implemented (their expansions use the
 * kernel itself, so with kin source and kout target dims the check ->
 * equivalent factors are (ns*kout) x r and r x (ns*kin), r = ns*min(kin, kout)).
 * `which`:
 * 0 UC2UE0, 1 UC2UE1, 2 DC2DE0, 3 DC2DE1, 4 U2U (8 stacked, child-major rows),
 * 5 D2D (8 stacked, child-major columns), 6 unit surface (ns x 3),
 * 7 V-list Hadamard operators (complex, [f][offset 26][j1 8][j2 8][k0][k1]),
 * 8 projector onto the upward equivalent directions above the FP32 cutoff,
 * 9 periodic boundary operator ((ns*kin) x (ns*kout): root upward
 * equivalent density -> root downward check potential of the periodic images
 * outside the root's 3x3x3 block; BC_Type of BoundaryType Periodic,
 * include/fmm_pts.txx:790-1232) as the reference's default build forms it
 * (PVFMM_EXTENDED_BC: the images of the 5x5x5 block), 10 the same operator
 * as the lattice sum over all images (the reference built without that
 * option; Laplace potential / gradient and Stokes velocity only).  Precision
 * is ignored for both.
 * Returns the element count needed (copies at most n).
 *
 * Operator cache (contexts and this function alike): when the environment
 * variable PVFMM_DIR names a directory, the pseudo-inverse factors (the SVD
 * part of the precompute) are read from PVFMM_DIR/Precomp_<kernel name>_m<m>.data
 * if it exists and written there otherwise, in the layout of the reference's
 * precompute files (include/precomp_mat.txx:213-345, file name
 * include/fmm_pts.txx:246-276): entry 0 of matrix types 0-3 (UC2UE0, UC2UE1,
 * DC2DE0, DC2DE1, FP64 cutoff); other entries are skipped on reading and left
 * empty on writing.  Operators built from the cache equal the computed ones.
 * A file that exists but is not a usable cache is an error; a directory that
 * cannot be written is skipped.  Without PVFMM_DIR no file is touched. */
long PVFMMPrecompOperator(enum PVFMMKernel kernel, int m, int precision, int which, double* out, long n);

#ifdef __cplusplus
}
#endif

#endif /* PVFMM_B200_PVFMM_H_ */
