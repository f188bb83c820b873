/* b200fmm -- Blackwell (sm_100a) implementation of the ScalFMM interpolation-FMM hot path.
 *
 * C ABI: plain pointers and sizes, no CUDA/PyTorch types.  Every function returns a b200fmm_status and
 * never exits, traps or throws; b200fmm_last_error() gives the message of the last failure on the calling
 * thread.  A handle is used by one host thread at a time and owns (or borrows) one CUDA stream.
 *
 * Reference interfaces replaced (paths relative to the ScalFMM project root):
 *   - the kernel operator surface FAbstractKernels (Src/Components/FAbstractKernels.hpp:23-210):
 *     P2M :36, M2M :50, M2L :81-83 (+ finishedLevelM2L :93-102), L2L :116, L2P :124, P2P :147-150,
 *     P2POuter :171-174, P2PRemote :203-208 -- here level-batched: one call runs the operator over
 *     every cell/leaf of a level, as FFmmAlgorithmThread's passes do (Src/Core/FFmmAlgorithmThread.hpp);
 *   - the algorithm entry FAbstractAlgorithm::execute(operationsToProceed) (Src/Core/FCoreCommon.hpp:73-78)
 *     with the FFmmOperations bits (FCoreCommon.hpp:17-29);
 *   - the C API of Addons/CKernelApi (CScalfmmApi.h:103-802: scalfmm_init, scalfmm_tree_insert_particles_xyz,
 *     scalfmm_set_physical_values, scalfmm_execute_fmm, scalfmm_get_potentials/forces_xyz) and the
 *     Chebyshev extern "C" operators ChebKernel_P2M ... ChebKernel_P2PRemote (FChebInterface.h:37-76);
 *   - the M2L operator file I/O of FChebSymM2LHandler (ComputeAndCompressAndStoreInBinaryFile /
 *     ReadFromBinaryFile, Src/Kernels/Chebyshev/FChebSymM2LHandler.hpp:471-567).
 */
#ifndef B200FMM_H
#define B200FMM_H

#if defined(__GNUC__)
#define B200FMM_API __attribute__((visibility("default")))
#else
#define B200FMM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  B200FMM_OK = 0,
  B200FMM_ERR_INVALID = 1,     /* bad argument (null pointer, size, order/height out of range, ...) */
  B200FMM_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  B200FMM_ERR_OOM = 3,         /* device allocation failed */
  B200FMM_ERR_STATE = 4,       /* call out of order (e.g. execute before set_particles) */
  B200FMM_ERR_DOMAIN = 5,      /* particle outside the box, or a non-finite coordinate */
  B200FMM_ERR_UNSUPPORTED = 6, /* configuration not built into this library */
  B200FMM_ERR_NUMERIC = 7      /* operator precompute failed (SVD did not converge) */
} b200fmm_status;

/* Interpolation kernels (Src/Kernels/Chebyshev/FChebSymKernel.hpp, FChebDenseKernel.hpp,
 * Src/Kernels/Uniform/FUnifKernel.hpp), all for the Laplace 1/r matrix kernel FInterpMatrixKernelR. */
typedef enum { B200FMM_CHEB_SYM = 0, B200FMM_CHEB_DENSE = 1, B200FMM_LAGRANGE = 2 } b200fmm_kernel;

/* FP64: every operator in FP64 (parity form).  MIXED: P2P in FP32 with per-target compensated sums,
 * M2L as split-FP16 tensor-core GEMMs (tcgen05) with FP32 accumulation and FP64 cross-group sums --
 * for CHEB_SYM over the compressed operators in their low-rank form (Y = V^T M per source cell, then
 * U Y per target tile), for CHEB_DENSE / LAGRANGE over the dense per-transfer-vector operators;
 * P2M/M2M/L2L/L2P stay FP64. */
typedef enum { B200FMM_FP64 = 0, B200FMM_MIXED = 1 } b200fmm_precision;

/* FFmmOperations (FCoreCommon.hpp:17-29) */
enum {
  B200FMM_P2P = 1,
  B200FMM_P2M = 2,
  B200FMM_M2M = 4,
  B200FMM_M2L = 8,
  B200FMM_L2L = 16,
  B200FMM_L2P = 32,
  B200FMM_NEAR_FIELD = 1,
  B200FMM_FAR_FIELD = 62,
  B200FMM_ALL = 63
};

typedef struct {
  int kernel;        /* b200fmm_kernel */
  int order;         /* interpolation order p, 3..8 */
  int height;        /* octree height (levels 0..height-1, leaves at height-1), 3..12 */
  int nrhs;          /* charge vectors sharing one tree (the reference's NVALS), 1..32 */
  int precision;     /* b200fmm_precision */
  double box_width;  /* cubic simulation box (FOctree ctor, Src/Containers/FOctree.hpp:95) */
  double center[3];
  double epsilon;    /* M2L compression accuracy for CHEB_SYM; <= 0 selects 10^-order
                        (FChebSymKernel.hpp:136-140) */
  void *stream;      /* cudaStream_t to run on; NULL makes the handle create its own */
  int device;        /* CUDA device ordinal; -1 keeps the calling thread's current device */
} b200fmm_config;

typedef struct b200fmm_context *b200fmm_handle;

/* Lifecycle.  create() also builds the interpolation tables and, for CHEB_SYM, the 16 compressed
 * operators (own FP64 precompute on the GPU: kernel evaluation at the nodes, then pACA + QR + SVD,
 * following FChebSymM2LHandler.hpp:39-281); for CHEB_DENSE / LAGRANGE it evaluates the dense
 * per-transfer-vector operators on the GPU in FP64. */
B200FMM_API b200fmm_status b200fmm_create(const b200fmm_config *cfg, b200fmm_handle *out);
B200FMM_API b200fmm_status b200fmm_destroy(b200fmm_handle h);
B200FMM_API const char *b200fmm_last_error(void);
B200FMM_API const char *b200fmm_version(void);

/* Compressed operators in the reference's storage layout: ranks[343] (non-zero for the 16 class slots),
 * uv = for each class slot in increasing order U (p^3 x r, column-major) then V (p^3 x r, column-major).
 * set_ replaces the handle's operators (ReadFromBinaryFile equivalent), get_ exports them. */
B200FMM_API b200fmm_status b200fmm_set_sym_operators(b200fmm_handle h, const int *ranks, const double *uv, long long uv_len);
B200FMM_API b200fmm_status b200fmm_get_sym_operators(b200fmm_handle h, int *ranks, double *uv, long long uv_cap,
                                         long long *uv_len);

/* Insert particles (FOctree::insert + FP2PParticleContainerIndexed, Src/Containers/FOctree.hpp:174-181)
 * and build the tree on the GPU: Morton keys, stable radix sort, leaf ranges, upper levels, neighbour
 * and interaction lists.  x, y, z: n doubles; q: nrhs*n doubles ([rhs][particle]).  Pointers are host
 * memory when on_device == 0, device memory otherwise.  Resets all expansions and results. */
B200FMM_API b200fmm_status b200fmm_set_particles(b200fmm_handle h, long long n, const double *x, const double *y,
                                     const double *z, const double *q, int on_device);
/* Replace the charges only (same positions, same tree). */
B200FMM_API b200fmm_status b200fmm_set_charges(b200fmm_handle h, const double *q, int on_device);

/* Whole evaluation (FFmmAlgorithmThread::executeCore, FFmmAlgorithmThread.hpp:118-159): zeroes the
 * expansions and results, then runs the passes selected by ops.  The second execute() with the same ops on
 * one tree (after set_charges(), say) captures the passes into a CUDA graph, and later ones replay it with
 * a single launch; set_particles() drops it.  Environment B200FMM_GRAPHS=0 keeps every call on plain
 * launches.  A stream that the caller is capturing always gets plain launches. */
B200FMM_API b200fmm_status b200fmm_execute(b200fmm_handle h, unsigned ops);

/* Autotuner (MIXED), on the current tree; the choices are kept by the handle:
 *  - the tensor-core M2L's work split: 1, 2, 3 or 4 ranges of equal work per CTA (pair); returned in splits
 *    with its kernel time (ms).  Dense trees always run lockstep waves of whole tiles, so the choice matters
 *    for sparse trees;
 *  - the near field's work items: the largest leaf one warp takes whole (32, 64 or 128 targets) and the size
 *    of the pieces a larger leaf is cut into (16, 32 or 64 targets).
 * It runs the M2L and the near field several times and leaves the expansions and results undefined: call
 * execute() afterwards.  A no-op (splits = 0) in FP64.  The choices change how FP32 partial sums are grouped,
 * so results move within the MIXED tolerance. */
B200FMM_API b200fmm_status b200fmm_autotune(b200fmm_handle h, int *splits, double *ms);
/* The handle's current choices: values[0] M2L work ranges per CTA (pair), values[1] the largest leaf taken
 * whole by one warp of the near field, values[2] the targets per piece of a larger leaf. */
B200FMM_API b200fmm_status b200fmm_get_tuning(b200fmm_handle h, int *values);

/* Algorithmic FLOPs of one M2L pass over all levels of the current tree, for the form the handle runs:
 * dense operators 2 p^6 per interaction pair; compressed operators 2 p^3 r per pair for U Y plus, in MIXED,
 * 2 p^3 (sum of the fed slots' ranks) per source cell for Y = V^T M (FP64 recomputes V^T M per pair:
 * 4 p^3 r per pair).  Times the number of right-hand sides. */
B200FMM_API b200fmm_status b200fmm_m2l_flops(b200fmm_handle h, double *flops);

/* Level-batched operators (FAbstractKernels).  They accumulate (+=) like the reference kernels.
 * m2m/l2l take the parent level; m2l the level of the target cells (2..height-1). */
B200FMM_API b200fmm_status b200fmm_reset_expansions(b200fmm_handle h);
/* Zero the potentials and forces only (the containers' resetToInitialState for the particle outputs,
 * Src/Components/FBasicParticleContainer.hpp:449-460), keeping the expansions. */
B200FMM_API b200fmm_status b200fmm_zero_results(b200fmm_handle h);
B200FMM_API b200fmm_status b200fmm_p2m(b200fmm_handle h);
B200FMM_API b200fmm_status b200fmm_m2m(b200fmm_handle h, int level);
B200FMM_API b200fmm_status b200fmm_m2l(b200fmm_handle h, int level);
B200FMM_API b200fmm_status b200fmm_l2l(b200fmm_handle h, int level);
B200FMM_API b200fmm_status b200fmm_l2p(b200fmm_handle h);
/* variant 0: each leaf against itself and its <=26 neighbours (P2P with inTargets == inSources:
 * P2POuter + P2PInner, FChebSymKernel.hpp:453-478); variant 1: neighbours only (P2PRemote, :481-486). */
B200FMM_API b200fmm_status b200fmm_p2p(b200fmm_handle h, int variant);

/* Results in the caller's original particle order, [rhs][particle]; host memory unless on_device. */
B200FMM_API b200fmm_status b200fmm_get_results(b200fmm_handle h, double *phi, double *fx, double *fy, double *fz,
                                   int on_device);
/* The same into host memory without waiting (no counterpart in the reference): the results are staged on the
 * handle's stream and copied on a stream of their own, so the copies overlap what the caller queues next
 * (set_particles of the next step uploads and builds its tree meanwhile).  The host arrays hold the results
 * once b200fmm_synchronize() has returned; page-locked arrays make the copies asynchronous.  Any array may be
 * NULL.  A later call of this function waits on the device for the earlier copies before it stages again. */
B200FMM_API b200fmm_status b200fmm_get_results_async(b200fmm_handle h, double *phi, double *fx, double *fy,
                                                     double *fz);
/* Makes the handle's stream wait (on the device, without blocking the host) for the result copies queued by
 * b200fmm_get_results_async, so that work or events queued on that stream afterwards follow them. */
B200FMM_API b200fmm_status b200fmm_join_results(b200fmm_handle h);
/* Target shard (the reference's MPI algorithm gives each process a Morton interval of cells per level,
 * FFmmAlgorithmThreadProc.hpp:84-128, and exchanges the cells its neighbours need).  With count > 1, execute() evaluates only the particles of
 * shard `rank`: the leaves of a Morton range holding about N / count of the sorted particles (whole leaves).
 * Every other particle's results stay zero, so the sum over rank = 0 .. count-1 of the results is the whole
 * evaluation: count processes or GPUs holding the same particles each run one shard and add their results
 * (an all-reduce).  The near field, L2P and the M2L of the shard's cells and their ancestors are divided; the
 * tree, P2M, M2M and the low-rank M2L's first product are computed whole by every shard.  count = 1 (the
 * default) evaluates every particle.  Applies to execute() from the next call on, for every later tree. */
B200FMM_API b200fmm_status b200fmm_set_shard(b200fmm_handle h, int rank, int count);
/* Blocks until the handle's work and its result copies are done; reports a device-side failure. */
B200FMM_API b200fmm_status b200fmm_synchronize(b200fmm_handle h);

/* Tree inspection (host memory).  ncells: height entries.  get_cells returns the cells of one level in
 * Morton order: keys[ncells[level]], multipoles/locals [ncells][nrhs][p^3] (either may be NULL). */
B200FMM_API b200fmm_status b200fmm_tree_info(b200fmm_handle h, long long *ncells, long long *nparticles);
B200FMM_API b200fmm_status b200fmm_get_cells(b200fmm_handle h, int level, long long *keys, double *multipoles,
                                 double *locals);
/* The tree's lists (host memory), in the cell numbering of get_cells.
 * get_leaf_neighbors: nbr[nleaves*27], for each leaf the leaf at neighbour position ((dx+1)*3+(dy+1))*3+(dz+1)
 *   (FAbstractKernels.hpp:134-136; 13 = the leaf itself), -1 when that leaf is empty or outside the box -- the
 *   neighbours FOctree::getLeafsNeighbors returns (Src/Containers/FOctree.hpp:1364-1400).
 * get_interaction_lists: for one level (2..height-1), src[ncells*189] the source cell of each of a cell's 189
 *   interaction-list candidates and pos[ncells*189] its position ((dx+3)*7+(dy+3))*7+(dz+3), both -1 where that
 *   cell is empty or outside the box -- the far neighbours FOctree::getInteractionNeighbors returns
 *   (FOctree.hpp:914-975, FTreeCoordinate.hpp:219-264).  Either pointer may be NULL. */
B200FMM_API b200fmm_status b200fmm_get_leaf_neighbors(b200fmm_handle h, int *nbr);
/* start[nleaves+1]: the particles of leaf i are sorted positions start[i] .. start[i+1]-1 (get_permutation maps
 * them to the caller's order) -- the leaf containers of FOctree (FOctree.hpp:174-181). */
B200FMM_API b200fmm_status b200fmm_get_leaf_ranges(b200fmm_handle h, long long *start);
B200FMM_API b200fmm_status b200fmm_get_interaction_lists(b200fmm_handle h, int level, int *src, int *pos);
/* Sorted position -> original particle index. */
B200FMM_API b200fmm_status b200fmm_get_permutation(b200fmm_handle h, long long *perm);

/* Device time of the passes of the last execute(), milliseconds:
 * [0] tree build (last set_particles), [1] P2M, [2] M2M, [3] M2L, [4] L2L, [5] L2P, [6] P2P, [7] total.
 * When P2P runs together with P2M or M2M it runs on a second stream beside them, so [6] overlaps [1] and [2]
 * and [7] is less than their sum.  After an execute() that replayed a CUDA graph only [0] and [7] are
 * measured; [1]..[6] are 0. */
B200FMM_API b200fmm_status b200fmm_last_timings(b200fmm_handle h, double *ms8);
/* Device time of single kernels of the last execute(), milliseconds: [0] the M2L kernel (the tensor-core
 * kernel alone in MIXED, the whole M2L pass in FP64), [1] the P2P kernel, [2] P2M, [3] L2P (all 0 after a
 * graph replay). */
B200FMM_API b200fmm_status b200fmm_last_kernel_times(b200fmm_handle h, double *ms4);
/* Work counts of the current tree: M2L (target, source) pairs over levels 2..height-1 and ordered P2P
 * particle pairs (i != j) over each leaf and its neighbours. */
B200FMM_API b200fmm_status b200fmm_tree_stats(b200fmm_handle h, long long *m2l_pairs, long long *p2p_pairs);
/* Number of kernel launches issued by the last set_particles() plus the last execute(). */
B200FMM_API b200fmm_status b200fmm_last_launch_count(b200fmm_handle h, long long *count);

/* Allocation-free near field.  This entry point has no counterpart in the reference.  It is for callers
 * that cannot allocate device memory while this step runs: applications that hand all device memory to their
 * own pool up front (so a cudaMalloc inside a library fails or steals from the pool), and loops where
 * cudaMalloc's implicit device synchronisation is not acceptable.  It runs the MIXED-precision P2P of
 * b200fmm_p2p (variant 0 or 1) on caller-owned device arrays and calls no cudaMalloc, cudaFree or other
 * allocating routine: its scratch (the FP32 leaf-local copies of the particles) lives in a fixed 24 MiB device
 * array inside this library, which every GPU that loads the library holds until the process exits, so it
 * accepts at most B200FMM_NOALLOC_MAX_PARTICLES particles and returns B200FMM_ERR_INVALID above that.
 *   x, y, z, q: n particles sorted by leaf (FP64, device); leaf_keys[nleaves] Morton keys of the non-empty
 *   leaves in increasing order; leaf_start[nleaves+1] their particle ranges (leaf_start[0] = 0,
 *   leaf_start[nleaves] = n); leaf_nbr[nleaves*27] the leaf index of each neighbour position
 *   ((dx+1)*3+(dy+1))*3+(dz+1) (13 = the leaf itself), -1 when empty; phi, fx, fy, fz: n outputs (FP64,
 *   device) to which the near field is ADDED.  stream: cudaStream_t.
 * The leaf tables are checked on the device before anything is read through them; inconsistent tables
 * return B200FMM_ERR_INVALID and leave the outputs untouched.  The call blocks the calling thread: it reads
 * the result of that check back before the near field runs, and the status of the near field's bounded waits
 * before it returns.
 * The first call on a device looks up that array's device address (cudaGetSymbolAddress) with the device
 * current.  All calls share the one array and its status
 * words, and it keeps the last call's contents; calls whose executions overlap on the GPU race on it:
 * serialise them (one stream, or events). */
#define B200FMM_NOALLOC_MAX_PARTICLES 262144LL
B200FMM_API b200fmm_status b200fmm_p2p_noalloc(long long n, const double *x, const double *y, const double *z,
                                               const double *q, long long nleaves, const long long *leaf_keys,
                                               const long long *leaf_start, const int *leaf_nbr, int height,
                                               double box_width, const double *center, int variant, double *phi,
                                               double *fx, double *fy, double *fz, void *stream);

/* Batches of independent problems of uneven size, each with its own order, height and box (the reference
 * runs one FFmmAlgorithm per problem).  The problems are dealt to nstreams worker streams, each driven by
 * its own host thread, by estimated cost (largest first, each to the least loaded worker), so that one
 * problem's tree build overlaps other problems' passes; every worker keeps one handle per (order, height, box)
 * it has met, so operators are computed once and device buffers are reused by later calls.  The schedule
 * depends only on the problem list, so a repeated call with the same list allocates nothing.  Host memory in
 * and out; nrhs = 1.  execute() returns when every problem's results are written, or the first failure (its
 * message names the problem). */
typedef struct {
  long long n;                  /* particles */
  const double *x, *y, *z, *q;  /* n each */
  double *phi, *fx, *fy, *fz;   /* n each, written (not accumulated), caller's particle order */
  int order, height;
  double box_width, center[3];
} b200fmm_problem;
typedef struct b200fmm_batch_context *b200fmm_batch;
B200FMM_API b200fmm_status b200fmm_batch_create(int kernel, int precision, int nstreams, int device,
                                                b200fmm_batch *out);
B200FMM_API b200fmm_status b200fmm_batch_execute(b200fmm_batch b, int nproblems, const b200fmm_problem *problems);
/* Host wall time of the last batch_execute(), milliseconds. */
B200FMM_API b200fmm_status b200fmm_batch_last_time(b200fmm_batch b, double *ms);
/* Device time of the last batch_execute(), milliseconds: from an event recorded before the first problem to
 * the last worker stream's end (CUDA events), host gaps between a worker's problems included. */
B200FMM_API b200fmm_status b200fmm_batch_last_device_time(b200fmm_batch b, double *ms);
B200FMM_API b200fmm_status b200fmm_batch_destroy(b200fmm_batch b);

/* Particle files of ScalFMM's FFmaGenericLoader / FFmaGenericWriter (Src/Files/FFmaGenericLoader.hpp:189-477):
 * binary when the name contains ".bfma" (unsigned int {8, nvalues}, long long n, double half width, double
 * centre[3], then n records of nvalues doubles), text when it contains ".fma" (the same fields, whitespace
 * separated, one particle per line).  Records are x, y, z, q and, with 8 values, phi, fx, fy, fz.
 * fma_read fills n, nvalues, box_width (twice the stored half width) and centre, and, when data is not NULL, the
 * n * nvalues values (B200FMM_ERR_INVALID if cap is smaller); call it once with data = NULL to size the buffer.
 * Host memory only; no GPU is involved. */
B200FMM_API b200fmm_status b200fmm_fma_read(const char *path, long long *n, int *nvalues, double *box_width,
                                            double *center, double *data, long long cap);
B200FMM_API b200fmm_status b200fmm_fma_write(const char *path, long long n, int nvalues, double box_width,
                                             const double *center, const double *data);

/* FP64 direct sum on the GPU (Examples/DirectComputation.cpp:104-142) for the listed targets (all if
 * ntargets < 0).  Host pointers; outputs have ntargets (or n) entries. */
B200FMM_API b200fmm_status b200fmm_direct(long long n, const double *x, const double *y, const double *z, const double *q,
                              long long ntargets, const long long *targets, double *phi, double *fx,
                              double *fy, double *fz);

#ifdef __cplusplus
}
#endif
#endif
