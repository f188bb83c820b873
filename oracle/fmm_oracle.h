/* CPU restatement of the ScalFMM (polatory fork, 1.5.2) FMM hot path, FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product and the "port" CPU
 * baseline; it is never linked into, loaded by, or called from the product path.
 *
 * Every function restates one reference routine; the citing comment names the file:line it follows
 * (paths relative to the reference project root).  Layout conventions match the reference:
 *   - node index n = nx + p*ny + p*p*nz  (FInterpTensor::setNodeIds, FInterpTensor.hpp:54-61)
 *   - Morton keys interleave x,y,z with x the most significant bit of each triple
 *     (FTreeCoordinate::getMortonIndex, FTreeCoordinate.hpp:91-113)
 *   - transfer-vector slot t = ((dx+3)*7 + (dy+3))*7 + (dz+3) (FTreeCoordinate.hpp:251)
 */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_CHEB_SYM = 0, ORC_CHEB_DENSE = 1, ORC_LAGRANGE = 2 };

/* operation bits, FCoreCommon.hpp:17-29 */
enum { ORC_P2P = 1, ORC_P2M = 2, ORC_M2M = 4, ORC_M2L = 8, ORC_L2L = 16, ORC_L2P = 32 };

typedef struct {
  int kind;         /* ORC_CHEB_SYM | ORC_CHEB_DENSE | ORC_LAGRANGE */
  int order;        /* interpolation order p (2..10) */
  int height;       /* octree height; leaves live at level height-1 */
  int nrhs;         /* number of charge vectors sharing the positions */
  int nthreads;
  double box_width;
  double center[3];
  /* ORC_CHEB_SYM: compressed operators of the 16 symmetry classes, indexed by slot t in 0..342.
   * ranks[t] > 0 only for the 16 class slots; uv holds, for each such slot in increasing t,
   * U (p^3 x r, column-major) then V (p^3 x r, column-major), exactly the reference's K[t]
   * (FChebSymM2LHandler.hpp:183-203). */
  const int *sym_ranks;
  const double *sym_uv;
} orc_config;

/* Optional dump of all expansions: cells ordered by level then Morton key. */
typedef struct {
  long long cap;      /* capacity in cells */
  long long count;    /* number of cells written (all levels 0..height-1 that hold particles) */
  int *levels;
  long long *mortons;
  double *multipoles; /* [cap][nrhs][p^3] */
  double *locals;     /* [cap][nrhs][p^3] */
} orc_dump;

/* Full FMM evaluation (FFmmAlgorithm::execute, FFmmAlgorithm.hpp / FFmmAlgorithmThread.hpp:118-159).
 * q, phi, fx, fy, fz are [nrhs][n] in the caller's particle order; outputs are overwritten. */
int orc_fmm(const orc_config *cfg, long long n, const double *x, const double *y, const double *z,
            const double *q, unsigned ops, double *phi, double *fx, double *fy, double *fz, orc_dump *dump);

/* FP64 direct sum (Examples/DirectComputation.cpp:104-142) for the listed targets (all if ntargets<0). */
int orc_direct(long long n, const double *x, const double *y, const double *z, const double *q,
               long long ntargets, const long long *targets, int nthreads,
               double *phi, double *fx, double *fy, double *fz);

/* Leaf coordinates + Morton keys of particles (FCoordinateComputer.hpp:16-40, FTreeCoordinate.hpp:91-113). */
int orc_morton_keys(long long n, const double *x, const double *y, const double *z, double box_width,
                    const double *center, int height, long long *keys);

/* Morton encode/decode of one coordinate triple. */
long long orc_morton_encode(int ix, int iy, int iz);
void orc_morton_decode(long long key, int *ix, int *iy, int *iz);

/* Symmetry tables (FInterpSymmetries.hpp:18-125): pindices[343], pvectors[343][p^3]. */
int orc_sym_tables(int order, unsigned *pindices, unsigned *pvectors);

/* Chebyshev roots in ascending order (FChebRoots.hpp:27-80). */
void orc_cheb_roots(int order, double *roots);

/* Leaf neighbour list (FTreeCoordinate::getNeighborsIndexes, FTreeCoordinate.hpp:189-216):
 * returns count; keys[26] and positions[26] ((dx+1)*3+(dy+1))*3+(dz+1). */
int orc_leaf_neighbors(int ix, int iy, int iz, int height, long long *keys, int *positions);

/* Interaction list (FTreeCoordinate::getInteractionNeighbors, FTreeCoordinate.hpp:219-264). */
int orc_interaction_list(int ix, int iy, int iz, int level, long long *keys, int *positions);

#ifdef __cplusplus
}
#endif
#endif
