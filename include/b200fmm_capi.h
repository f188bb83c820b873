/* b200fmm_capi -- the C user API of ScalFMM (Addons/CKernelApi/Src/CScalfmmApi.h) over the b200fmm library.
 *
 * An existing C caller of ScalFMM's built-in interpolation kernels switches over by compiling against this
 * header instead of CScalfmmApi.h and linking libb200fmm.so: the function names, argument lists, enums and
 * descriptor structs are the reference's (CScalfmmApi.h:47-886), so the caller's code is unchanged.  Every
 * call forwards to one b200fmm handle (include/b200fmm.h):
 *   scalfmm_init (CScalfmmApi.h:103) + scalfmm_build_tree (:259)       -> b200fmm_create
 *   scalfmm_tree_insert_particles[_xyz] (:317, :324), set_positions,    -> host copies, then b200fmm_set_particles
 *     add_to_positions, update_tree (:402-467)                               at the next execute
 *   scalfmm_set_physical_values[_npart] (:339-365)                      -> b200fmm_set_charges at the next execute
 *   scalfmm_execute_fmm[_far_field] (:738, :745)                        -> b200fmm_execute(ALL or far field)
 *   scalfmm_get_potentials / get_forces[_xyz][_npart] (:383-423)        -> b200fmm_get_results, accumulated
 *   scalfmm_get_timers / get_nb_timers (:790-802)                       -> b200fmm_last_timings
 * Semantics kept from the reference:
 *   - particles are numbered in insertion order, and every get/set takes or returns values in that order
 *     (or in the order of the idxOfParticles list for the _npart variants);
 *   - potentials and forces start at 0 after insertion, and each execute ADDS the computed field to them, as
 *     the reference's particle containers do (FP2PParticleContainer, "+="); set_potentials / set_forces
 *     overwrite them;
 *   - kernels: chebyshev is FChebSymKernel at order 7 over FInterpMatrixKernelR (FScalfmmApiInit.cpp:44);
 *     lagrange (FUnifKernel at order 7), which the reference's C API leaves commented out, runs the same way;
 *   - sequential and multi_thread algorithms give the same results (one GPU either way).
 * Differences, because the reference's behaviour there is to abort the process:
 *   - no call exits: a failure prints one line on stderr and is kept in b200fmm_last_error();
 *     b200fmm_capi_status() returns the status of the handle's last failing call (0 when all went well);
 *   - user_defined_kernel (callbacks per operator), the periodic, source_target and adaptive algorithms,
 *     set_upper_limit > 2 and the MPI partitioning calls are not part of this library: init returns NULL for
 *     user_defined_kernel, the others report B200FMM_ERR_UNSUPPORTED.
 * Extensions (not in the reference): b200fmm_capi_set_precision selects FP64 (default, the parity form) or
 * MIXED before build_tree; b200fmm_capi_status.
 */
#ifndef B200FMM_CAPI_H
#define B200FMM_CAPI_H

#include "b200fmm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef long long int FSize;

typedef enum kernel_type { user_defined_kernel = 0, chebyshev = 1, lagrange = 2 } scalfmm_kernel_type;

typedef enum scalfmm_algorithm_config {
  sequential = 0,
  multi_thread = 1,
  periodic = 2,
  source_target = 3,
  adaptiv = 4,
  mpi = 5
} scalfmm_algorithm;

typedef void *scalfmm_handle;

typedef enum particule_type { SOURCE = 0, TARGET = 1, BOTH = 2 } PartType;

/* Cell and leaf callbacks of user-defined kernels (CScalfmmApi.h:114-190).  The built-in kernels ignore them;
 * they are declared so that callers written against the reference compile unchanged. */
typedef void *(*Callback_init_cell)(int level, long long morton_index, int *tree_position, double *spatial_position,
                                    void *inDatas);
typedef void (*Callback_free_cell)(void *);
typedef FSize (*Callback_get_cell_size)(int level, long long morton_index, void *userData);
typedef void (*Callback_copy_cell)(void *userDatas, FSize size, void *memoryAllocated);
typedef FSize (*Callback_get_leaf_size)(FSize nbParts);
typedef void (*Callback_copy_leaf)(FSize nbParts, void *userDatas, void *memAllocated);
typedef void *(*Callback_restore_leaf)(FSize nbParts, void *memAllocated);
typedef void (*Callback_apply_on_leaf)(int level, FSize nbParts, const FSize *idxParts, long long morton_index,
                                       double llc[3], void *cellDatas, void *leafDatas, void *userDatas);
typedef void *(*Callback_init_leaf)(int level, FSize nbParts, const FSize *idxParts, long long morton_index,
                                    double llc[3], void *cellDatas, void *userDatas);
typedef void (*Callback_free_leaf)(void *cellDatas, FSize nbParts, const FSize *idxParts, void *leafData,
                                   void *userDatas);
typedef void *(*Callback_restore_cell)(int level, void *arrayTobeRead);

typedef struct User_Scalfmm_Cell_Descriptor {
  Callback_free_cell user_free_cell;
  Callback_init_cell user_init_cell;
  Callback_get_cell_size user_get_size;
  Callback_copy_cell user_copy_cell;
  Callback_restore_cell user_restore_cell;
} Scalfmm_Cell_Descriptor;

typedef struct User_Scalfmm_Leaf_Descriptor {
  Callback_init_leaf user_init_leaf;
  Callback_free_leaf user_free_leaf;
  Callback_get_leaf_size user_get_size;
  Callback_copy_leaf user_copy_leaf;
  Callback_restore_leaf user_restore_leaf;
} Scalfmm_Leaf_Descriptor;

/* Operator callbacks of user-defined kernels (CScalfmmApi.h:510-696). */
typedef void (*Callback_P2M)(void *cellData, void *leafData, FSize nbParticles, const FSize *particleIndexes,
                             void *userData);
typedef void (*Callback_M2M)(int level, void *parentCell, int childPosition, void *childCell, void *userData);
typedef void (*Callback_M2M_Full)(int level, void *parentCell, void *childCell[8], void *userData);
typedef void (*Callback_M2L)(int level, void *targetCell, int sourceCellPosition, void *sourceCell, void *userData);
typedef void (*Callback_M2L_Ext)(int level, void *targetCell, void *sourceCell, int tranfer[3], void *userData);
typedef void (*Callback_M2LFull)(int level, void *targetCell, const int *neighborPosition, const int size,
                                 void **sourceCell, void *userData);
typedef void (*Callback_L2L)(int level, void *parentCell, int childPosition, void *childCell, void *userData);
typedef void (*Callback_L2L_Full)(int level, void *parentCell, void *childCell[8], void *userData);
typedef void (*Callback_L2P)(void *cellData, void *leafData, FSize nbParticles, const FSize *particleIndexes,
                             void *userData);
typedef void (*Callback_P2P)(void *targetLeaf, FSize nbParticles, const FSize *particleIndexes, void *sourceLeaf,
                             FSize nbSourceParticles, const FSize *sourceParticleIndexes, void *userData);
typedef void (*Callback_P2PFull)(void *targetLeaf, FSize nbParticles, const FSize *particleIndexes,
                                 void **sourceLeaves, const FSize **sourceParticleIndexes, FSize *sourceNbPart,
                                 const int *sourcePosition, const int size, void *userData);
typedef void (*Callback_P2PInner)(void *targetLeaf, FSize nbParticles, const FSize *particleIndexes, void *userData);
typedef void (*Callback_P2PSym)(void *targetLeaf, FSize nbParticles, const FSize *particleIndexes, void *sourceLeaf,
                                FSize nbSourceParticles, const FSize *sourceParticleIndexes, void *userData);
typedef void (*Callback_P2PRemote)(void *targetLeaf, FSize nbParticles, const FSize *particleIndexes,
                                   void **sourceLeaves, const FSize **sourceParticleIndexes, FSize *sourceNbPart,
                                   const int *sourcePosition, const int size, void *userData);
typedef void (*Callback_apply_on_cell)(int level, long long morton_index, int *tree_position, double *spatial_position,
                                       void *userCell, void *userData);

typedef struct User_Scalfmm_Kernel_Descriptor {
  Callback_P2M p2m;
  Callback_M2M m2m;
  Callback_M2M_Full m2m_full;
  Callback_M2L m2l;
  Callback_M2L_Ext m2l_ext;
  Callback_M2LFull m2l_full;
  Callback_L2L l2l;
  Callback_L2L_Full l2l_full;
  Callback_L2P l2p;
  Callback_P2P p2p;
  Callback_P2PFull p2p_full;
  Callback_P2PInner p2pinner;
  Callback_P2PSym p2p_sym;
  Callback_P2PRemote p2p_remote;
} Scalfmm_Kernel_Descriptor;

/* ---- init and tree (CScalfmmApi.h:103, 259-324) ---- */
B200FMM_API scalfmm_handle scalfmm_init(scalfmm_kernel_type KernelType, scalfmm_algorithm algo);
B200FMM_API void scalfmm_build_tree(scalfmm_handle handle, int TreeHeight, double BoxWidth, double *BoxCenter,
                                    Scalfmm_Cell_Descriptor user_cell_descriptor,
                                    Scalfmm_Leaf_Descriptor user_leaf_descriptor);
B200FMM_API void scalfmm_tree_abstract_insert(scalfmm_handle Handle, int NbPartToInsert, int nbAttributeToInsert,
                                              int *strideForEachAtt, double *rawDatas);
B200FMM_API void scalfmm_tree_insert_particles(scalfmm_handle Handle, int NbPositions, double *arrayX, double *arrayY,
                                               double *arrayZ, PartType type);
B200FMM_API void scalfmm_tree_insert_particles_xyz(scalfmm_handle Handle, int NbPositions, double *XYZ, PartType type);

/* ---- physical values, forces, potentials (CScalfmmApi.h:339-423) ---- */
B200FMM_API void scalfmm_set_physical_values(scalfmm_handle Handle, int nbPhysicalValues, double *physicalValues,
                                             PartType type);
B200FMM_API void scalfmm_get_physical_values(scalfmm_handle Handle, int nbPhysicalValues, double *physicalValues,
                                             PartType type);
B200FMM_API void scalfmm_set_physical_values_npart(scalfmm_handle Handle, int nbPhysicalValues, int *idxOfParticles,
                                                   double *physicalValues, PartType type);
B200FMM_API void scalfmm_get_physical_values_npart(scalfmm_handle Handle, int nbPhysicalValues, int *idxOfParticles,
                                                   double *physicalValues, PartType type);
B200FMM_API void scalfmm_get_forces_xyz(scalfmm_handle Handle, int nbParts, double *forcesToFill, PartType type);
B200FMM_API void scalfmm_get_forces_xyz_npart(scalfmm_handle Handle, int nbParts, int *idxOfParticles,
                                              double *forcesToFill, PartType type);
B200FMM_API void scalfmm_get_forces(scalfmm_handle Handle, int nbParts, double *fX, double *fY, double *fZ,
                                    PartType type);
B200FMM_API void scalfmm_get_forces_npart(scalfmm_handle Handle, int nbParts, int *idxOfParticles, double *fX,
                                          double *fY, double *fZ, PartType type);
B200FMM_API void scalfmm_set_forces_xyz(scalfmm_handle Handle, int nbParts, double *forcesToFill, PartType type);
B200FMM_API void scalfmm_set_forces_xyz_npart(scalfmm_handle Handle, int nbParts, int *idxOfParticles,
                                              double *forcesToFill, PartType type);
B200FMM_API void scalfmm_set_forces(scalfmm_handle Handle, int nbParts, double *fX, double *fY, double *fZ,
                                    PartType type);
B200FMM_API void scalfmm_set_forces_npart(scalfmm_handle Handle, int nbParts, int *idxOfParticles, double *fX,
                                          double *fY, double *fZ, PartType type);
B200FMM_API void scalfmm_get_potentials(scalfmm_handle Handle, int nbParts, double *potentialsToFill, PartType type);
B200FMM_API void scalfmm_set_potentials(scalfmm_handle Handle, int nbParts, double *potentialsToRead, PartType type);
B200FMM_API void scalfmm_get_potentials_npart(scalfmm_handle Handle, int nbParts, int *idxOfParticles,
                                              double *potentialsToFill, PartType type);
B200FMM_API void scalfmm_set_potentials_npart(scalfmm_handle Handle, int nbParts, int *idxOfParticles,
                                              double *potentialsToRead, PartType type);

/* ---- moving particles (CScalfmmApi.h:436-472) ---- */
B200FMM_API void scalfmm_add_to_positions_xyz(scalfmm_handle Handle, int NbPositions, double *updatedXYZ,
                                              PartType type);
B200FMM_API void scalfmm_add_to_positions(scalfmm_handle Handle, int NbPositions, double *X, double *Y, double *Z,
                                          PartType type);
B200FMM_API void scalfmm_add_to_positions_xyz_npart(scalfmm_handle Handle, int NbPositions, int *idxOfParticles,
                                                    double *updatedXYZ, PartType type);
B200FMM_API void scalfmm_add_to_positions_npart(scalfmm_handle Handle, int NbPositions, int *idxOfParticles,
                                                double *X, double *Y, double *Z, PartType type);
B200FMM_API void scalfmm_set_positions_xyz(scalfmm_handle Handle, int NbPositions, double *updatedXYZ, PartType type);
B200FMM_API void scalfmm_set_positions(scalfmm_handle Handle, int NbPositions, double *X, double *Y, double *Z,
                                       PartType type);
B200FMM_API void scalfmm_set_positions_xyz_npart(scalfmm_handle Handle, int NbPositions, int *idxOfParticles,
                                                 double *updatedXYZ, PartType type);
B200FMM_API void scalfmm_set_positions_npart(scalfmm_handle Handle, int NbPositions, int *idxOfParticles, double *X,
                                             double *Y, double *Z, PartType type);
B200FMM_API void scalfmm_update_tree(scalfmm_handle handle);
B200FMM_API void scalfmm_get_positions_xyz(scalfmm_handle Handle, int NbPositions, double *positionsToFill,
                                           PartType type);
B200FMM_API void scalfmm_get_positions(scalfmm_handle Handle, int NbPositions, double *X, double *Y, double *Z,
                                       PartType type);
B200FMM_API void scalfmm_get_positions_xyz_npart(scalfmm_handle Handle, int NbPositions, int *idxOfParticles,
                                                 double *positionsToFill, PartType type);
B200FMM_API void scalfmm_get_positions_npart(scalfmm_handle Handle, int NbPositions, int *idxOfParticles, double *X,
                                             double *Y, double *Z, PartType type);

/* ---- algorithm, kernel, execution (CScalfmmApi.h:491-753) ---- */
B200FMM_API void scalfmm_algorithm_config(scalfmm_handle Handle, scalfmm_algorithm config);
B200FMM_API void scalfmm_user_kernel_config(scalfmm_handle Handle, Scalfmm_Kernel_Descriptor userKernel,
                                            void *userDatas);
B200FMM_API void scalfmm_execute_fmm(scalfmm_handle Handle);
B200FMM_API void scalfmm_execute_fmm_far_field(scalfmm_handle Handle);
/* Each leaf in Morton order: level = height-1, its particles' insertion indices, its Morton index and lower-left
 * corner; cellDatas, leafDatas and userDatas are NULL (the built-in kernels keep no user data). */
B200FMM_API void scalfmm_apply_on_leaf(scalfmm_handle Handle, Callback_apply_on_leaf function);

/* ---- release, monitoring, utilities (CScalfmmApi.h:772-830) ---- */
B200FMM_API void scalfmm_dealloc_handle(scalfmm_handle handle, Callback_free_cell cellDestroyer);
B200FMM_API void scalfmm_apply_on_cell(scalfmm_handle handle, Callback_apply_on_cell function);
/* FAlgorithmTimers::nbTimers (Src/Utils/FAlgorithmTimers.hpp:31) */
B200FMM_API int scalfmm_get_nb_timers(scalfmm_handle handle);
/* Seconds of the last execute, in the reference's order: P2M, M2M, M2L, L2L, L2P, P2P, NearField (P2P + L2P),
 * then 0 for the M2P and P2L timers that the interpolation kernels do not use. */
B200FMM_API void scalfmm_get_timers(scalfmm_handle handle, double *Timers);
B200FMM_API void scalfmm_set_upper_limit(scalfmm_handle handle, int upperLimit);
B200FMM_API void scalfmm_utils_parentChildPosition(int childPosition, int *childFullPosition);
B200FMM_API void scalfmm_utils_interactionPosition(int interactionPosition, int *srcPosition);
B200FMM_API void scalfmm_print_everything(scalfmm_handle handle);

/* ---- extensions ---- */
/* B200FMM_FP64 (default) or B200FMM_MIXED; call before scalfmm_build_tree. */
B200FMM_API b200fmm_status b200fmm_capi_set_precision(scalfmm_handle handle, int precision);
/* Status of the handle's last failing call, B200FMM_OK if none failed. */
B200FMM_API b200fmm_status b200fmm_capi_status(scalfmm_handle handle);

#ifdef __cplusplus
}
#endif
#endif
