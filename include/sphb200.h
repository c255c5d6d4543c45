/*
 * sphb200 — C ABI of the B200 (sm_100a) SPH-VE hydro hot path.
 *
 * Plain C types only: device pointers are passed as typed pointers into device memory, CUDA streams as void*
 * (a cudaStream_t; NULL = the legacy default stream). Every function returns an sphb status code and never exits
 * the process (the reference's checkGpuErrors calls exit(), cstone/cuda/errorcheck.cuh:15-26).
 *
 * Two layers:
 *   1. kernel entry points on caller-owned device arrays — the drop-in for the cstone::*Gpu and sph::gpu::*
 *      functions that the reference's host dispatchers call under HaveGpu<Accelerator> (each cited below);
 *   2. an opaque simulation object (sphb_sim) that owns the particle dataset in HBM and runs the whole step of
 *      HydroVeProp (main/src/propagator/ve_hydro.hpp:126-220): domain sync, neighbour search, VE chain, integration.
 */
#ifndef SPHB200_H
#define SPHB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------------------------------------------- */
/* status codes                                                                                                     */
/* ---------------------------------------------------------------------------------------------------------------- */
#define SPHB_OK 0
#define SPHB_ERR_ARG 1           /* invalid argument (null pointer, bad size, ng0 > ngmax, ...)                     */
#define SPHB_ERR_CUDA 2          /* a CUDA runtime call failed; message printed to stderr                           */
#define SPHB_ERR_CAPACITY 3      /* a bounded device buffer or wait was exhausted (scratch, traversal, lookback)    */
#define SPHB_ERR_NOT_CONVERGED 4 /* smoothing-length iteration left particles with nc <= 1 (update_h_gpu.cu:51-55) */
#define SPHB_ERR_STATE 5         /* call out of order (e.g. step before upload)                                    */
#define SPHB_ERR_TIMEOUT 6       /* a bounded device-side wait gave up (the sort's look-back); outputs are undefined */

/* precision of the neighbour sums (the SPH-VE J-loops) */
#define SPHB_FP64 0  /* every field and sum in double: the plain drop-in                                           */
#define SPHB_MIXED 1 /* FP32 neighbour sums with compensated accumulation on FP64 relative coordinates            */

/*! Coordinate box; replaces cstone::Box<double> (domain/include/cstone/sfc/box.hpp:94-174). periodic[k] != 0 makes
 *  axis k periodic, else open. */
typedef struct
{
    double lo[3];
    double hi[3];
    int periodic[3];
} sphb_box;

/*! Physics settings; defaults of ParticlesData (sph/include/sph/particles_data.hpp:85-143). */
typedef struct
{
    uint32_t ng0;           /* target neighbour count (100)                                */
    uint32_t ngmax;         /* neighbour list capacity per particle (150)                  */
    double gamma;           /* adiabatic index (5/3)                                       */
    double mui;             /* mean molecular weight of ions (10)                          */
    double Kcour;           /* Courant factor (0.2)                                        */
    double Krho;            /* 1/|divv| time-step factor (0.06)                            */
    double alphamin;        /* AV switch floor (0.05)                                      */
    double alphamax;        /* AV switch ceiling (1.0)                                     */
    double decay_constant;  /* AV decay (0.2)                                              */
    double sinc_index;      /* exponent n of the sinc^n kernel (6)                         */
    double minDt;           /* initial time step                                           */
    double minDt_m1;        /* previous time step                                          */
    int precision;          /* SPHB_FP64 or SPHB_MIXED                                     */
    uint32_t bucket_focus;  /* max particles per leaf of the neighbour-search tree (64)    */
    int av_clean;           /* 1: AV cleaning in MomentumEnergy (HydroVeProp<avClean = true>,
                               momentum_energy_kern.hpp:43-63,165-169); 0 (default): off   */
    double nb_skin;         /* relative skin of the reused candidate lists (0.05); 0: search the
                               tree every step. The lists are the same either way: every
                               step keeps exactly the j with |x_i - x_j| < 2 h_i.           */
} sphb_params;

/* element types of caller arrays in sphb_field */
#define SPHB_F32 1 /* float          */
#define SPHB_F64 2 /* double         */
#define SPHB_U32 3 /* uint32 (nc)    */
#define SPHB_U64 4 /* uint64 (id, keys) */

/*! One caller array of a particle field: the field's name in the reference's ParticlesData
 *  (sph/include/sph/particles_data.hpp:262-266), the array's first element, and its element type (SPHB_F32 ...).
 *  With the reference's default SphTypes (sph/types.hpp:39-46) x, y, z, temp, u and du are double, and h, m, vx,
 *  vy, vz, x_m1, y_m1, z_m1, du_m1, alpha and the derived hydro fields are float. */
typedef struct
{
    const char* name;
    void* data;
    int dtype;
} sphb_field;

/*! Fill p with the reference defaults listed above (precision = SPHB_FP64). */

void sphb_default_params(sphb_params* p);

/*! Library version string. */
const char* sphb_version(void);

/* ---------------------------------------------------------------------------------------------------------------- */
/* 1. Kernel entry points on caller-owned device arrays                                                             */
/* ---------------------------------------------------------------------------------------------------------------- */

/*! Hilbert SFC keys of n particles; keys equal to the removal key (1<<63) are kept as they are.
 *  Replaces cstone::computeSfcKeysGpu (domain/include/cstone/sfc/sfc_gpu.cu:35-43; key math sfc.hpp:141-178,
 *  hilbert.hpp:43-94). */
int sphb_compute_sfc_keys(const double* x, const double* y, const double* z, uint64_t* keys, size_t n,
                          const sphb_box* box, void* stream);

/*! Scratch bytes needed by sphb_sort_by_key for n elements.
 *  Replaces cstone::sortByKeyTempStorage (domain/include/cstone/primitives/primitives_gpu.cu:297-306). */
size_t sphb_sort_by_key_scratch_bytes(size_t n);

/*! Stable ascending sort of n (uint64 key, uint32 value) pairs in place, using caller scratch of at least
 *  sphb_sort_by_key_scratch_bytes(n) bytes. If init_values != 0, values are first set to 0..n-1 (the sequence +
 *  sort of GlobalAssignment::assign, domain/include/cstone/domain/assignment.hpp:110-112). Host-blocking: it reads
 *  the digit histogram and the error word back. A look-back wait that gives up returns SPHB_ERR_TIMEOUT.
 *  Replaces cstone::sortByKeyGpu (domain/include/cstone/primitives/primitives_gpu.cu:308-339). */
int sphb_sort_by_key(uint64_t* keys, uint32_t* values, size_t n, int init_values, void* scratch, size_t scratch_bytes,
                     void* stream);

/*! Same result as sphb_sort_by_key with init_values = 1, for keys that are nearly in order (the particles of the
 *  previous step, which moved a fraction of a smoothing length). If no adjacent pair is out of order nothing moves
 *  and *identity is set to 1. Otherwise the 2048-key tiles that hold inversions are sorted in shared memory (two
 *  overlapping tilings), and the full radix sort runs only if inversions remain. Host-blocking (two small reads).
 *  No counterpart in the reference (it sorts from scratch every step, assignment.hpp:112). */
int sphb_sort_by_key_nearly_sorted(uint64_t* keys, uint32_t* values, size_t n, void* scratch, size_t scratch_bytes,
                                   int* identity, void* stream);

/*! Same sort as sphb_sort_by_key, for callers that cannot allocate device memory: for example code whose device
 *  memory all belongs to another allocator (a framework's caching pool), or code running where cudaMalloc is not
 *  allowed. It calls no cudaMalloc, cudaFree or other allocating routine; its scratch is a fixed array of about
 *  12.6 MB inside this library. The array is reserved on a device when the library's device code is loaded there
 *  (with lazy module loading, at the first call on that device at the latest) and kept until the process exits.
 *  n may be at most sphb_sort_by_key_static_max() (1,048,576); larger n returns SPHB_ERR_CAPACITY and sorts
 *  nothing. The first call in a CUDA context looks up the array's device address (once per context). Like
 *  sphb_sort_by_key, every call blocks the calling host thread: it
 *  waits for the stream twice (the digit histogram and the error word are read back). All calls share the one
 *  array: calls that overlap on the GPU (on different streams or from different threads) race with each other, so
 *  run them one after another. The array keeps the previous call's contents; every call clears what it needs
 *  before use. A look-back wait that gives up returns SPHB_ERR_TIMEOUT.
 *  No counterpart in the reference. */
int sphb_sort_by_key_static(uint64_t* keys, uint32_t* values, size_t n, int init_values, void* stream);

/*! Largest n accepted by sphb_sort_by_key_static. */
size_t sphb_sort_by_key_static_max(void);

/*! dst_f[i] = src_f[order[i]] for num_fields arrays of 8-byte elements (double or uint64).
 *  Replaces cstone::gatherGpu (domain/include/cstone/primitives/primitives_gpu.cu:73-88) applied per field by
 *  Domain::updateLayout (domain/include/cstone/domain/domain.hpp:491-537). */
int sphb_gather8(const uint32_t* order, size_t n, int num_fields, const void* const* src, void* const* dst,
                 void* stream);

/*! The internal (linked) octree of a cornerstone leaf array in the reference's OctreeData layout
 *  (cstone/tree/octree.hpp:283-358): nodes sorted by level, then SFC key. With num_internal = (num_leaves - 1) / 7
 *  and num_nodes = num_leaves + num_internal, the device arrays receive: prefixes [num_nodes] (placeholder-bit
 *  keys), child_offsets [num_nodes] (first child, 0 for leaves), parents [max(1, (num_nodes - 1) / 8)] (parent of
 *  every group of 8 siblings), internal_to_leaf [num_nodes] (leaf index, negative for internal nodes),
 *  leaf_to_internal [num_nodes] (sorted node index by the reference's unsorted index: internal nodes first, then
 *  leaves); level_range (host, 23 ints) the first node of every level. Host-blocking.
 *  Replaces cstone::buildOctreeGpu (domain/include/cstone/tree/octree_gpu.cu:137-165) and its CPU twin
 *  buildOctreeCpu (octree.hpp:170-196). */
int sphb_build_octree(const uint64_t* leaves, size_t num_leaves, uint64_t* prefixes, int* child_offsets,
                      int* parents, int* level_range, int* internal_to_leaf, int* leaf_to_internal, void* stream);

/*! The ideal-gas EOS on caller arrays, per particle i in [first, last), in FP64 and stored in each array's type:
 *  rho = kx m / xm, p = rho u (gamma - 1) with u = cv(mui, gamma) temp (or u itself if given),
 *  c = sqrt(gamma u (gamma - 1)), prho = p / (kx m^2 gradh). fields names temp or u, m, kx, xm, gradh (read) and
 *  prho, c, and optionally rho and p (written), each SPHB_F32 or SPHB_F64, device memory. Asynchronous on stream.
 *  Replaces sph::gpu::computeIdealGasEOS (sph/include/sph/sph_gpu.hpp:42-45; hydro_ve/eos_gpu.cu:44-61;
 *  sph/include/sph/eos.hpp:19-50). */
int sphb_ideal_gas_eos(size_t first, size_t last, double mui, double gamma, const sphb_field* fields, int num_fields,
                       void* stream);

/*! Fully converged cornerstone leaf array for sorted keys (host-blocking: loops until no node splits or merges).
 *  Writes num_leaves + 1 keys to leaves and num_leaves counts, if num_leaves + 1 <= capacity.
 *  Replaces cstone::computeOctree / updateOctree (domain/include/cstone/tree/csarray.hpp:409-440) and their GPU
 *  counterparts computeNodeCountsGpu / rebalanceTreeGpu (csarray_gpu.cu:85-213). */
int sphb_compute_octree(const uint64_t* sorted_keys, size_t n, unsigned bucket, uint64_t* leaves, uint32_t* counts,
                        size_t capacity, size_t* num_leaves, void* stream);

/*! Leaf counts of a rank's sorted keys in the shared global tree: counts[i] = keys in [leaves[i], leaves[i + 1]).
 *  leaves holds num_leaves + 1 keys of a cornerstone array. Device arrays; stream-ordered.
 *  Replaces cstone::computeNodeCounts as cstone::updateOctreeGlobal calls it before its count all-reduce
 *  (domain/include/cstone/tree/update_mpi.hpp:64-99; csarray.hpp:181-235, GPU twin computeNodeCountsGpu
 *  csarray_gpu.cu:85-119). */
int sphb_leaf_counts(const uint64_t* leaves, size_t num_leaves, const uint64_t* sorted_keys, size_t n,
                     uint32_t* counts, void* stream);

/*! One rebalance step of a cornerstone tree on given (all-reduced) leaf counts: leaves with more than bucket particles
 *  split, groups of 8 sibling leaves with at most bucket together merge. new_leaves (not aliasing leaves) receives
 *  *num_new + 1 keys if *num_new + 1 <= capacity (else SPHB_ERR_CAPACITY; *num_new and *converged are always
 *  written); *converged = 1 if the step changed nothing. Device arrays; host-blocking.
 *  Replaces cstone::rebalanceDecision + rebalanceTree as updateOctreeGlobal applies them
 *  (domain/include/cstone/tree/update_mpi.hpp:64-99; csarray.hpp:248-389, GPU twins rebalanceDecisionGpu /
 *  rebalanceTreeGpu csarray_gpu.cu:121-213). */
int sphb_rebalance_tree(const uint64_t* leaves, size_t num_leaves, const uint32_t* counts, unsigned bucket,
                        uint64_t* new_leaves, size_t capacity, size_t* num_new, int* converged, void* stream);

/*! Halo discovery of one rank on the shared global tree (num_leaves + 1 keys). The rank owns the leaves
 *  [first_leaf, last_leaf); its particles are in SFC order in x, y, z, h (h_dtype SPHB_F32 or SPHB_F64), leaf
 *  first_leaf + i holding the particles [layout[i], layout[i + 1]) (last_leaf - first_leaf + 1 offsets). The search
 *  box of an owned leaf is the smallest box holding the leaf's geometric centre and the cube x +- h * 2 search_ext of
 *  each of its particles (the radius rounded in h's type); flags[l] (num_leaves bytes) becomes 1 for every leaf l
 *  outside the owned range whose cell overlaps a search box (minimum image on periodic axes), else 0. Device arrays;
 *  host-blocking. Replaces cstone::FocusedOctree::discoverHalos (domain/include/cstone/focus/
 *  octree_focus_mpi.hpp:513-571: computeBoundingBoxGpu, focus/source_center_gpu.cu:23-92, and findHalosGpu,
 *  traversal/collisions.hpp:40-104), on the global tree instead of the focus tree. */
int sphb_find_halos(const uint64_t* leaves, size_t num_leaves, const double* x, const double* y, const double* z,
                    const void* h, int h_dtype, const uint32_t* layout, size_t first_leaf, size_t last_leaf,
                    const sphb_box* box, float search_ext, uint8_t* flags, void* stream);

/*! Spatial target groups of the particles [first, last), which are in SFC order: fixed runs of group_size (32 or 64)
 *  consecutive particles, each split after every particle whose successor lies farther than
 *  min(tol_factor * the run's smallest leaf edge, 2 h) (lengths relative to the box; the leaf edge from leaves
 *  (num_leaves + 1 keys) and layout (first particle of each leaf) of the focus tree). groups receives
 *  num_groups + 1 boundaries, group g being [groups[g], groups[g + 1]), if num_groups + 1 <= capacity (else
 *  SPHB_ERR_CAPACITY; *num_groups is always written). h may be NULL (no smoothing-length criterion); h_dtype
 *  (SPHB_F32 or SPHB_F64) is its type and the precision of the threshold, as in the reference. Device arrays;
 *  host-blocking. Replaces cstone::computeGroupSplits (domain/include/cstone/traversal/groups_gpu.cu:108-137,
 *  groups_gpu.cuh:37-216) as sph::computeSpatialGroups calls it (sph/include/sph/groups.hpp:41-55: tol_factor 2,
 *  group_size 32). */
int sphb_compute_group_splits(size_t first, size_t last, const double* x, const double* y, const double* z,
                              const void* h, int h_dtype, const uint64_t* leaves, size_t num_leaves,
                              const uint32_t* layout, const sphb_box* box, unsigned group_size, float tol_factor,
                              uint32_t* groups, size_t capacity, size_t* num_groups, void* stream);

/* ---------------------------------------------------------------------------------------------------------------- */
/* 2. Simulation object: the whole hydro step of HydroVeProp                                                        */
/* ---------------------------------------------------------------------------------------------------------------- */
typedef struct sphb_sim sphb_sim;

/*! Create a simulation of n particles on the current CUDA device; allocates every field in HBM.
 *  Mirrors Domain(rank 0 of 1, bucketSize = max(64, n/100), bucketSizeFocus, theta 1) + ParticlesData
 *  (main/src/sphexa/sphexa.cpp:129-138). */
int sphb_sim_create(sphb_sim** sim, size_t n, const sphb_box* box, const sphb_params* params);
int sphb_sim_destroy(sphb_sim* sim);

/*! Copy the conserved fields in. fields holds 14 arrays of n doubles in the order
 *  x,y,z,h,m,temp,vx,vy,vz,x_m1,y_m1,z_m1,du_m1,alpha; id holds n uint64. on_device != 0: the pointers are device
 *  memory, else host memory (pinned or pageable). Resets the step state (first-call tree convergence). */
int sphb_sim_upload(sphb_sim* sim, const double* const* fields, const uint64_t* id, int on_device);

/*! The sync that the reference main program performs once before the first step (sphexa.cpp:141). */
int sphb_sim_initial_sync(sphb_sim* sim);

/*! First half of a step: HydroVeProp::computeForces (ve_hydro.hpp:126-203): domain sync (keys, sort, global and
 *  focus cornerstone trees, gather), neighbour search with smoothing-length iteration, XMass, VeDefGradh, EOS,
 *  IAD + divv/curlv, rho time step, AV switches, momentum-energy with Courant time step; then the conserved
 *  quantities (main/src/observables/conserved_quantities.hpp:117-175). */
int sphb_sim_compute_forces(sphb_sim* sim);

/*! Second half: computeTimestep, computePositions, updateSmoothingLength (ve_hydro.hpp:205-220).
 *  Returns SPHB_ERR_NOT_CONVERGED if any particle ended with nc <= 1 (its key is set to the removal key). */
int sphb_sim_integrate(sphb_sim* sim);

/*! compute_forces + integrate. */
int sphb_sim_step(sphb_sim* sim);

/*! Block time steps: switch this simulation to the propagator of main/src/propagator/ve_hydro_bdt.hpp
 *  (HydroVeBdtProp<avClean>, avClean from sphb_params.av_clean). The groups are the reference's spatial target
 *  groups of at most 32 SFC-consecutive particles (sph::computeSpatialGroups, as sphb_compute_group_splits), formed
 *  at every full sync (ve_hydro_bdt.hpp:185). Each group gets
 *  the time step min(Courant, Krho / |max divv|, eta_acc (h^2/|a|^2)^(1/4)) over its particles (ts_groups.cu), the
 *  groups are sorted by it into up to 4 power-of-two rungs (ts_rungs.hpp:116-166), and a block step of
 *  2^(numRungs - 1) substeps computes forces only on the groups of the active rungs while the others drift.
 *  eta_acc: the acceleration criterion (ParticlesData::etaAcc, 0.2). After this call sphb_sim_compute_forces,
 *  sphb_sim_step and the stage calls return SPHB_ERR_STATE; sphb_sim_upload resets the block-step state. */
int sphb_sim_bdt_enable(sphb_sim* sim, double eta_acc);

/*! One substep of the block time-step propagator: computeForces (domain sync at the first substep of a block,
 *  neighbour search of every particle, the SPH-VE chain on the active groups, EOS of every particle, group time
 *  steps) then integrate (rungs, kick-drift of the rungs that complete their step, drift of the others, h update of
 *  the active groups) (ve_hydro_bdt.hpp:224-380). SPHB_ERR_NOT_CONVERGED as sphb_sim_integrate. */
int sphb_sim_bdt_step(sphb_sim* sim);

/*! sph::Timestep of the block time-step propagator (sph/include/sph/timestep.h:17-31) after the last substep. */
typedef struct
{
    float next_dt, elapsed_dt, total_dt;
    int num_rungs, substep;
    uint32_t rung_ranges[5]; /* groups [rung_ranges[r], rung_ranges[r+1]) of the dt-sorted order are rung r */
    float dt_m1[4];          /* last full step per rung                                             */
    float dt_drift[4];       /* time each rung has drifted since its last full step                 */
    uint32_t num_active;     /* groups whose forces the last substep computed                        */
} sphb_bdt_timestep;

int sphb_sim_bdt_timestep(const sphb_sim* sim, sphb_bdt_timestep* out);

/* The force computation one stage at a time, for a caller that runs its own code between the stages as the
 * reference's propagator does (HydroVeProp::computeForces, ve_hydro.hpp:126-203, exchanges halos between them).
 * sphb_sim_compute_forces runs exactly these eight calls. Each stage must follow the previous one of the same force
 * computation (else SPHB_ERR_STATE); sphb_sim_sync may start a new one at any time, and sphb_sim_integrate needs
 * sphb_sim_conserved to have completed. */

/*! Domain::sync (cstone/domain/domain.hpp:165-213): box, keys, sort, gather, trees, packed positions. */
int sphb_sim_sync(sphb_sim* sim);

/*! The neighbour search with the smoothing-length iteration (sph/include/sph/find_neighbors.hpp:10-41; GPU:
 *  computeXMass's traversal, sph/include/sph/hydro_ve/xmass_gpu.cu:78-92). */
int sphb_sim_find_neighbors(sphb_sim* sim);

/*! sph::gpu::computeXMass (sph/include/sph/hydro_ve/xmass_gpu.cu, xmass_kern.hpp:50-79). */
int sphb_sim_xmass(sphb_sim* sim);

/*! sph::gpu::computeVeDefGradh + computeEOS (ve_def_gradh_kern.hpp:43-90, hydro_ve/eos.hpp:52-94). */
int sphb_sim_ve_def_gradh_eos(sphb_sim* sim);

/*! sph::gpu::computeIadDivvCurlv (iad_kern.hpp:43-110, divv_curlv_kern.hpp:43-123). */
int sphb_sim_iad_divv_curlv(sphb_sim* sim);

/*! sph::gpu::computeAVswitches (av_switches_kern.hpp:43-137); uses the current minDt. */
int sphb_sim_av_switches(sphb_sim* sim);

/*! sph::gpu::computeMomentumEnergy (momentum_energy_kern.hpp:65-222). If min_dt_courant is not NULL it receives
 *  the minimum Courant time step (momentum_energy_gpu.cu:109-116), which costs one device synchronisation. */
int sphb_sim_momentum_energy(sphb_sim* sim, double* min_dt_courant);

/*! computeConservedQuantities (conserved_quantities.hpp:117-175) and the time-step reductions; completes the force
 *  computation. If out is not NULL it receives {kinetic energy, internal energy, total energy, |linear momentum|,
 *  |angular momentum|}. */
int sphb_sim_conserved(sphb_sim* sim, double* out);

/*! Number of owned particles. */
size_t sphb_sim_size(const sphb_sim* sim);

/*! Copy a field, by its reference name (particles_data.hpp:262-266: x y z h m temp vx vy vz x_m1 y_m1 z_m1 du_m1
 *  alpha xm kx gradh prho c c11 c12 c13 c22 c23 c33 divv curlv ax ay az du nc keys id), converted to double, into
 *  out (n doubles; host memory if on_device == 0, else device memory). keys and id are copied as uint64 bits. */
int sphb_sim_get_field(sphb_sim* sim, const char* name, double* out, int on_device);

/*! Overwrite a field by name from n doubles (host memory if on_device == 0). */
int sphb_sim_set_field(sphb_sim* sim, const char* name, const double* in, int on_device);

/*! Scalars: minDt, minDt_m1, minDtCourant, minDtRho, ttot, etot, ecin, eint, linmom, angmom, totalNeighbors,
 *  iteration, box xmin, xmax, ymin, ymax, zmin, zmax (18 doubles). */
int sphb_sim_scalars(sphb_sim* sim, double* out);

/*! Focus-tree leaves (num_leaves + 1 keys), leaf counts and particle layout (num_leaves + 1), host memory.
 *  With null arrays only *num_leaves is written. */
int sphb_sim_tree(sphb_sim* sim, size_t* num_leaves, uint64_t* leaves, uint32_t* counts, uint32_t* layout);

/*! Neighbour lists of the last force computation as [n][ngmax] uint32 (host memory), entries beyond
 *  min(nc-1, ngmax) undefined. */
int sphb_sim_neighbors(sphb_sim* sim, uint32_t* out);

/*! Per-stage device time of the last step in milliseconds (CUDA events): sync, neighbours, xmass, ve_def_gradh,
 *  eos, iad_divv_curlv, av_switches, momentum_energy, integrate (9 floats). */
int sphb_sim_stage_times(sphb_sim* sim, float* out);

/*! Number of kernels this library has launched in this process (for launch accounting). */
uint64_t sphb_sim_kernel_launches(const sphb_sim* sim);

/*! How the neighbour stage ran since creation: out[0] tree searches of every group, out[1] skin-row builds (each
 *  also counted in out[0]), out[2] steps served by refiltering the skin rows, out[3] groups those steps deferred to
 *  the tree search, out[4] domain syncs whose sort moved particles while rows were kept. No counterpart in the reference, which searches the tree every step
 *  (sph/include/sph/find_neighbors.hpp:10-41); the lists are the same either way. */
int sphb_sim_search_stats(const sphb_sim* sim, uint64_t* out);

/*! The CUDA stream (a cudaStream_t) on which the simulation issues all its work. */
void* sphb_sim_stream(sphb_sim* sim);

/*! Replace the 14 conserved fields and the ids of the current particles (same count, same layout as
 *  sphb_sim_upload) without resetting the domain state (trees, time step, iteration): the per-step host round trip of
 *  a caller that keeps the particle state in its own host buffers. */
int sphb_sim_load_state(sphb_sim* sim, const double* const* fields, const uint64_t* id, int on_device);

/*! Copy the 14 conserved fields and the ids out (current SFC order), host memory if on_device == 0. */
int sphb_sim_store_state(sphb_sim* sim, double* const* fields, uint64_t* id, int on_device);

/*! sphb_sim_upload with the caller's own element types: fields must name the 14 conserved fields (SPHB_F32 or
 *  SPHB_F64 each) and "id" (SPHB_U64), in any order. Host arrays cross the bus at their own width and are converted
 *  on the device, so a Dataset with the reference's default types (a mix of float and double) passes as it is. */
int sphb_sim_upload_fields(sphb_sim* sim, const sphb_field* fields, int num_fields, int on_device);

/*! One step of a caller that keeps the particle state in host memory, in its own element types: the typed load of in
 *  (host arrays, the fields of sphb_sim_upload_fields), sphb_sim_step, and the typed store of out (host arrays of any
 *  fields sphb_sim_store_fields accepts). Returns after every output is in host memory. The same results as the
 *  three calls one after another; the copies overlap the step where the data allow: the load's copies as in
 *  sphb_sim_load_fields; the outputs m and id (final after the sync) and alpha (final after the AV switches) leave
 *  the device while the later stages run; of the rest, the fields in their own type leave first, while the others
 *  are converted. */
int sphb_sim_step_fields(sphb_sim* sim, const sphb_field* in, int num_in, const sphb_field* out, int num_out);

/*! sphb_sim_load_state with the caller's own element types (the fields of sphb_sim_upload_fields). From host memory,
 *  x, y, z and m are copied first; the copies of the other fields may still run when the call returns, in the order
 *  the next step reads them: h and the ids beside its sync (unless the sync reorders the particles), temp beside
 *  the neighbour search, vx, vy, vz and alpha beside XMass and VeDefGradh, and x_m1, y_m1, z_m1 and du_m1 beside the
 *  J-loops. The host
 *  arrays must stay unchanged until the next call on the simulation returns (every call waits for the copies). */
int sphb_sim_load_fields(sphb_sim* sim, const sphb_field* fields, int num_fields, int on_device);

/*! Copy fields out by name, each converted to the element type of its descriptor: any name of
 *  sphb_sim_get_field (conserved, derived, du, nc, keys, id; keys and id only as SPHB_U64). Host memory if
 *  on_device == 0. */
int sphb_sim_store_fields(sphb_sim* sim, const sphb_field* fields, int num_fields, int on_device);

/* ---------------------------------------------------------------------------------------------------------------- */
/* 2b. The force stages on a caller's dataset, in place                                                             */
/* ---------------------------------------------------------------------------------------------------------------- */

/* These replace the reference's per-stage GPU dispatch of HydroVeProp (main/src/propagator/ve_hydro.hpp:126-220):
 * sph::gpu::computeXMass, computeVeDefGradh, computeIdealGasEOS, computeIadDivvCurlv, computeAVswitches,
 * computeMomentumEnergy<avClean = false> (sph/include/sph/sph_gpu.hpp:24-45), computePositionsGpu and
 * updateSmoothingLengthGpu (sph_gpu.hpp:79-87). Each reads and writes the arrays of a caller's Dataset on the device,
 * bound once by field name, in the caller's element types; the simulation object only holds this library's own
 * state (octree, neighbour lists, records). first/last are the GroupView's particle range (firstBody, lastBody;
 * cstone/traversal/groups.hpp:28-34); at one rank without halos it must be [0, sphb_sim_size(sim)). box is the
 * Domain's box of this force computation; the later stages must pass the box of its sphb_dataset_xmass
 * (SPHB_ERR_STATE otherwise). The stages keep the reference's order (the stage ABI's SPHB_ERR_STATE rule). Positions
 * and h must not change between sphb_dataset_xmass and the later stages of the same force computation, as within
 * computeForces. Not available with block time steps or AV cleaning (SPHB_ERR_STATE). */

/*! Bind the caller's device arrays (each of sphb_sim_size(sim) elements) by field name: any field of
 *  sphb_sim_get_field plus rho, p and u (the EOS's optional fields), reals as SPHB_F32 or SPHB_F64, nc as SPHB_U32,
 *  id and keys as SPHB_U64. Replaces any previous binding and restarts the step state (as an upload). */
int sphb_sim_bind_fields(sphb_sim* sim, const sphb_field* fields, int num_fields);

/*! sph::gpu::computeXMass (sph_gpu.hpp:24-25; xmass_gpu.cu:103-124): builds this library's octree from the bound
 *  particles, which must already be in the SFC order of box (as after the reference's Domain::sync; otherwise
 *  SPHB_ERR_STATE), then runs the neighbour search with the smoothing-length iteration and XMass.
 *  Reads id, x, y, z, h, m; writes h, nc, xm. */
int sphb_dataset_xmass(sphb_sim* sim, size_t first, size_t last, const sphb_box* box);

/*! sph::gpu::computeVeDefGradh (sph_gpu.hpp:30-31; ve_def_gradh_kern.hpp:43-90). Reads xm (and x, y, z, h, m of the
 *  preceding sphb_dataset_xmass); writes kx, gradh. */
int sphb_dataset_ve_def_gradh(sphb_sim* sim, size_t first, size_t last, const sphb_box* box);

/*! sph::gpu::computeIadDivvCurlv (sph_gpu.hpp:33-34; iad_kern.hpp:43-110, divv_curlv_kern.hpp:43-123). Reads vx,
 *  vy, vz, xm, kx, c, prho; writes c11, c12, c13, c22, c23, c33, divv, curlv. */
int sphb_dataset_iad_divv_curlv(sphb_sim* sim, size_t first, size_t last, const sphb_box* box);

/*! sph::gpu::computeAVswitches (sph_gpu.hpp:36-37; av_switches_kern.hpp:43-137) with the previous time step min_dt.
 *  Reads vx, vy, vz, xm, kx, c, prho, c11 ... c33, divv, alpha; writes alpha. */
int sphb_dataset_av_switches(sphb_sim* sim, size_t first, size_t last, const sphb_box* box, double min_dt);

/*! sph::gpu::computeMomentumEnergy<avClean = false> (sph_gpu.hpp:39-40; momentum_energy_kern.hpp:65-222). Reads vx,
 *  vy, vz, xm, kx, c, prho, c11 ... c33, divv, alpha; writes ax, ay, az, du and, if not NULL, *min_dt_courant (the
 *  float the reference's kernel reduces, momentum_energy_gpu.cu:109-116). */
int sphb_dataset_momentum_energy(sphb_sim* sim, size_t first, size_t last, const sphb_box* box,
                                 float* min_dt_courant);

/*! computePositionsGpu of the global step (sph_gpu.hpp:79-83; positions_gpu.cu:118-183) with time steps dt and
 *  dt_m1. Reads x, y, z, vx, vy, vz, x_m1, y_m1, z_m1, temp, du, du_m1, ax, ay, az; writes x, y, z, vx, vy, vz,
 *  x_m1, y_m1, z_m1, temp, du_m1. */
int sphb_dataset_positions(sphb_sim* sim, size_t first, size_t last, double dt, double dt_m1, const sphb_box* box);

/*! updateSmoothingLengthGpu (sph_gpu.hpp:86-87; update_h_gpu.cu:41-71). Reads nc, h; writes h, and keys (if bound)
 *  with the removal key for particles left with nc <= 1, in which case it returns SPHB_ERR_NOT_CONVERGED. */
int sphb_dataset_update_h(sphb_sim* sim, size_t first, size_t last, unsigned ng0);

/* ---------------------------------------------------------------------------------------------------------------- */
/* 3. Differentiation of the step                                                                                   */
/* ---------------------------------------------------------------------------------------------------------------- */

/*! Use a fixed time step dt instead of computeTimestep (sph/include/sph/ts_global.hpp:100-128); dt = 0 restores the
 *  adaptive step. With dt > 0, minDt and minDt_m1 are set to dt (the AV switches and the integration read them).
 *  No counterpart in the reference (its propagators always compute the step); required by sphb_sim_step_vjp. */
int sphb_sim_set_fixed_dt(sphb_sim* sim, double dt);

/*! Replace the physics parameters of a simulation (gamma, mui, Kcour, Krho, alphamin, alphamax, decay_constant) as
 *  between steps of the reference's propagator (ParticlesData members, particles_data.hpp:85-143). ng0, ngmax,
 *  precision, sinc_index and bucket_focus must be unchanged (SPHB_ERR_ARG otherwise). */
int sphb_sim_set_params(sphb_sim* sim, const sphb_params* params);

/*! Adjoint (vector-Jacobian product) of one step of the VE propagator (main/src/propagator/ve_hydro.hpp:126-220)
 *  with a fixed time step and the step's discrete structure held fixed (sort permutation, neighbour lists and
 *  counts, smoothing-length iterations, branch choices). Precondition: the simulation holds the state the step
 *  starts from (after sphb_sim_load_state of a stored state, or the state before an sphb_sim_step) and a fixed
 *  time step is set. The call recomputes the step's forces (neighbour search and chain) with a tape, then maps
 *  adj_post, the adjoint of the state after the step (14 device arrays of n doubles, conserved-field order,
 *  indexed like the state sphb_sim_store_state returns after the step), to adj_pre, the adjoint of the state before
 *  the step (indexed like the state the step starts from); *alphamax_bar (host) is incremented by the derivative
 *  with respect to alphamax. The adjoint of m is passed through unchanged. Precision follows the simulation: FP64
 *  adjoint for SPHB_FP64, FP32 J-loop adjoints for SPHB_MIXED. Afterwards the simulation holds the recomputed
 *  post-force state, not the state after the step. Not available with AV cleaning (SPHB_ERR_STATE).
 *  No counterpart in the reference. */
int sphb_sim_step_vjp(sphb_sim* sim, const double* const* adj_post, double* const* adj_pre, double* alphamax_bar);

/*! Reserve device memory for `slots` recorded steps (about 1 KB per particle each). Recording replaces the force
 *  recomputation of sphb_sim_step_vjp when the caller replays a segment of steps anyway (checkpointing). */
int sphb_sim_tape_reserve(sphb_sim* sim, int slots);

/*! One step (as sphb_sim_step, fixed time step required) that also records in `slot` everything the step's adjoint
 *  reads: the post-sync state, lists, derived fields and the adjoint tape. */
int sphb_sim_step_record(sphb_sim* sim, int slot);

/*! sphb_sim_step_vjp for the step recorded in `slot`, without recomputing its forces. Leaves the simulation holding
 *  that step's recorded post-force state. */
int sphb_sim_step_vjp_recorded(sphb_sim* sim, int slot, const double* const* adj_post, double* const* adj_pre,
                               double* alphamax_bar);

/* ---------------------------------------------------------------------------------------------------------------- */
/* 4. Batched ensemble                                                                                              */
/* ---------------------------------------------------------------------------------------------------------------- */

/*! Many independent simulations stepped together: every stage of the VE step runs as one launch over all instances,
 *  the step has no host synchronisation, and sphb_ensemble_step replays it as one captured CUDA graph. Each instance
 *  evolves exactly as an sphb_sim of the same particles and parameters would. No counterpart in the reference (it
 *  runs one simulation per process). */
typedef struct sphb_ensemble sphb_ensemble;

/*! num instances (1..254) with sizes[k] particles each, in one periodic box shared by all. params[k] per instance:
 *  gamma, mui, minDt and minDt_m1 may differ; ng0, ngmax, precision, sinc_index, bucket_focus, Kcour, Krho and the
 *  AV constants must be equal (SPHB_ERR_ARG otherwise). Open boundaries are not supported (SPHB_ERR_ARG). */
int sphb_ensemble_create(sphb_ensemble** ens, int num, const size_t* sizes, const sphb_box* box,
                         const sphb_params* params);

int sphb_ensemble_destroy(sphb_ensemble* ens);

/*! The 14 conserved fields and ids of instance k (as sphb_sim_upload). */
int sphb_ensemble_upload(sphb_ensemble* ens, int k, const double* const* fields, const uint64_t* id, int on_device);

/*! Sort every instance into SFC order and build its trees (host-driven; after all uploads). */
int sphb_ensemble_initial_sync(sphb_ensemble* ens);

/*! Rebuild the per-instance focus trees from the current particle order (outside the captured step). */
int sphb_ensemble_rebuild_trees(sphb_ensemble* ens);

/*! Block sizes (multiples of 32, at most 256; the AV switches of a mixed-precision ensemble at most 384) of the five
 *  J-loop launches: XMass, VeDefGradh+EOS, IAD+divv/curlv, AV switches, MomentumEnergy. */
int sphb_ensemble_set_threads(sphb_ensemble* ens, const int* threads5);

/*! Time every J-loop at 64, 128 and 256 threads per block (the AV switches of a mixed-precision ensemble also at
 *  384) on the current state, keep the fastest, and write the choice to threads5_out (5 ints, may be null). The
 *  particle state is unchanged. */
int sphb_ensemble_autotune(sphb_ensemble* ens, int* threads5_out);

/*! Advance every instance by steps steps; use_graph != 0 replays one captured step (captured on first use). */
int sphb_ensemble_step(sphb_ensemble* ens, int steps, int use_graph);

/*! Stage times in ms of the last step (9 floats: sync, neighbours, XMass, VeDefGradh + EOS, IAD + divv/curlv, AV
 *  switches, MomentumEnergy, conserved sums, integration), from CUDA events recorded inside the step. Waits for the
 *  stream. SPHB_ERR_STATE before the first step. No counterpart in the reference. */
int sphb_ensemble_stage_times(sphb_ensemble* ens, float* out);

/*! How the neighbour stage ran since the last upload or initial sync (the mode of each step is chosen on the
 *  device from the skin rows' state, sphb_params.nb_skin of the first instance): out[0] tree searches of every group,
 *  out[1] skin-row builds (each also counted in out[0]), out[2] steps served by refiltering the rows, out[3] groups
 *  deferred to the tree search. All zero when nb_skin is 0. No counterpart in the reference. */
int sphb_ensemble_search_stats(sphb_ensemble* ens, uint64_t* out);

/*! Number of particles of instance k. */
size_t sphb_ensemble_size(const sphb_ensemble* ens, int k);

/*! Field of instance k by name (as sphb_sim_get_field), n_k doubles in host memory, in the instance's SFC order. */
int sphb_ensemble_get_field(sphb_ensemble* ens, int k, const char* name, double* out);

/*! Scalars of instance k: minDt, minDt_m1, ttot, etot, ecin, eint, linmom, angmom, totalNeighbors (9 doubles; the
 *  conserved quantities of the last force computation). */
int sphb_ensemble_scalars(sphb_ensemble* ens, int k, double* out);

/*! The CUDA stream of the ensemble. */
void* sphb_ensemble_stream(sphb_ensemble* ens);

/* ---------------------------------------------------------------------------------------------------------------- */
/* 5. Measurement helper                                                                                            */
/* ---------------------------------------------------------------------------------------------------------------- */

/*! Measure the CUDA-core FMA throughput of the current device: which = 0 for FP32, 1 for FP64, 2 for packed FP32
 *  (two FP32 FMAs per instruction, sm_100 FFMA2). Runs a short register-resident FMA kernel over all SMs and returns
 *  the achieved TFLOP/s (2 flops per FMA) in *tflops.
 *  No counterpart in the reference: it supplies the roofline denominator of the FP32/FP64-bound neighbour sums. */
int sphb_probe_fma_peak(int which, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* SPHB200_H */
