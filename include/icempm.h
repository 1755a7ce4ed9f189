/*
 * icempm.h -- C-ABI of the B200-native MLS-MPM step library (libicempm_b200.so).
 *
 * The library replaces the per-step hot path of iceMPM_multi run as ONE
 * partition on ONE GPU: grid reset, P2G scatter, grid-node update with the
 * rigid indenter, G2P gather fused with the Drucker-Prager return mapping.
 * Every entry point returns an int status: 0 = OK, otherwise one of the
 * ICY_ERR_* codes below.  No C++ exception crosses this boundary; the C++
 * host layer (icempm_multi_b200/host) turns non-zero codes into
 * std::runtime_error, as the reference does for every CUDA failure
 * (simulation/gpu_partition.cu:19-20,151-156 and similar).
 *
 * Particle data uses the reference HSSOA layout: 16 lines of doubles, line
 * stride = capacity (simulation/hssoa/host_side_soa.h:52-74), line order as
 * in simulation/parameters_sim.h:27-35.  Line 0 holds the 64-bit utility word
 * bit-cast into a double (grain id bits 0-15, crushed 0x10000, disabled
 * 0x20000, liquid 0x40000; simulation/kernels.cuh:12-14).
 */
#ifndef ICEMPM_H
#define ICEMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* status codes                                                         */
/* ------------------------------------------------------------------ */
enum {
    ICY_OK = 0,
    /* device error byte values kept from the reference
       (simulation/kernels.cuh:94-97 and :506) */
    ICY_ERR_NO_SPACE = 5,          /* capacity exceeded                        */
    ICY_ERR_OUT_OF_GRID_XLO = 70,  /* particle stencil left the grid: x < -halo */
    ICY_ERR_OUT_OF_GRID_YLO = 71,  /* y < 0                                     */
    ICY_ERR_OUT_OF_GRID_XHI = 72,  /* x > GridX + halo - 3                      */
    ICY_ERR_OUT_OF_GRID_YHI = 73,  /* y > GridY - 3                             */
    /* host-side errors of this library */
    ICY_ERR_INVALID_ARGUMENT = 100,
    ICY_ERR_CUDA = 101,            /* a CUDA runtime call failed                */
    ICY_ERR_OUT_OF_MEMORY = 102,   /* device allocation refused or over budget  */
    ICY_ERR_JSON = 103,            /* configuration text is not a JSON object   */
    ICY_ERR_CONFIG_MISSING = 104,  /* "InputRawPoints" missing                  */
    ICY_ERR_FILE = 105,            /* configuration file not found / unreadable */
    ICY_ERR_CAPACITY = 106,        /* host HSSOA capacity too small             */
    ICY_ERR_POINT_COUNT = 107,     /* active point count changed                */
    ICY_ERR_TIMEOUT = 108,         /* a bounded device wait gave up             */
    ICY_ERR_NOT_SUPPORTED = 109,
    ICY_ERR_DRIFT = 110            /* FP32: a point moved further in one step than the
                                      grid update fused into the tile kernel allows
                                      (excluded by the test of the step before)   */
};

/* ------------------------------------------------------------------ */
/* SimParams                                                            */
/* ------------------------------------------------------------------ */
/*
 * Field-for-field mirror of icy::SimParams (simulation/parameters_sim.h:37-85):
 * same names, types and order, so the structs have the same layout and a
 * caller holding an icy::SimParams may pass a pointer to it directly
 * (the layout is checked by static_assert in oracle/ref_driver_common.h).
 */
typedef struct icy_sim_params {
    int n_indenter_subdivisions;
    int tpb_P2G, tpb_Upd, tpb_G2P;
    int nPtsTotal;
    int GridXTotal, GridY, GridTotal;
    double GridXDimension;
    double InitialTimeStep, SimulationEndTime;
    int UpdateEveryNthStep;
    int SimulationStep;
    double SimulationTime;
    double Gravity, Density, WaterDensity, PoissonsRatio, YoungsModulus;
    double lambda, mu, kappa;
    double IceCompressiveStrength, IceTensileStrength, IceShearStrength, IceTensileStrength2;
    double NACC_beta, NACC_M, NACC_Msq;
    double DP_tan_phi, DP_threshold_p;
    double IndDiameter, IndRSq, IndVelocity, IndDepth;
    double cellsize, cellsize_inv, Dp_inv;
    double xmin, xmax, ymin, ymax;
    int nxmin, nxmax, nymin, nymax;
    double ParticleVolume, ParticleMass, WaterParticleMass, ParticleViewSize;
    double indenter_x, indenter_x_initial, indenter_y, indenter_y_initial;
    double Volume;
    int SetupType;
    double GrainVariability;
    int GridHaloSize;
    double ExtraSpaceForIncomingPoints;
    double PointsTransferBufferFraction;
    double RebalanceThresholdFreeSpaceRemaining;
    double RebalanceThresholdDisabledPercentage;
    int PointTransferFrequency;
    int nPartitions;
    int VectorCapacity_transfer;
    double dt_vol_Dpinv, dt_Gravity, vmax, vmax_squared;
    int gbOffset;
} icy_sim_params;

/* HSSOA line indices (simulation/parameters_sim.h:27-35) */
enum {
    ICY_IDX_UTILITY = 0, ICY_IDX_P = 1, ICY_IDX_Q = 2, ICY_IDX_JP_INV = 3,
    ICY_POSX = 4, ICY_VELX = 6, ICY_FE00 = 8, ICY_BP00 = 12, ICY_N_PTS_ARRAYS = 16
};
/* utility-word status bits (simulation/kernels.cuh:12-14) */
#define ICY_STATUS_CRUSHED  0x10000LL
#define ICY_STATUS_DISABLED 0x20000LL
#define ICY_STATUS_LIQUID   0x40000LL

/* SimParams::Reset -- defaults (simulation/parameters_sim.cpp:5-60). */
void icy_params_reset(icy_sim_params *p);
/* SimParams::ComputeLame (simulation/parameters_sim.cpp:128-133). */
void icy_params_compute_lame(icy_sim_params *p);
/* SimParams::ComputeCamClayParams2 (simulation/parameters_sim.cpp:155-165). */
void icy_params_compute_camclay(icy_sim_params *p);
/* SimParams::ComputeHelperVariables (simulation/parameters_sim.cpp:135-153). */
void icy_params_compute_helpers(icy_sim_params *p);
/*
 * SimParams::ParseFile on in-memory JSON text (simulation/parameters_sim.cpp:63-126):
 * the same keys, DP_phi in degrees converted to DP_tan_phi, then
 * ComputeCamClayParams2 + ComputeHelperVariables.  The "InputRawPoints"
 * string is copied into raw_points (NUL-terminated, truncated to cap-1).
 * Returns ICY_ERR_JSON if the text is not a JSON object and
 * ICY_ERR_CONFIG_MISSING if "InputRawPoints" is absent (the parameters are
 * still updated in that case, as in the reference, which throws after parsing).
 */
int icy_params_parse_json(icy_sim_params *p, const char *json_text,
                          char *raw_points, size_t cap);
/* SimParams::ParseFile on a file path (ICY_ERR_FILE if it does not exist). */
int icy_params_parse_file(icy_sim_params *p, const char *path,
                          char *raw_points, size_t cap);

/* ------------------------------------------------------------------ */
/* scene set-up (host only)                                             */
/* ------------------------------------------------------------------ */
/*
 * Seeded synthetic ice block, replacing the HDF5 point cloud read by
 * SnapshotManager::LoadRawPoints (simulation/snapshotmanager.cpp:29-121):
 * a block of block_w x block_h metres, ppc particles per cell of size
 * p->cellsize, each jittered uniformly inside its cell by a counter-based
 * hash of (seed, cell, k); grain ids from a seeded Voronoi partition with
 * n_grains sites (0 = all grain 0).  Writes x, y and the utility word into
 * the HSSOA (line stride = capacity), then applies LoadRawPoints' placement
 * rules: block centred in x and lifted by 2h (:71-78), points sorted by
 * cell (:81, host_side_soa.cpp:50-61), Fe = I and Jp_inv = 1 (:82,
 * host_side_soa.cpp:94-105), indenter start (:84-105), ParticleVolume =
 * Volume/N and ComputeHelperVariables (:108-109).  On return *n_points holds N.
 * Returns ICY_ERR_CAPACITY if N > capacity.
 */
int icy_scene_block(icy_sim_params *p, double block_w, double block_h, int ppc,
                    uint64_t seed, int n_grains, double *hssoa, unsigned capacity,
                    unsigned *n_points);
/* Number of points icy_scene_block would create (for sizing the HSSOA). */
unsigned icy_scene_block_count(const icy_sim_params *p, double block_w, double block_h, int ppc);
/*
 * The placement half of SnapshotManager::LoadRawPoints
 * (simulation/snapshotmanager.cpp:62-109) for a point cloud whose x, y and
 * utility lines are already in the HSSOA (*n_points points, e.g. read from
 * the reference's HDF5 files): block extent into xmin..ymax, block centred
 * in x and lifted by 2h, RemoveDisabledAndSort (points with the disabled bit
 * dropped, the rest stable-sorted by ProxyPoint::getCellIndex), the other
 * lines cleared and InitializeBlock (Fe = I, Jp_inv = 1), indenter start,
 * nPtsTotal, Volume = volume, ParticleVolume = volume / (points loaded) and
 * ComputeHelperVariables.  On return *n_points holds the points kept.
 */
int icy_scene_place(icy_sim_params *p, double *hssoa, unsigned capacity, unsigned *n_points,
                    double volume);

/*
 * Page-locked host memory for an HSSOA buffer, as HostSideSOA::Allocate
 * takes it with cudaMallocHost (simulation/hssoa/host_side_soa.cpp:64-79);
 * the memory is cleared.  Lets a host that links only this library keep its
 * transfers asynchronous.  icy_host_free(NULL) is a no-op.
 */
int icy_host_alloc(size_t bytes, void **ptr);
int icy_host_free(void *ptr);

/* ------------------------------------------------------------------ */
/* one simulation instance on one device                                */
/* ------------------------------------------------------------------ */
typedef struct icy_mpm icy_mpm;

/* Precision of the device state. */
enum { ICY_PRECISION_FP64 = 0, ICY_PRECISION_FP32_SPLIT = 1 };

/*
 * GPU_Partition::initialize + allocate for a single partition
 * (simulation/gpu_partition.cu:113-197): creates the stream, device particle
 * SoA for `capacity` points, the grid covering x in [-halo, GridX+halo) and
 * y in [0, GridY), the indenter accumulator and the status word.
 */
int icy_mpm_create(const icy_sim_params *p, int device, unsigned capacity,
                   int precision, icy_mpm **out);
/* GPU_Partition::~GPU_Partition (simulation/gpu_partition.cu:88-111). */
int icy_mpm_destroy(icy_mpm *h);
/* Run the instance's work on an external cudaStream_t (NULL = own stream). */
int icy_mpm_set_stream(icy_mpm *h, void *cuda_stream);
void *icy_mpm_get_stream(icy_mpm *h);
/* GPU_Partition::update_constants (simulation/gpu_partition.cu:200-208):
   copy the parameters and clear the device error code. */
int icy_mpm_update_constants(icy_mpm *h, const icy_sim_params *p);
/* GPU_Implementation5::transfer_ponts_to_device for one partition
   (simulation/gpu_implementation5.cpp:346-356, gpu_partition.cu:49-68). */
int icy_mpm_transfer_points_to_device(icy_mpm *h, const double *hssoa,
                                      unsigned capacity, unsigned size);
/*
 * GPU_Implementation5::transfer_from_device for one partition
 * (simulation/gpu_implementation5.cpp:360-436, gpu_partition.cu:16-46):
 * copies the 16 lines back in the order they were uploaded, the indenter
 * accumulator (2*n_indenter_subdivisions doubles, may be NULL) and the device
 * error code; synchronises.  Returns the device error code if it is set and
 * ICY_ERR_POINT_COUNT if the number of non-disabled points differs from
 * p->nPtsTotal.  *size receives the number of points.
 */
int icy_mpm_transfer_from_device(icy_mpm *h, double *hssoa, unsigned capacity,
                                 unsigned *size, double *indenter_force_bins);
/* GPU_Partition::reset_indenter_force_accumulator (gpu_partition.cu:212-217). */
int icy_mpm_reset_indenter_force_accumulator(icy_mpm *h);
/* Sum of the indenter accumulator bins, read back synchronously (force[2]). */
int icy_mpm_indenter_force(icy_mpm *h, double *force_xy, double *bins);

/* Per-phase calls of GPU_Implementation5 (simulation/gpu_implementation5.h:44-51). */
int icy_mpm_reset_grid(icy_mpm *h);                         /* gpu_partition.cu:221-228 */
int icy_mpm_p2g(icy_mpm *h);                                /* gpu_partition.cu:230-242 */
int icy_mpm_receive_halos(icy_mpm *h);                      /* no-op: one partition     */
int icy_mpm_update_nodes(icy_mpm *h, double indenter_x,
                         double indenter_y, double simulation_time); /* :244-257 */
int icy_mpm_g2p(icy_mpm *h, int recordPQ, int enablePointTransfer); /* :259-293;
                                   enablePointTransfer must be 0 (one domain) */
int icy_mpm_receive_points(icy_mpm *h);                     /* no-op: one partition     */

/*
 * The sub-step loop of icy::Model::Step (simulation/model.cpp:38-54) on the
 * device, with no host synchronisation: for k = 0..nsteps-1,
 *   t += dt;  indenter_x = indenter_x_initial + t*IndVelocity;
 *   reset grid; P2G; grid update(indenter at (indenter_x, indenter_y));
 *   G2P(recordPQ = ((step0 + k) % UpdateEveryNthStep == 0)).
 * `*sim_time` is advanced in place.  Work is queued on the instance stream
 * (use icy_mpm_synchronize or a download to wait).
 */
int icy_mpm_step(icy_mpm *h, int step0, int nsteps, double *sim_time);
int icy_mpm_synchronize(icy_mpm *h);
/* Read (synchronously) and return the device error code (0 if none). */
int icy_mpm_status(icy_mpm *h);
/*
 * Tuning options of an instance (no counterpart in the reference, whose
 * launch shapes come from tpb_* in SimParams):
 *   "resort_every"  re-bin the points by tile every N steps (0 = only after upload)
 *   "tiled"         1 = binned, tile-staged kernels (default); 0 = one thread per
 *                   point / node, unsorted (the reference's kernel structure)
 *   "pipe"          1 = the fused step kernel is fed by a producer warp with
 *                   bulk copies into a shared-memory ring (default 0)
 *   "pipe_fault_test" 1 = (tests of the timeout path) the producer leaves the
 *                   ring's first stage unfilled: every wait on it gives up
 *                   after 1 s and the next download reports ICY_ERR_TIMEOUT
 *   "fuse_update"   FP32 split precision: 1 = the grid update of the next step is
 *                   done inside the tile kernel, node tile by node tile, by the CTA
 *                   that finishes its last neighbouring cell tile; a step in which
 *                   a point could leave its tile's staged margin falls back to the
 *                   list-driven update kernel; 0 = always the update kernel
 *                   (default: the counting at every tile's end costs the tile
 *                   kernel more than the update kernel takes)
 *   "tile_shape"    FP32 split precision: cells per tile of the binned kernels,
 *                   0 = 32 x 8 (default), 1 = 16 x 16, 2 = 16 x 8; the points are
 *                   binned again at the next step (icempm_multi_b200/autotune.py
 *                   times the shapes on a workload); the fused grid update runs
 *                   with 32 x 8 tiles only; FP64 instances: 0 only
 *   "profile_every" n = icy_mpm_profile times every n-th launch of each kernel
 *                   (default 1; every re-binning is timed whatever n); an event
 *                   pair on the stream costs the step loop a few microseconds, so
 *                   sampling keeps a profiled run close to an unprofiled one
 */
int icy_mpm_set_option(icy_mpm *h, const char *name, double value);

/* Number of kernels this instance launched since creation. */
int64_t icy_mpm_kernel_launches(icy_mpm *h);
/*
 * Device counters since creation (synchronous read; no counterpart in the
 * reference): P2G contributions of points that had left the cell they were
 * binned into (a re-binning hint), FP32 tile launches that fused the grid
 * update, and FP32 tile launches that fell back to the update kernel because
 * a point could leave its tile's staged margin (option "fuse_update").
 * Any pointer may be NULL.
 */
int icy_mpm_counters(icy_mpm *h, int64_t *moved_points, int64_t *fused_launches,
                     int64_t *fallback_launches);
/*
 * Per-kernel timing with CUDA events recorded on the instance stream around
 * every kernel launch, or every n-th launch of each kernel with the option
 * "profile_every" (the event pairs of GPU_Partition::record_timings,
 * simulation/gpu_partition.cu:344-401, but per kernel and read only on
 * request).  enable=1 clears and starts recording, enable=0 stops.
 */
int icy_mpm_profile(icy_mpm *h, int enable);
/*
 * Synchronises and returns up to `max` kernel entries: names (max x 48 chars,
 * NUL-terminated), total milliseconds and counts of the timed launches;
 * *count receives the number of distinct kernels recorded.
 */
int icy_mpm_profile_read(icy_mpm *h, int max, char *names, double *ms_total,
                         int64_t *launches, int *count);

/* ------------------------------------------------------------------ */
/* batches of independent instances                                     */
/* ------------------------------------------------------------------ */
/*
 * No counterpart in the reference (which runs one scenario per process).
 * A batch advances many independent floe scenarios together on one GPU:
 * every member is an FP32 split-precision instance with its own parameters,
 * grid and points, and one batch step is four kernel launches whatever the
 * number of members (clocks, grid update, mark clearing, tile kernel over
 * the (member, tile) work list), replayed as a CUDA graph per step count.
 * Each member keeps its own simulation time and step index on the device,
 * so members admitted at different times progress independently.
 */
typedef struct icy_batch icy_batch;
int icy_batch_create(int device, int max_instances, icy_batch **out);
int icy_batch_destroy(icy_batch *b);
/* Admit a scenario (SimParams + HSSOA, line stride = capacity, `size` points);
   *slot receives its member index.  ICY_ERR_NO_SPACE if all slots are taken. */
int icy_batch_add(icy_batch *b, const icy_sim_params *p, const double *hssoa,
                  unsigned capacity, unsigned size, int *slot);
/* Admission without waiting: the upload, conversion and binning run on the
   batch's side stream while the rounds already queued go on; the next round
   waits for them.  The HSSOA buffer must stay valid and unchanged until
   icy_batch_synchronize returns or a round queued after this call has
   finished.  No counterpart in the reference (one scenario per process). */
int icy_batch_add_async(icy_batch *b, const icy_sim_params *p, const double *hssoa,
                        unsigned capacity, unsigned size, int *slot);
/* Take a member out of the batch after the work already queued: its state
   (HSSOA in upload order, when hssoa is not NULL), indenter bins (when bins
   is not NULL), simulation time and step index are copied to the host on the
   side stream while later rounds run without it (a page-locked hssoa lets
   the call return at once; a pageable one makes it wait for the queued
   rounds).  The slot stays reserved until icy_batch_collect reports the copy
   done, and fills `bins` then; the buffers must stay valid until then.  No
   counterpart in the reference. */
int icy_batch_retire(icy_batch *b, int slot, double *hssoa, unsigned capacity, double *bins);
/* Finish a retirement: *done = 0 if the copy is still running (wait = 0),
   else *done = 1, the member's size, time and step, its device status code
   as the return value (or ICY_ERR_POINT_COUNT as for
   icy_mpm_transfer_from_device), and its slot and device memory are freed. */
int icy_batch_collect(icy_batch *b, int slot, int wait, int *done, unsigned *size,
                      double *sim_time, int64_t *step);
/* Free a member's slot and device memory. */
int icy_batch_remove(icy_batch *b, int slot);
/* Advance every member by nsteps sub-steps of icy::Model::Step (asynchronous). */
int icy_batch_step(icy_batch *b, int nsteps);
/* Download one member: HSSOA in its upload order, indenter bins (may be
   NULL), its simulation time and next step index (may be NULL); synchronises. */
int icy_batch_download(icy_batch *b, int slot, double *hssoa, unsigned capacity,
                       unsigned *size, double *bins, double *sim_time, int64_t *step);
int icy_batch_synchronize(icy_batch *b);
/* Block until at most `in_flight` of the icy_batch_step calls made so far are
   unfinished on the device (0: all finished), so that a host loop can queue
   the next round while the current one runs.  The last 8 calls are tracked:
   a larger in_flight waits as for 7. */
int icy_batch_wait_steps(icy_batch *b, int in_flight);
/* Set a member's simulation time and next step index (and its indenter
   position x0 + t V), e.g. to resume a member evicted with
   icy_batch_download at that time and step. */
int icy_batch_set_clock(icy_batch *b, int slot, double sim_time, int64_t step);
/* "resort_every" (steps between re-binning, 0 = never), "tile_ctas"
   (persistent CTAs of the tile kernel), "update_ctas" (CTAs of the grid
   update); the CTA counts take effect from the next step call (the captured
   graphs are dropped); "tile_shape" (the members' cells per tile, as the
   instance option; only while the batch has no members, else
   ICY_ERR_NOT_SUPPORTED).  icempm_multi_b200/autotune.py picks them by timing. */
int icy_batch_set_option(icy_batch *b, const char *name, double value);
/* Live members, their total points, kernels launched so far, the batch stream. */
int icy_batch_info(icy_batch *b, int *live, int64_t *points, int64_t *kernel_launches,
                   void **stream);
/* Device bytes of one member. */
int64_t icy_batch_device_bytes(icy_batch *b, int slot);
/* Device bytes an instance of this size and precision allocates. */
int64_t icy_mpm_device_bytes(const icy_sim_params *p, unsigned capacity, int precision);
/* Grows the memory pool that instances and batch members of `device` allocate
   from to at least `bytes`, kept for them (no counterpart in the reference).
   A server that reserves its budget up front admits requests without mapping
   new device memory while rounds run (about 9 ms per admission otherwise). */
int icy_mpm_reserve(int device, int64_t bytes);

/* ------------------------------------------------------------------ */
/* one instance in slabs of grid columns (partitions)                   */
/* ------------------------------------------------------------------ */
/*
 * GPU_Implementation5 with several partitions
 * (simulation/gpu_implementation5.cpp:31-204,221-326): the grid's columns
 * are cut into slabs, each partition holding its columns plus GridHaloSize
 * columns on both sides and the points whose stencil base lies in its
 * columns, on its own device (several on one device, as the reference
 * allows, or one device each with peer access between neighbours).  FP64,
 * one thread per point / node (the reference's kernel structure).  Per
 * sub-step: P2G; the 2*GridHaloSize boundary columns of mass and momentum
 * copied to each neighbour and added there (the reference's
 * receive_halos); grid update; G2P; every UpdateEveryNthStep /
 * PointTransferFrequency sub-steps, points more than 3 columns past their
 * slab move to the neighbour (packed, then appended by the neighbour from
 * the sender's memory: the reference's receive_points).  Results match the
 * one-domain path within FP64 round-off (the order of the sums differs);
 * each node's indenter force is counted once, by the partition owning its
 * column (the reference adds the boundary columns' forces in both).
 */
typedef struct icy_part icy_part;
/* The split of GPU_Implementation5::split_hssoa_into_partitions
   (gpu_implementation5.cpp:284-326): the HSSOA's points (sorted by cell, as
   LoadRawPoints leaves them) in equal shares, each boundary at the x cell of
   the first point of the next share.  Per partition: first column x0[i],
   columns width[i], first point first[i], points count[i].
   ICY_ERR_INVALID_ARGUMENT if a slab would be narrower than 2*GridHaloSize
   columns (its boundary regions would not cover what its neighbours'
   points can reach). */
int icy_part_plan(const icy_sim_params *p, const double *hssoa, unsigned capacity, unsigned size,
                  int n_partitions, int *x0, int *width, unsigned *first, unsigned *count);
/* n_partitions partitions, partition i on device devices[i] (NULL: all on
   device 0), each with room for capacity_per_partition points (points that
   move in are appended; ICY_ERR_NO_SPACE, the reference's code 5, when full).
   Neighbours on different devices need peer access (ICY_ERR_NOT_SUPPORTED). */
int icy_part_create(const icy_sim_params *p, int n_partitions, const int *devices,
                    unsigned capacity_per_partition, icy_part **out);
/* Split the HSSOA (line stride = capacity) by icy_part_plan and upload. */
int icy_part_upload(icy_part *h, const double *hssoa, unsigned capacity, unsigned size);
/* Sub-steps step0 .. step0+nsteps-1 of icy::Model::Step (model.cpp:38-54),
   queued on the partitions' streams; *sim_time is advanced. */
int icy_part_step(icy_part *h, int step0, int nsteps, double *sim_time);
/* All points back in upload order (synchronises), the indenter force bins
   summed over the partitions (may be NULL), *size = points uploaded; the
   first partition's device error code, ICY_ERR_POINT_COUNT if points were
   lost. */
int icy_part_download(icy_part *h, double *hssoa, unsigned capacity, unsigned *size, double *bins);
/* Partition `part`: first column, columns, points in its slots (moved-away
   slots included), device. */
int icy_part_info(icy_part *h, int part, int *x0, int *width, unsigned *count, int *device);
int icy_part_destroy(icy_part *h);

/* ------------------------------------------------------------------ */
/* stepping without allocation                                          */
/* ------------------------------------------------------------------ */
/*
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- e.g. a plug-in inside a host framework that owns all device
 * memory through its own pool and forbids cudaMalloc / cudaFree (which may
 * synchronise the device), or code on a latency-critical path that must not
 * allocate after start-up.  Runs nsteps sub-steps of icy::Model::Step
 * (simulation/model.cpp:38-54) on a particle buffer the caller keeps in
 * device memory: d_hssoa holds the 16 HSSOA lines with a line stride of
 * `pitch` doubles and n points, and is updated in place in its own order.
 * d_indenter_bins (2*n_indenter_subdivisions doubles in device memory, or
 * NULL) accumulates the indenter force.  Work is queued on `stream` (NULL =
 * the default stream); the call then synchronises that stream and returns
 * the device error code (0, or the reference's 70..73).  n may be at most
 * INT_MAX.  If a CUDA call fails part way, the call waits for the sub-steps
 * already queued, leaves *sim_time at the end of the last of them (so the
 * caller knows how far d_hssoa advanced) and returns ICY_ERR_CUDA.
 *
 * It runs the one-thread-per-item FP64 kernels (the reference's own kernel
 * structure: global FP64 atomics, no binning, which would need a second
 * particle buffer), about half the speed of the binned, tile-staged path of
 * icy_mpm_step on the same instance.
 *
 * It allocates nothing: the grid (5 arrays of GridY*(GridX+2*halo) doubles)
 * and the status word live in one file-scope device array of
 * ICY_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit.  Grids that need more return ICY_ERR_CAPACITY (icy_last_error says
 * how much was needed); the limit allows about 838,000 grid nodes.  The
 * first call on each device resolves the array's device address, so make
 * that first call before any stream capture.  All calls share the array and
 * each clears what must start at zero; calls that overlap on the GPU race.
 */
#define ICY_NOALLOC_SCRATCH_BYTES (32u << 20)
int icy_step_noalloc(const icy_sim_params *p, double *d_hssoa, unsigned pitch, unsigned n,
                     int step0, int nsteps, double *sim_time, double *d_indenter_bins,
                     void *stream);

/* Library build description, e.g. "icempm_b200 sm_100a". */
const char *icy_version(void);
/* Text of the last error recorded on the calling thread ("" if none). */
const char *icy_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* ICEMPM_H */
