/*
 * icempm_host.h -- C entry points of the host library (libicempm_host.so),
 * the C++ layer of icempm_multi_b200/host that mirrors the reference's host
 * classes (icy::Model, GPU_Implementation5, HostSideSOA, SnapshotManager).
 * These are the parts a non-C++ host needs without the classes: reading the
 * reference's HDF5 point clouds and the frame-log number format.  Status
 * codes are those of icempm.h; icy_host_last_error() describes the last
 * failure on the calling thread.
 */
#ifndef ICEMPM_HOST_H
#define ICEMPM_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "icempm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of points (the length of "llGrainIDs") of an HDF5 point cloud
   (simulation/snapshotmanager.cpp:34-38).  ICY_ERR_FILE if it cannot be read. */
int icy_h5_count(const char *path, unsigned *n_points);

/*
 * SnapshotManager::LoadRawPoints without the device part
 * (simulation/snapshotmanager.cpp:29-109): reads "x", "y" and "llGrainIDs"
 * into the HSSOA lines (utility word = the 64-bit grain value), the "volume"
 * attribute as a float, then applies icy_scene_place.  *n_points receives
 * the points kept.  ICY_ERR_CAPACITY if the file has more than `capacity`.
 */
int icy_h5_load(icy_sim_params *p, const char *path, double *hssoa, unsigned capacity,
                unsigned *n_points);

/* Shortest round-trip text of v as the fmt library's "{}" writes a double
   (the indenter_force.csv number format, simulation/model.cpp:79). */
int icy_format_double(double v, char *buf, size_t cap);

const char *icy_host_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
