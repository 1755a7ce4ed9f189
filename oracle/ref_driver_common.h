// ref_driver_common.h -- TEST INFRASTRUCTURE.
// Shared part of the two drivers that run the reference's own kernels
// (simulation/kernels.cuh, compiled unmodified from the reference tree) as
// one partition: static checks that icy_sim_params (include/icempm.h) has the
// exact layout of icy::SimParams, and the single-partition sizes that
// GPU_Partition::allocate / update_nodes use (simulation/gpu_partition.cu:137-197,
// :244-257, gpu_implementation5.cpp:329-342).
#pragma once
#include <cstddef>
#include "../include/icempm.h"

#define ICY_SAME_FIELD(f)                                                                  \
    static_assert(offsetof(icy::SimParams, f) == offsetof(icy_sim_params, f), #f " offset"); \
    static_assert(sizeof(((icy::SimParams *)0)->f) == sizeof(((icy_sim_params *)0)->f), #f " size");

ICY_SAME_FIELD(n_indenter_subdivisions) ICY_SAME_FIELD(tpb_P2G) ICY_SAME_FIELD(tpb_Upd)
ICY_SAME_FIELD(tpb_G2P) ICY_SAME_FIELD(nPtsTotal) ICY_SAME_FIELD(GridXTotal) ICY_SAME_FIELD(GridY)
ICY_SAME_FIELD(GridTotal) ICY_SAME_FIELD(GridXDimension) ICY_SAME_FIELD(InitialTimeStep)
ICY_SAME_FIELD(SimulationEndTime) ICY_SAME_FIELD(UpdateEveryNthStep) ICY_SAME_FIELD(SimulationStep)
ICY_SAME_FIELD(SimulationTime) ICY_SAME_FIELD(Gravity) ICY_SAME_FIELD(Density) ICY_SAME_FIELD(WaterDensity)
ICY_SAME_FIELD(PoissonsRatio) ICY_SAME_FIELD(YoungsModulus) ICY_SAME_FIELD(lambda) ICY_SAME_FIELD(mu)
ICY_SAME_FIELD(kappa) ICY_SAME_FIELD(IceCompressiveStrength) ICY_SAME_FIELD(IceTensileStrength)
ICY_SAME_FIELD(IceShearStrength) ICY_SAME_FIELD(IceTensileStrength2) ICY_SAME_FIELD(NACC_beta)
ICY_SAME_FIELD(NACC_M) ICY_SAME_FIELD(NACC_Msq) ICY_SAME_FIELD(DP_tan_phi) ICY_SAME_FIELD(DP_threshold_p)
ICY_SAME_FIELD(IndDiameter) ICY_SAME_FIELD(IndRSq) ICY_SAME_FIELD(IndVelocity) ICY_SAME_FIELD(IndDepth)
ICY_SAME_FIELD(cellsize) ICY_SAME_FIELD(cellsize_inv) ICY_SAME_FIELD(Dp_inv) ICY_SAME_FIELD(xmin)
ICY_SAME_FIELD(xmax) ICY_SAME_FIELD(ymin) ICY_SAME_FIELD(ymax) ICY_SAME_FIELD(nxmin) ICY_SAME_FIELD(nxmax)
ICY_SAME_FIELD(nymin) ICY_SAME_FIELD(nymax) ICY_SAME_FIELD(ParticleVolume) ICY_SAME_FIELD(ParticleMass)
ICY_SAME_FIELD(WaterParticleMass) ICY_SAME_FIELD(ParticleViewSize) ICY_SAME_FIELD(indenter_x)
ICY_SAME_FIELD(indenter_x_initial) ICY_SAME_FIELD(indenter_y) ICY_SAME_FIELD(indenter_y_initial)
ICY_SAME_FIELD(Volume) ICY_SAME_FIELD(SetupType) ICY_SAME_FIELD(GrainVariability) ICY_SAME_FIELD(GridHaloSize)
ICY_SAME_FIELD(ExtraSpaceForIncomingPoints) ICY_SAME_FIELD(PointsTransferBufferFraction)
ICY_SAME_FIELD(RebalanceThresholdFreeSpaceRemaining) ICY_SAME_FIELD(RebalanceThresholdDisabledPercentage)
ICY_SAME_FIELD(PointTransferFrequency) ICY_SAME_FIELD(nPartitions) ICY_SAME_FIELD(VectorCapacity_transfer)
ICY_SAME_FIELD(dt_vol_Dpinv) ICY_SAME_FIELD(dt_Gravity) ICY_SAME_FIELD(vmax) ICY_SAME_FIELD(vmax_squared)
ICY_SAME_FIELD(gbOffset)
static_assert(sizeof(icy::SimParams) == sizeof(icy_sim_params), "SimParams size");
static_assert(icy::SimParams::nPtsArrays == ICY_N_PTS_ARRAYS, "nPtsArrays");
static_assert(icy::SimParams::posx == ICY_POSX && icy::SimParams::velx == ICY_VELX &&
              icy::SimParams::Fe00 == ICY_FE00 && icy::SimParams::Bp00 == ICY_BP00 &&
              icy::SimParams::idx_Jp_inv == ICY_IDX_JP_INV, "SoA line indices");

// one partition: GridX_partition = GridXTotal, GridX_offset = 0,
// grid pitch >= GridY*(GridX + 6*halo) (gpu_partition.cu:148),
// updated nodes = GridY*(GridX + 2*halo) (gpu_partition.cu:247)
inline size_t ref_grid_pitch(const icy_sim_params *p) {
    return (size_t)p->GridY * (p->GridXTotal + 6 * p->GridHaloSize);
}
inline int ref_update_nodes(const icy_sim_params *p) {
    return p->GridY * (p->GridXTotal + 2 * p->GridHaloSize);
}
