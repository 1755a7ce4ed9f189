/*
 * oracle.h -- CPU parity oracle for the MLS-MPM hot path.
 *
 * TEST INFRASTRUCTURE.  A serial, deterministic FP64 restatement in plain C
 * of the reference kernels (simulation/kernels.cuh:24-122 P2G,
 * :164-301 grid update, :305-414 G2P, :521-674 SVD/plasticity,
 * simulation/helper_math.cuh:27-140, simulation/givens.cuh:67-166).  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it,
 * and only as the checker; the product never links or calls it.
 *
 * Arithmetic follows the reference expressions term by term with the Eigen
 * semantics spelled out in oracle/refshim/eigen/Eigen/Core (linear
 * reductions, (s*A)*B for scalar*(A*B), normalize of a zero vector is a
 * no-op).  Compiled without FMA contraction (-ffp-contract=off), it agrees
 * bit for bit with the reference sources compiled for the host
 * (oracle/_ref/libref_host.so) run on one thread.
 *
 * P2G accumulates particles in index order, nodes in (i outer, j inner)
 * order.  Grid layout is the reference's single-partition layout: node
 * (gx, gy), gx in [-halo, GridX+halo), gy in [0, GridY), at
 * (gx + halo)*GridY + gy (simulation/kernels.cuh:114-120, :191).
 *
 * Out-of-grid particles: the reference records code 70..73 and still writes
 * out of bounds (simulation/kernels.cuh:94-97); the oracle records the same
 * code and skips that particle's P2G and G2P instead.
 */
#ifndef ICEMPM_ORACLE_H
#define ICEMPM_ORACLE_H

#include "../include/icempm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* number of grid nodes of one array: GridY*(GridX + 2*halo) */
long oracle_grid_nodes(const icy_sim_params *p);

/* P2G into zeroed grid arrays gm/gpx/gpy (simulation/kernels.cuh:46-122).
   Returns the error code (0 or 70..73, last one wins as in the reference). */
int oracle_p2g(const icy_sim_params *p, const double *soa, unsigned pitch, unsigned n,
               double *gm, double *gpx, double *gpy);

/* grid update in place: gpx/gpy become velocities (simulation/kernels.cuh:164-301).
   bins: 2*n_indenter_subdivisions accumulator (may be NULL). */
void oracle_update(const icy_sim_params *p, double *gm, double *gpx, double *gpy,
                   double ind_x, double ind_y, double *bins);

/* G2P + plasticity (simulation/kernels.cuh:305-414).  Returns error code. */
int oracle_g2p(const icy_sim_params *p, double *soa, unsigned pitch, unsigned n,
               const double *gvx, const double *gvy, int recordPQ);

/*
 * nsteps sub-steps of icy::Model::Step for one partition
 * (simulation/model.cpp:38-54): t += dt; indenter_x = x0 + t*v; zero grid;
 * P2G; update; G2P(recordPQ = (step0+k) % UpdateEveryNthStep == 0).
 * *sim_time is advanced in place; bins accumulate (caller zeroes them).
 * Returns the first non-zero error code (the run stops there).
 */
int oracle_run(const icy_sim_params *p, double *soa, unsigned pitch, unsigned n,
               int step0, int nsteps, double *sim_time, double *bins);

/* ---- device-math pieces exposed for unit tests ---- */
/* Kirchhoff stress tau (row-major 2x2) of F (simulation/kernels.cuh:24-34). */
void oracle_kirchhoff(const icy_sim_params *p, const double F[4], double tau[4]);
/* p, q, Je of F (simulation/kernels.cuh:547-557). */
void oracle_pq(const icy_sim_params *p, const double F[4], double *ptr, double *qtr, double *Je);
/* SVD as the reference builds it (simulation/kernels.cuh:530-538,
   helper_math.cuh:81-140): U, V row-major 2x2, sigma[2]. */
void oracle_svd(const double F[4], double U[4], double sigma[2], double V[4]);
/* failure-surface test: returns 1 if the point is crushed (kernels.cuh:598-619). */
int oracle_failure(const icy_sim_params *p, int grain, double ptr, double qtr);
/* return mapping of one crushed point (kernels.cuh:540-545, 623-674): F, Jp in/out. */
void oracle_return_map(const icy_sim_params *p, double F[4], double *Jp,
                       double ptr, double qtr, double Je);

#ifdef __cplusplus
}
#endif
#endif
