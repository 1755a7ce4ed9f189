// icy_host.hpp -- C++ host layer over the C-ABI of include/icempm.h, with the
// class names, members and call order of the reference's host code so that
// its drivers (cli/main.cpp, gui/backgroundworker.cpp) compile against it:
//
//   icy::SimParams       simulation/parameters_sim.h:17-105
//   HostSideSOA          simulation/hssoa/host_side_soa.h:52-74
//   GPU_Implementation5  simulation/gpu_implementation5.h:25-59 (one partition, one GPU)
//   icy::Model           simulation/model.h:32-57, model.cpp:1-139
//   icy::SnapshotManager simulation/snapshotmanager.h:14-30 (LoadRawPoints; checkpoints)
//
// Every failing library call throws std::runtime_error carrying the library's
// message, as the reference throws on CUDA errors (simulation/gpu_partition.cu:19-20).
#pragma once

#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <fstream>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/icempm.h"

namespace icy {

// throws std::runtime_error("<what>: <library message> (status N)") when status != ICY_OK
void check(int status, const char *what);

// the few Eigen::Vector2d operations the reference's host code applies to positions and forces
struct Vector2d {
    double v[2] = {0, 0};
    Vector2d() = default;
    Vector2d(double x, double y) { v[0] = x; v[1] = y; }
    double &x() { return v[0]; }
    double &y() { return v[1]; }
    double x() const { return v[0]; }
    double y() const { return v[1]; }
    double &operator[](int i) { return v[i]; }
    double operator[](int i) const { return v[i]; }
    double norm() const { return std::sqrt(v[0] * v[0] + v[1] * v[1]); }
    void setZero() { v[0] = v[1] = 0; }
    Vector2d &operator+=(const Vector2d &o) { v[0] += o.v[0]; v[1] += o.v[1]; return *this; }
    Vector2d &operator/=(double s) { v[0] /= s; v[1] /= s; return *this; }
};

struct SimParams : public icy_sim_params {
    constexpr static double pi = 3.14159265358979323846;
    constexpr static int dim = 2;
    constexpr static int nGridArrays = 3;
    constexpr static size_t idx_utility_data = ICY_IDX_UTILITY;
    constexpr static size_t idx_P = ICY_IDX_P;
    constexpr static size_t idx_Q = ICY_IDX_Q;
    constexpr static size_t idx_Jp_inv = ICY_IDX_JP_INV;
    constexpr static size_t posx = ICY_POSX;
    constexpr static size_t velx = ICY_VELX;
    constexpr static size_t Fe00 = ICY_FE00;
    constexpr static size_t Bp00 = ICY_BP00;
    constexpr static size_t nPtsArrays = ICY_N_PTS_ARRAYS;

    SimParams() { Reset(); }
    void Reset() { icy_params_reset(this); }
    // parses the JSON configuration; returns "InputRawPoints" (throws if absent or unreadable)
    std::string ParseFile(std::string fileName);
    void ComputeLame() { icy_params_compute_lame(this); }
    void ComputeCamClayParams2() { icy_params_compute_camclay(this); }
    void ComputeHelperVariables() { icy_params_compute_helpers(this); }
    double PointsPerCell() const { return nPtsTotal / (Volume / (cellsize * cellsize)); }
    int AnimationFrameNumber() const { return SimulationStep / UpdateEveryNthStep; }
    size_t IndenterArraySize() const { return sizeof(double) * n_indenter_subdivisions * dim; }
    int CellIdx(float x) const { return (int)(x * cellsize_inv + 0.5); }
    int PointCellIndex(float x, float y) const { return CellIdx(x) * GridY + CellIdx(y); }
};
static_assert(sizeof(SimParams) == sizeof(icy_sim_params), "SimParams adds no data to icy_sim_params");

class Model;
class SnapshotManager;

// the frame hand-off lock of icy::Model: Step() locks it before the download and the
// transfer-completion callback unlocks it, possibly from another thread (cli/main.cpp:51-61);
// unlike std::mutex that is allowed here
class CycleMutex {
public:
    void lock();
    void unlock();
    bool try_lock();

private:
    std::mutex m_;
    std::condition_variable cv_;
    bool locked_ = false;
};

}  // namespace icy

// page-locked line-major particle buffer: 16 lines of `capacity` doubles
class HostSideSOA {
public:
    double *host_buffer = nullptr;
    unsigned capacity = 0;
    unsigned size = 0;

    HostSideSOA() = default;
    HostSideSOA(const HostSideSOA &) = delete;
    HostSideSOA &operator=(const HostSideSOA &) = delete;
    ~HostSideSOA();

    void Allocate(unsigned capacity);          // cleared, page-locked (icy_host_alloc)
    void RemoveDisabledAndSort(double hinv, unsigned GridY);
    unsigned FindFirstPointAtGridXIndex(const int index_grid_x, const double hinv);
    void InitializeBlock();                    // Fe = I, Jp_inv = 1

    double *getPointerToPosX() { return host_buffer + (size_t)capacity * icy::SimParams::posx; }
    double *getPointerToPosY() { return host_buffer + (size_t)capacity * (icy::SimParams::posx + 1); }
    double *getPointerToLine(int idxLine) { return host_buffer + (size_t)capacity * idxLine; }
    double &value(size_t line, unsigned i) { return host_buffer[line * capacity + i]; }
    int64_t utility(unsigned i) const;
    bool disabled(unsigned i) const { return utility(i) & ICY_STATUS_DISABLED; }

    std::pair<icy::Vector2d, icy::Vector2d> getBlockDimensions();
    void offsetBlock(icy::Vector2d offset);
};

class GPU_Implementation5 {
public:
    icy::Model *model = nullptr;
    HostSideSOA hssoa;
    icy::Vector2d indenter_force;
    std::vector<double> indenter_force_bins;    // 2 per subdivision, summed over the frame
    std::function<void()> transfer_completion_callback;

    int device = 0;                             // CUDA device of the single partition
    int precision = ICY_PRECISION_FP64;         // ICY_PRECISION_FP64 or ICY_PRECISION_FP32_SPLIT

    GPU_Implementation5() = default;
    GPU_Implementation5(const GPU_Implementation5 &) = delete;
    GPU_Implementation5 &operator=(const GPU_Implementation5 &) = delete;
    ~GPU_Implementation5();

    void allocate_arrays();                     // creates the device instance (capacity = hssoa.capacity)
    void split_hssoa_into_partitions();         // one partition: every point
    void transfer_ponts_to_device();
    void initialize_and_enable_peer_access();   // one device: selects it
    void transfer_from_device();

    void synchronize();
    void update_constants();
    void reset_grid();
    void reset_indenter_force_accumulator();

    void p2g();
    void receive_halos();
    void update_nodes(double simulation_time);
    void g2p(const bool recordPQ, const bool enablePointTransfer);
    void receive_points();
    void record_timings(const bool enablePointTransfer);

    // nsteps sub-steps of Model::Step's loop queued on the device in one call
    // (icy_mpm_step); advances simulation_time exactly as that loop does
    void run_steps(int step0, int nsteps, double &simulation_time);
    void set_option(const std::string &name, double value);
    int status();
    icy_mpm *handle() const { return h_; }

private:
    icy_mpm *h_ = nullptr;
    void need_instance(const char *what) const;
};

class icy::Model {
public:
    Model();
    ~Model();
    void Reset();
    void Prepare();
    bool Step();
    void RequestAbort() { abortRequested = true; }
    void UnlockCycleMutex();

    icy::SimParams prms;
    GPU_Implementation5 gpu;
    int max_points_transferred = 0, max_pt_deviation = 0;
    bool SyncTopologyRequired = true;
    // true: Step() runs the reference's per-phase loop (reset_grid, p2g, update_nodes, g2p per
    // sub-step); false (default): the whole frame is queued by one icy_mpm_step call
    bool per_phase_loop = false;

    icy::CycleMutex processing_current_cycle_data;   // std::mutex in the reference
    std::mutex accessing_point_data;

    // "logs/indenter_force.csv" as the reference opens it (truncated); another path or "" (none)
    void SetForceLog(const std::string &path);
    // "logs/timings.csv": per frame the columns of simulation/model.cpp:91-95 from per-kernel
    // CUDA events (microseconds per sub-step; the fused G2P+P2G launch is under P2G)
    void SetTimingsLog(const std::string &path);

private:
    bool abortRequested = false;
    std::unique_ptr<std::ofstream> log_indenter_force;
    std::unique_ptr<std::ofstream> log_timings;
    void write_timings(int cycles);
};

class icy::SnapshotManager {
public:
    icy::Model *model = nullptr;

    // reads "x", "y", "llGrainIDs" and its "volume" attribute from an HDF5 point cloud,
    // then places, sorts and uploads the points as simulation/snapshotmanager.cpp:29-121 does
    void LoadRawPoints(std::string fileName);
    // the same set-up from a seeded synthetic block (icy_scene_block)
    void LoadSyntheticBlock(double block_w, double block_h, int ppc, uint64_t seed, int n_grains);
    // checkpoint of the whole model state (parameters, step, time, particles) and its restore;
    // the reference's snapshot code is disabled (cli/main.cpp:57), this is the resume path
    void SaveSnapshot(std::string fileName);
    void ReadSnapshot(std::string fileName);

private:
    void finish_setup(unsigned n_points);
};

namespace icy {
// shortest round-trip decimal text of a double in the style of the fmt library's "{}"
// (fixed notation for decimal exponents -5 < e < 16, else d.ddde+XX)
std::string format_double(double v);
}  // namespace icy
