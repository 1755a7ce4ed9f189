// icy_host.cpp -- see icy_host.hpp.
#include "icy_host.hpp"

#include <algorithm>
#include <charconv>
#include <cstring>
#include <filesystem>
#include <numeric>

#include "../../include/icempm_host.h"

namespace icy {

void check(int status, const char *what)
{
    if (status == ICY_OK) return;
    std::string m = std::string(what) + ": ";
    const char *e = icy_last_error();
    m += (e && *e) ? e : "error";
    m += " (status " + std::to_string(status) + ")";
    throw std::runtime_error(m);
}

std::string SimParams::ParseFile(std::string fileName)
{
    char raw[4096] = {0};
    const int rc = icy_params_parse_file(this, fileName.c_str(), raw, sizeof(raw));
    if (rc == ICY_ERR_FILE) throw std::runtime_error("configuration file is not found");
    if (rc == ICY_ERR_CONFIG_MISSING) throw std::runtime_error("raw point file is not provided");
    check(rc, "SimParams::ParseFile");
    return std::string(raw);
}

void CycleMutex::lock()
{
    std::unique_lock<std::mutex> g(m_);
    cv_.wait(g, [&] { return !locked_; });
    locked_ = true;
}

void CycleMutex::unlock()
{
    {
        std::lock_guard<std::mutex> g(m_);
        locked_ = false;
    }
    cv_.notify_one();
}

bool CycleMutex::try_lock()
{
    std::lock_guard<std::mutex> g(m_);
    if (locked_) return false;
    locked_ = true;
    return true;
}

std::string format_double(double v)
{
    if (std::isnan(v)) return "nan";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    char b[64];
    auto r = std::to_chars(b, b + sizeof(b), v, std::chars_format::scientific);
    std::string s(b, r.ptr);
    std::string sign;
    if (s[0] == '-') { sign = "-"; s.erase(0, 1); }
    const size_t epos = s.find('e');
    std::string digits = s.substr(0, epos);
    digits.erase(std::remove(digits.begin(), digits.end(), '.'), digits.end());
    const int E = std::stoi(s.substr(epos + 1));
    if (digits == "0") return sign + "0";
    std::string out;
    if (E >= -4 && E < 16) {
        if (E >= 0) {
            if ((int)digits.size() <= E + 1) out = digits + std::string(E + 1 - digits.size(), '0');
            else out = digits.substr(0, E + 1) + "." + digits.substr(E + 1);
        } else {
            out = "0." + std::string(-E - 1, '0') + digits;
        }
    } else {
        out = digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        char eb[16];
        std::snprintf(eb, sizeof(eb), "e%c%02d", E < 0 ? '-' : '+', std::abs(E));
        out += eb;
    }
    return sign + out;
}

}  // namespace icy

// ---------------------------------------------------------------- HostSideSOA

HostSideSOA::~HostSideSOA() { icy_host_free(host_buffer); }

void HostSideSOA::Allocate(unsigned capacity_)
{
    icy_host_free(host_buffer);
    host_buffer = nullptr;
    capacity = capacity_;
    size = 0;
    void *p = nullptr;
    icy::check(icy_host_alloc(sizeof(double) * (size_t)capacity * icy::SimParams::nPtsArrays, &p),
               "allocating host buffer for points");
    host_buffer = static_cast<double *>(p);
}

int64_t HostSideSOA::utility(unsigned i) const
{
    int64_t u;
    std::memcpy(&u, host_buffer + i, 8);
    return u;
}

void HostSideSOA::RemoveDisabledAndSort(double hinv, unsigned GridY)
{
    // host_side_soa.cpp:50-61: drop disabled points, then order by ProxyPoint::getCellIndex
    // (the reference's std::sort is not stable; a stable sort gives one defined order)
    std::vector<unsigned> keep;
    keep.reserve(size);
    for (unsigned i = 0; i < size; i++)
        if (!disabled(i)) keep.push_back(i);
    auto cell = [&](unsigned i) {
        const double x = host_buffer[(size_t)icy::SimParams::posx * capacity + i];
        const double y = host_buffer[(size_t)(icy::SimParams::posx + 1) * capacity + i];
        return (long)(int)(x * hinv + 0.5) * (long)GridY + (int)(y * hinv + 0.5);
    };
    std::vector<long> key(size);
    for (unsigned i : keep) key[i] = cell(i);
    std::stable_sort(keep.begin(), keep.end(), [&](unsigned a, unsigned b) { return key[a] < key[b]; });
    std::vector<double> tmp(keep.size());
    for (size_t l = 0; l < icy::SimParams::nPtsArrays; l++) {
        double *L = host_buffer + l * capacity;
        for (size_t k = 0; k < keep.size(); k++) tmp[k] = L[keep[k]];
        std::copy(tmp.begin(), tmp.end(), L);
    }
    size = (unsigned)keep.size();
}

unsigned HostSideSOA::FindFirstPointAtGridXIndex(const int index_grid_x, const double hinv)
{
    // host_side_soa.cpp:81-91: first point whose (int)(x*hinv + 0.5) >= index (points sorted by cell)
    const double *X = getPointerToPosX();
    unsigned lo = 0, hi = size;
    while (lo < hi) {
        const unsigned mid = lo + (hi - lo) / 2;
        if ((int)(X[mid] * hinv + 0.5) < index_grid_x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

void HostSideSOA::InitializeBlock()
{
    for (unsigned i = 0; i < size; i++) {
        value(icy::SimParams::idx_Jp_inv, i) = 1.0;
        value(icy::SimParams::Fe00, i) = 1.0;
        value(icy::SimParams::Fe00 + 3, i) = 1.0;
    }
}

std::pair<icy::Vector2d, icy::Vector2d> HostSideSOA::getBlockDimensions()
{
    icy::Vector2d lo(0, 0), hi(0, 0);
    for (int k = 0; k < 2; k++) {
        const double *L = getPointerToLine((int)icy::SimParams::posx + k);
        if (size == 0) continue;
        auto mm = std::minmax_element(L, L + size);
        lo[k] = *mm.first;
        hi[k] = *mm.second;
    }
    return {lo, hi};
}

void HostSideSOA::offsetBlock(icy::Vector2d offset)
{
    double *X = getPointerToPosX(), *Y = getPointerToPosY();
    for (unsigned i = 0; i < size; i++) { X[i] += offset.x(); Y[i] += offset.y(); }
}

// ---------------------------------------------------------------- GPU_Implementation5

GPU_Implementation5::~GPU_Implementation5()
{
    if (h_) icy_mpm_destroy(h_);
}

void GPU_Implementation5::need_instance(const char *what) const
{
    if (!h_) throw std::runtime_error(std::string(what) + ": device arrays are not allocated");
}

void GPU_Implementation5::initialize_and_enable_peer_access()
{
    if (model && model->prms.nPartitions > 1)
        throw std::runtime_error("initialize_and_enable_peer_access: one partition per process is supported");
}

void GPU_Implementation5::split_hssoa_into_partitions()
{
    // one partition spanning the whole grid holds every point
}

void GPU_Implementation5::allocate_arrays()
{
    if (!model) throw std::runtime_error("allocate_arrays: no model");
    if (h_) { icy_mpm_destroy(h_); h_ = nullptr; }
    const unsigned cap = std::max(hssoa.capacity, 1u);
    icy::check(icy_mpm_create(&model->prms, device, cap, precision, &h_), "allocate_arrays");
    indenter_force_bins.assign(2 * (size_t)model->prms.n_indenter_subdivisions, 0.0);
}

void GPU_Implementation5::transfer_ponts_to_device()
{
    need_instance("transfer_ponts_to_device");
    icy::check(icy_mpm_transfer_points_to_device(h_, hssoa.host_buffer, hssoa.capacity, hssoa.size),
               "transfer_ponts_to_device");
}

void GPU_Implementation5::transfer_from_device()
{
    need_instance("transfer_from_device");
    indenter_force_bins.assign(2 * (size_t)model->prms.n_indenter_subdivisions, 0.0);
    unsigned n = 0;
    icy::check(icy_mpm_transfer_from_device(h_, hssoa.host_buffer, hssoa.capacity, &n, indenter_force_bins.data()),
               "transfer_from_device");
    hssoa.size = n;
    indenter_force.setZero();
    for (int j = 0; j < model->prms.n_indenter_subdivisions; j++) {
        indenter_force.x() += indenter_force_bins[2 * j + 0];
        indenter_force.y() += indenter_force_bins[2 * j + 1];
    }
    if (transfer_completion_callback) transfer_completion_callback();
}

void GPU_Implementation5::synchronize()
{
    if (h_) icy::check(icy_mpm_synchronize(h_), "synchronize");
}

void GPU_Implementation5::update_constants()
{
    need_instance("update_constants");
    icy::check(icy_mpm_update_constants(h_, &model->prms), "update_constants");
}

void GPU_Implementation5::reset_grid() { need_instance("reset_grid"); icy::check(icy_mpm_reset_grid(h_), "reset_grid"); }

void GPU_Implementation5::reset_indenter_force_accumulator()
{
    need_instance("reset_indenter_force_accumulator");
    icy::check(icy_mpm_reset_indenter_force_accumulator(h_), "reset_indenter_force_accumulator");
}

void GPU_Implementation5::p2g() { need_instance("p2g"); icy::check(icy_mpm_p2g(h_), "p2g"); }
void GPU_Implementation5::receive_halos() { need_instance("receive_halos"); icy::check(icy_mpm_receive_halos(h_), "receive_halos"); }

void GPU_Implementation5::update_nodes(double simulation_time)
{
    need_instance("update_nodes");
    icy::check(icy_mpm_update_nodes(h_, model->prms.indenter_x, model->prms.indenter_y, simulation_time),
               "update_nodes");
}

void GPU_Implementation5::g2p(const bool recordPQ, const bool enablePointTransfer)
{
    need_instance("g2p");
    icy::check(icy_mpm_g2p(h_, recordPQ ? 1 : 0, 0), "g2p");
    (void)enablePointTransfer;   // one partition: no point leaves it
}

void GPU_Implementation5::receive_points() { need_instance("receive_points"); icy::check(icy_mpm_receive_points(h_), "receive_points"); }

void GPU_Implementation5::record_timings(const bool) {}

void GPU_Implementation5::run_steps(int step0, int nsteps, double &simulation_time)
{
    need_instance("run_steps");
    icy::check(icy_mpm_step(h_, step0, nsteps, &simulation_time), "run_steps");
}

void GPU_Implementation5::set_option(const std::string &name, double value)
{
    need_instance("set_option");
    icy::check(icy_mpm_set_option(h_, name.c_str(), value), "set_option");
}

int GPU_Implementation5::status()
{
    need_instance("status");
    return icy_mpm_status(h_);
}

// ---------------------------------------------------------------- icy::Model

icy::Model::Model()
{
    prms.Reset();
    gpu.model = this;
    SetForceLog("logs/indenter_force.csv");
    SetTimingsLog("logs/timings.csv");
}

icy::Model::~Model() = default;

void icy::Model::SetForceLog(const std::string &path)
{
    log_indenter_force.reset();
    if (path.empty()) return;
    std::filesystem::path p(path);
    if (p.has_parent_path()) std::filesystem::create_directories(p.parent_path());
    log_indenter_force = std::make_unique<std::ofstream>(path, std::ios::trunc);
    if (!*log_indenter_force) throw std::runtime_error("cannot open " + path);
}

void icy::Model::SetTimingsLog(const std::string &path)
{
    log_timings.reset();
    if (path.empty()) return;
    std::filesystem::path p(path);
    if (p.has_parent_path()) std::filesystem::create_directories(p.parent_path());
    log_timings = std::make_unique<std::ofstream>(path, std::ios::trunc);
    if (!*log_timings) throw std::runtime_error("cannot open " + path);
}

void icy::Model::write_timings(int cycles)
{
    // simulation/model.cpp:91-95 (one partition): frame, partition, points, free, disabled,
    // points sent, max deviation, P2G+halo, accept halo, update, G2P, sent, accepted, total
    const int mx = 32;
    std::vector<char> names(48 * mx);
    std::vector<double> ms(mx);
    std::vector<int64_t> n(mx);
    int count = 0;
    icy::check(icy_mpm_profile_read(gpu.handle(), mx, names.data(), ms.data(), n.data(), &count), "timings");
    double p2g = 0, upd = 0, g2p = 0, total = 0;
    for (int k = 0; k < std::min(count, mx); k++) {
        const std::string name(&names[48 * k]);
        total += ms[k];
        if (name == "k_tile_g2p2g" || name == "k_tile_p2g" || name == "k_p2g_simple" || name == "memset_grid")
            p2g += ms[k];
        else if (name == "k_update_nodes" || name == "k_update_simple") upd += ms[k];
        else if (name == "k_tile_g2p" || name == "k_g2p_simple") g2p += ms[k];
    }
    const double coeff = 1000.0 / std::max(cycles, 1);
    const HostSideSOA &s = gpu.hssoa;
    int disabled = 0;
    for (unsigned i = 0; i < s.size; i++) disabled += s.disabled(i) ? 1 : 0;
    char line[256];
    std::snprintf(line, sizeof(line), "%d, %2d,%8u,%8u,%7d,%3d,%3d,%5.1f,%5.1f,%5.1f,%5.1f,%5.1f,%5.1f,%6.1f",
                  prms.AnimationFrameNumber(), 0, s.size, s.capacity - s.size, disabled, 0, 0, p2g * coeff, 0.0,
                  upd * coeff, g2p * coeff, 0.0, 0.0, total * coeff);
    *log_timings << line << '\n';
    log_timings->flush();
}

void icy::Model::Reset()
{
    max_points_transferred = 0;
    prms.SimulationStep = 0;
    prms.SimulationTime = 0;
    SyncTopologyRequired = true;
}

void icy::Model::Prepare()
{
    abortRequested = false;
    gpu.update_constants();
}

void icy::Model::UnlockCycleMutex() { processing_current_cycle_data.unlock(); }

bool icy::Model::Step()
{
    // simulation/model.cpp:27-114 for one partition
    double simulation_time = prms.SimulationTime;
    int count_unupdated_steps = 0;
    gpu.reset_indenter_force_accumulator();
    if (log_timings) icy::check(icy_mpm_profile(gpu.handle(), 1), "timings");

    if (per_phase_loop) {
        do {
            simulation_time += prms.InitialTimeStep;
            prms.indenter_x = prms.indenter_x_initial + simulation_time * prms.IndVelocity;
            gpu.reset_grid();
            gpu.p2g();
            gpu.receive_halos();
            gpu.update_nodes(simulation_time);
            const bool isZeroStep = (prms.SimulationStep + count_unupdated_steps) % prms.UpdateEveryNthStep == 0;
            gpu.g2p(isZeroStep, false);
            gpu.record_timings(false);
            count_unupdated_steps++;
        } while ((prms.SimulationStep + count_unupdated_steps) % prms.UpdateEveryNthStep != 0);
    } else {
        count_unupdated_steps = prms.UpdateEveryNthStep - prms.SimulationStep % prms.UpdateEveryNthStep;
        gpu.run_steps(prms.SimulationStep, count_unupdated_steps, simulation_time);
        prms.indenter_x = prms.indenter_x_initial + simulation_time * prms.IndVelocity;
    }

    processing_current_cycle_data.lock();   // held until the previous frame's data is processed
    {
        std::lock_guard<std::mutex> g(accessing_point_data);
        const bool has_callback = (bool)gpu.transfer_completion_callback;
        gpu.transfer_from_device();
        max_pt_deviation = 0;
        prms.SimulationTime = simulation_time;
        prms.SimulationStep += count_unupdated_steps;
        gpu.indenter_force /= (double)count_unupdated_steps;
        if (log_timings) {
            write_timings(count_unupdated_steps);
            icy::check(icy_mpm_profile(gpu.handle(), 0), "timings");
        }
        if (log_indenter_force) {
            *log_indenter_force << icy::format_double(prms.SimulationTime) << ','
                                << icy::format_double(gpu.indenter_force.norm()) << ','
                                << icy::format_double(gpu.indenter_force.x()) << ','
                                << icy::format_double(gpu.indenter_force.y()) << '\n';
            log_indenter_force->flush();
        }
        // with no callback nobody would release the frame lock: release it here
        // (the reference always installs one, cli/main.cpp:51-61)
        if (!has_callback) processing_current_cycle_data.unlock();
    }
    return prms.SimulationTime < prms.SimulationEndTime;
}

// ---------------------------------------------------------------- icy::SnapshotManager

void icy::SnapshotManager::finish_setup(unsigned n_points)
{
    (void)n_points;
    model->gpu.initialize_and_enable_peer_access();
    model->gpu.split_hssoa_into_partitions();
    model->gpu.allocate_arrays();
    model->gpu.transfer_ponts_to_device();
    model->Reset();
    model->Prepare();
}

void icy::SnapshotManager::LoadRawPoints(std::string fileName)
{
    // simulation/snapshotmanager.cpp:29-121
    if (!std::filesystem::exists(fileName)) throw std::runtime_error("error reading raw points file - no file");
    auto host_check = [](int rc, const char *what) {
        if (rc != ICY_OK)
            throw std::runtime_error(std::string(what) + ": " + icy_host_last_error() + " (status " +
                                     std::to_string(rc) + ")");
    };
    unsigned nPoints = 0;
    host_check(icy_h5_count(fileName.c_str(), &nPoints), "LoadRawPoints");
    icy::SimParams &p = model->prms;
    p.nPtsTotal = (int)nPoints;
    HostSideSOA &s = model->gpu.hssoa;
    s.Allocate((unsigned)(nPoints * (1 + p.ExtraSpaceForIncomingPoints)));
    unsigned n = 0;
    host_check(icy_h5_load(&p, fileName.c_str(), s.host_buffer, s.capacity, &n), "LoadRawPoints");
    s.size = n;
    finish_setup(n);
}

void icy::SnapshotManager::LoadSyntheticBlock(double block_w, double block_h, int ppc, uint64_t seed, int n_grains)
{
    icy::SimParams &p = model->prms;
    icy_params_compute_helpers(&p);
    const unsigned n = icy_scene_block_count(&p, block_w, block_h, ppc);
    HostSideSOA &s = model->gpu.hssoa;
    s.Allocate((unsigned)(n * (1 + p.ExtraSpaceForIncomingPoints)) + 1);
    unsigned got = 0;
    icy::check(icy_scene_block(&p, block_w, block_h, ppc, seed, n_grains, s.host_buffer, s.capacity, &got),
               "LoadSyntheticBlock");
    s.size = got;
    finish_setup(got);
}

namespace {
const char kCkptMagic[8] = {'I', 'C', 'Y', 'C', 'K', 'P', 'T', '1'};
}

void icy::SnapshotManager::SaveSnapshot(std::string fileName)
{
    GPU_Implementation5 &gpu = model->gpu;
    HostSideSOA &s = gpu.hssoa;
    std::lock_guard<std::mutex> g(model->accessing_point_data);
    if (gpu.handle()) {
        unsigned n = 0;
        icy::check(icy_mpm_transfer_from_device(gpu.handle(), s.host_buffer, s.capacity, &n, nullptr), "SaveSnapshot");
        s.size = n;
    }
    std::filesystem::path fp(fileName);
    if (fp.has_parent_path()) std::filesystem::create_directories(fp.parent_path());
    std::ofstream f(fileName, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("cannot write " + fileName);
    const uint32_t hdr[6] = {1u, (uint32_t)sizeof(icy_sim_params), s.capacity, s.size, (uint32_t)gpu.precision, 0u};
    f.write(kCkptMagic, 8);
    f.write(reinterpret_cast<const char *>(hdr), sizeof(hdr));
    f.write(reinterpret_cast<const char *>(static_cast<const icy_sim_params *>(&model->prms)), sizeof(icy_sim_params));
    for (size_t l = 0; l < icy::SimParams::nPtsArrays; l++)
        f.write(reinterpret_cast<const char *>(s.getPointerToLine((int)l)), sizeof(double) * s.size);
    if (!f) throw std::runtime_error("short write of " + fileName);
}

void icy::SnapshotManager::ReadSnapshot(std::string fileName)
{
    std::ifstream f(fileName, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + fileName);
    char magic[8];
    uint32_t hdr[6];
    f.read(magic, 8);
    f.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    if (!f || std::memcmp(magic, kCkptMagic, 8) != 0 || hdr[0] != 1u || hdr[1] != sizeof(icy_sim_params))
        throw std::runtime_error(fileName + " is not a checkpoint of this library version");
    icy_sim_params prm;
    f.read(reinterpret_cast<char *>(&prm), sizeof(prm));
    const unsigned capacity = hdr[2], size = hdr[3];
    if (size > capacity) throw std::runtime_error("corrupt checkpoint header");
    GPU_Implementation5 &gpu = model->gpu;
    HostSideSOA &s = gpu.hssoa;
    s.Allocate(capacity);
    s.size = size;
    for (size_t l = 0; l < icy::SimParams::nPtsArrays; l++)
        f.read(reinterpret_cast<char *>(s.getPointerToLine((int)l)), sizeof(double) * size);
    if (!f) throw std::runtime_error("truncated checkpoint " + fileName);
    static_cast<icy_sim_params &>(model->prms) = prm;
    gpu.precision = (int)hdr[4];
    gpu.initialize_and_enable_peer_access();
    gpu.allocate_arrays();
    gpu.transfer_ponts_to_device();
    model->Prepare();   // the step counter and time come from the checkpoint, not Reset()
}
