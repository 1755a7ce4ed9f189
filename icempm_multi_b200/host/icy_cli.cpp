// icy_cli.cpp -- headless driver with the structure of the reference's
// cli/main.cpp: a Model and a SnapshotManager, the configuration file parsed
// with SimParams::ParseFile, the point cloud loaded, a transfer-completion
// callback that hands each frame to a worker thread which unlocks the cycle
// mutex, and a simulation thread calling Model::Step until the end time.
//
//   icy_cli CONFIG.json [--frames N] [--precision fp64|fp32] [--device D]
//           [--block W H] [--ppc K] [--seed S] [--grains G]
//           [--per-phase] [--option NAME=VALUE]... [--log FILE]
//           [--resume CHECKPOINT] [--checkpoint FILE]
//
// "InputRawPoints" naming an .h5 file is read as the reference reads it; the
// value "synthetic" (or --block) builds a seeded block of W x H metres at K
// points per cell instead.  The frame loop stops at SimulationEndTime, after
// N frames, or when "q" is read on standard input (--interactive).  At exit
// the final state is written with SnapshotManager::SaveSnapshot if
// --checkpoint is given; --resume starts from such a file.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "icy_host.hpp"

namespace {

void usage()
{
    std::fprintf(stderr,
                 "usage: icy_cli CONFIG.json [--frames N] [--precision fp64|fp32] [--device D]\n"
                 "               [--block W H] [--ppc K] [--seed S] [--grains G] [--per-phase]\n"
                 "               [--option NAME=VALUE]... [--log FILE] [--resume CKPT] [--checkpoint FILE]\n"
                 "               [--interactive]\n");
}

}  // namespace

int main(int argc, char **argv)
{
    std::string config, log_path = "logs/indenter_force.csv", resume, checkpoint;
    long frames = -1;
    int device = 0, precision = ICY_PRECISION_FP64, ppc = 4, grains = 16;
    double block_w = 0, block_h = 0;
    unsigned long long seed = 1;
    bool per_phase = false, interactive = false;
    std::vector<std::pair<std::string, double>> options;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&](const char *what) -> std::string {
            if (i + 1 >= argc) { std::fprintf(stderr, "%s needs a value\n", what); usage(); std::exit(2); }
            return argv[++i];
        };
        if (a == "--frames") frames = std::stol(next("--frames"));
        else if (a == "--precision") {
            std::string p = next("--precision");
            if (p == "fp64") precision = ICY_PRECISION_FP64;
            else if (p == "fp32") precision = ICY_PRECISION_FP32_SPLIT;
            else { usage(); return 2; }
        } else if (a == "--device") device = std::stoi(next("--device"));
        else if (a == "--block") { block_w = std::stod(next("--block")); block_h = std::stod(next("--block")); }
        else if (a == "--ppc") ppc = std::stoi(next("--ppc"));
        else if (a == "--seed") seed = std::stoull(next("--seed"));
        else if (a == "--grains") grains = std::stoi(next("--grains"));
        else if (a == "--per-phase") per_phase = true;
        else if (a == "--interactive") interactive = true;
        else if (a == "--log") log_path = next("--log");
        else if (a == "--resume") resume = next("--resume");
        else if (a == "--checkpoint") checkpoint = next("--checkpoint");
        else if (a == "--option") {
            std::string kv = next("--option");
            size_t eq = kv.find('=');
            if (eq == std::string::npos) { usage(); return 2; }
            options.push_back({kv.substr(0, eq), std::stod(kv.substr(eq + 1))});
        } else if (a == "-h" || a == "--help") { usage(); return 0; }
        else if (!a.empty() && a[0] != '-' && config.empty()) config = a;
        else { std::fprintf(stderr, "unknown argument %s\n", a.c_str()); usage(); return 2; }
    }
    if (config.empty() && resume.empty()) { usage(); return 2; }

    try {
        icy::Model model;
        icy::SnapshotManager snapshot;
        model.SetForceLog(log_path);
        model.per_phase_loop = per_phase;
        model.gpu.device = device;
        model.gpu.precision = precision;
        model.Reset();
        snapshot.model = &model;

        if (!resume.empty()) {
            snapshot.ReadSnapshot(resume);
        } else {
            std::string pointCloudFile = model.prms.ParseFile(config);
            const bool synthetic = block_w > 0 || pointCloudFile == "synthetic";
            if (synthetic) {
                if (block_w <= 0) { std::fprintf(stderr, "\"synthetic\" points need --block W H\n"); return 2; }
                snapshot.LoadSyntheticBlock(block_w, block_h, ppc, seed, grains);
            } else {
                snapshot.LoadRawPoints(pointCloudFile);
            }
        }
        for (auto &o : options) model.gpu.set_option(o.first, o.second);
        std::printf("points %u, grid %d x %d, h %g, dt %g, frames of %d steps, end time %g\n", model.gpu.hssoa.size,
                    model.prms.GridXTotal, model.prms.GridY, model.prms.cellsize, model.prms.InitialTimeStep,
                    model.prms.UpdateEveryNthStep, model.prms.SimulationEndTime);

        std::thread snapshot_thread;
        std::atomic<bool> request_terminate{false};
        std::atomic<long> frames_done{0};
        model.gpu.transfer_completion_callback = [&]() {
            if (snapshot_thread.joinable()) snapshot_thread.join();
            snapshot_thread = std::thread([&]() {
                const int frame = model.prms.AnimationFrameNumber();
                (void)frame;
                model.UnlockCycleMutex();
            });
        };

        std::thread simulation_thread([&]() {
            bool result;
            do {
                result = model.Step();
                const long f = ++frames_done;
                std::printf("frame %d t %s F %s\n", model.prms.AnimationFrameNumber(),
                            icy::format_double(model.prms.SimulationTime).c_str(),
                            icy::format_double(model.gpu.indenter_force.norm()).c_str());
                std::fflush(stdout);
                if (frames >= 0 && f >= frames) break;
            } while (!request_terminate && result);
            request_terminate = true;
        });

        if (interactive) {
            std::string user_input;
            while (!request_terminate && std::cin >> user_input)
                if (!user_input.empty() && user_input[0] == 'q') request_terminate = true;
        }
        simulation_thread.join();
        model.gpu.synchronize();
        if (snapshot_thread.joinable()) snapshot_thread.join();
        if (!checkpoint.empty()) snapshot.SaveSnapshot(checkpoint);
        std::printf("cm done\n");
    } catch (const std::exception &e) {
        std::fprintf(stderr, "icy_cli: %s\n", e.what());
        return 1;
    }
    return 0;
}
