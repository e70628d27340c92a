// cm -- command-line driver of the MLS-MPM indentation model, the
// counterpart of iceMPM's cli/main.cpp: a simulation thread steps the model
// frame by frame; each frame's completion callback hands the frame to a
// snapshot thread that writes it and releases the model's cycle mutex;
// console input "s" asks for a full snapshot, "q" for a snapshot and exit.
//
//   cm config.json [--out DIR] [--form fp32|fp64|stepwise] [--frames N]
//                  [--resume FILE] [--block CX CY] [--pq] [--quiet]
//
// The point cloud is the configuration's InputRawPoints file (HDF5,
// LoadRawPoints), or with --block a seeded synthetic block of CX x CY cells
// (4 particles per cell). --frames stops after N frames; without it the run
// ends at SimulationEndTime or on "q". --resume continues from a snapshot
// written by an earlier run. End of input on stdin is not a command.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <iostream>
#include <string>
#include <thread>

#include "icempm.hpp"

namespace {

struct Options {
    std::string config, out = "cm_snapshots", resume;
    int form = ICM_FORM_FP32, frames = -1, block_x = 0, block_y = 0;
    bool pq = false, quiet = false;
};

int usage()
{
    std::fprintf(stderr,
                 "usage: cm config.json [--out DIR] [--form fp32|fp64|stepwise] [--frames N] [--resume FILE]\n"
                 "                      [--block CX CY] [--pq] [--quiet]\n");
    return 2;
}

bool parse(int argc, char **argv, Options &o)
{
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&](const char *&v) {
            if (i + 1 >= argc) return false;
            v = argv[++i];
            return true;
        };
        const char *v = nullptr;
        if (a == "--out") { if (!next(v)) return false; o.out = v; }
        else if (a == "--form") {
            if (!next(v)) return false;
            std::string f = v;
            if (f == "fp32") o.form = ICM_FORM_FP32;
            else if (f == "fp64") o.form = ICM_FORM_FP64;
            else if (f == "stepwise") o.form = ICM_FORM_FP64_STEPWISE;
            else return false;
        }
        else if (a == "--frames") { if (!next(v)) return false; o.frames = std::atoi(v); }
        else if (a == "--resume") { if (!next(v)) return false; o.resume = v; }
        else if (a == "--block") {
            const char *w = nullptr;
            if (!next(v) || !next(w)) return false;
            o.block_x = std::atoi(v);
            o.block_y = std::atoi(w);
        }
        else if (a == "--pq") o.pq = true;
        else if (a == "--quiet") o.quiet = true;
        else if (!a.empty() && a[0] != '-' && o.config.empty()) o.config = a;
        else return false;
    }
    return !o.config.empty();
}

// the synthetic stand-in for LoadRawPoints (a seeded ice block)
void load_block(icy::Model &model, int cx, int cy)
{
    icm_block_desc d{};
    d.cells_x = cx;
    d.cells_y = cy;
    d.ind_y_above_floor = 0.2;
    d.grain_size = 0.05;
    d.seed = 12345;
    int n = 0;
    icy::icm_check(icm_scene_block(&model.prms, &d, nullptr, &n));
    model.gpu.cuda_allocate_arrays((size_t)model.prms.GridX * model.prms.GridY, (size_t)n);
    icy::icm_check(icm_scene_block(&model.prms, &d, model.gpu.tmp_transfer_buffer, &n));
    model.gpu.transfer_ponts_to_device();
    model.Reset();
    model.Prepare();
}

}  // namespace

int main(int argc, char **argv)
{
    Options opt;
    if (!parse(argc, argv, opt)) return usage();
    try {
        icy::Model model;
        icy::SnapshotManager snapshot;
        snapshot.model = &model;
        std::thread snapshot_thread;
        std::atomic<bool> request_terminate{false};
        std::atomic<bool> request_full_snapshot{false};
        std::atomic<int> frames_done{0};

        model.gpu.initialize();
        model.Reset();
        const std::string raw = model.prms.ParseFile(opt.config);
        model.gpu.set_form(opt.form);
        if (!opt.resume.empty()) {
            const int frame = snapshot.ReadSnapshot(opt.resume);
            if (!opt.quiet) std::printf("resumed from %s (frame %d)\n", opt.resume.c_str(), frame);
        } else if (opt.block_x > 0 && opt.block_y > 0) {
            load_block(model, opt.block_x, opt.block_y);
        } else {
            snapshot.LoadRawPoints(raw);
        }
        std::filesystem::create_directories(opt.out);

        // what to do once a frame is on the host (cli/main.cpp:51-62)
        model.gpu.transfer_completion_callback = [&]() {
            if (snapshot_thread.joinable()) snapshot_thread.join();
            snapshot_thread = std::thread([&]() {
                const int number = model.prms.SimulationStep / model.prms.UpdateEveryNthStep;
                if (request_terminate && !request_full_snapshot) {
                    model.UnlockCycleMutex();
                    return;
                }
                const std::string path = snapshot.SaveSnapshot(opt.out);
                if (opt.pq) snapshot.SavePQ(opt.out);
                request_full_snapshot = false;
                if (!opt.quiet)
                    std::printf("frame %d -> %s (%.3f ms per substep)\n", number, path.c_str(),
                                model.compute_time_per_cycle);
                frames_done++;
                model.UnlockCycleMutex();
            });
        };

        std::atomic<bool> sim_done{false};
        std::thread simulation_thread([&]() {
            int frames = 0;
            bool go = true;
            do {
                go = model.Step();
                frames++;
                if (opt.frames > 0 && frames >= opt.frames) go = false;
            } while (go && !request_terminate);
            sim_done = true;
        });

        // console commands; without a terminal (or at end of input) the run
        // goes on to its end
        std::thread console([&]() {
            std::string in;
            while (!sim_done && std::cin >> in) {
                if (in[0] == 's') {
                    request_full_snapshot = true;
                    std::printf("requested to save a full snapshot\n");
                } else if (in[0] == 'q') {
                    request_terminate = true;
                    request_full_snapshot = true;
                    std::printf("requested to save the snapshot and terminate\n");
                    break;
                }
            }
        });
        console.detach();

        simulation_thread.join();
        // the last frame's completion callback runs on the stream, so it has
        // started its snapshot thread once the stream is idle
        model.gpu.synchronize();
        // the cycle lock is free again once that thread has written the frame
        model.processing_current_cycle_data.lock();
        if (snapshot_thread.joinable()) snapshot_thread.join();
        model.processing_current_cycle_data.unlock();
        std::printf("cm done: %d frames, step %d, error %d\n", frames_done.load(), model.prms.SimulationStep,
                    model.gpu.error_code);
        std::fflush(stdout);
        std::_Exit(model.gpu.error_code ? 1 : 0);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "cm: %s\n", e.what());
        return 1;
    }
}
