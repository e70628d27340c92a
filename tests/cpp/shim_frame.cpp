// Drives one frame of a small indentation scene through the header-only
// GPU_Implementation5 / icy::Model shim, the way iceMPM's CLI drives its
// model (cli.cpp:28-50): ParseFile, a synthetic block, allocate, upload,
// Reset, Prepare, Step, wait for the completion callback. Writes the
// particle SoA after the frame to argv[2] (raw doubles) and prints
// "frame ok <n> ...".
// Without a CUDA device, initialize() throws and the program prints the
// message and exits 3.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "icempm.hpp"

int main(int argc, char **argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: shim_frame config.json out.bin form cells_x cells_y\n");
        return 2;
    }
    icy::Model model;
    icy::SimParams &p = model.prms;
    try {
        std::string raw = p.ParseFile(argv[1]);
        std::printf("raw points: %s\n", raw.c_str());
    } catch (const std::runtime_error &e) {
        std::printf("config: %s\n", e.what());
        return 1;
    }
    icm_block_desc d{};
    d.cells_x = std::atoi(argv[4]);
    d.cells_y = argc > 5 ? std::atoi(argv[5]) : 8;
    d.ind_y_above_floor = 0.05;
    d.grain_size = 0.02;
    d.seed = 7;
    int n = 0;
    // first call sizes the block, second fills the SoA
    if (icm_scene_block(&p, &d, nullptr, &n) != ICM_OK) {
        std::printf("scene: %s\n", icm_last_error());
        return 1;
    }
    try {
        model.gpu.cuda_allocate_arrays((size_t)p.GridX * p.GridY, (size_t)n);
    } catch (const std::runtime_error &e) {
        std::printf("no device: %s\n", e.what());
        return 3;
    }
    if (icm_scene_block(&p, &d, model.gpu.tmp_transfer_buffer, &n) != ICM_OK) {
        std::printf("scene: %s\n", icm_last_error());
        return 1;
    }
    model.gpu.set_form(std::atoi(argv[3]));
    model.gpu.transfer_ponts_to_device();
    model.Reset();
    model.Prepare();
    std::atomic<int> done{0};
    model.gpu.transfer_completion_callback = [&]() {
        done = 1;
        model.UnlockCycleMutex();
    };
    model.Step();
    model.gpu.synchronize();
    if (!done) {
        std::printf("callback did not run\n");
        return 1;
    }
    std::FILE *f = std::fopen(argv[2], "wb");
    if (!f) return 1;
    std::fwrite(model.gpu.tmp_transfer_buffer, sizeof(double), p.nPtsPitch * icy::SimParams::nPtsArrays, f);
    std::fclose(f);
    std::printf("frame ok %d step %d err %d\n", n, p.SimulationStep, model.gpu.error_code);
    return model.gpu.error_code ? 1 : 0;
}
