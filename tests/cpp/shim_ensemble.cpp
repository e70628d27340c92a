// Two small indentation scenes advanced together through the header-only
// icy::Ensemble (icm_ensemble_*): each case is an icy::Model set up as for
// Step; after run(n) each case's particle SoA is written to argv[2] + ".<i>"
// (raw doubles) and "ensemble ok" is printed. Without a CUDA device the
// first call that needs one throws and the program exits 3.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>
#include "icempm.hpp"

int main(int argc, char **argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: shim_ensemble config.json out_prefix substeps cells_x [cells_y]\n");
        return 2;
    }
    const int n = std::atoi(argv[3]);
    std::vector<std::unique_ptr<icy::Model>> cases;
    try {
        icy::Ensemble ens(ICM_FORM_FP32, 1, 128, 0);
        for (int i = 0; i < 2; i++) {
            auto m = std::make_unique<icy::Model>();
            icy::SimParams &p = m->prms;
            p.ParseFile(argv[1]);
            icm_block_desc d{};
            d.cells_x = std::atoi(argv[4]) + 8 * i;
            d.cells_y = argc > 5 ? std::atoi(argv[5]) : 8;
            d.ind_y_above_floor = 0.05;
            d.grain_size = 0.02;
            d.seed = 7 + i;
            int np = 0;
            if (icm_scene_block(&p, &d, nullptr, &np) != ICM_OK) {
                std::printf("scene: %s\n", icm_last_error());
                return 1;
            }
            m->gpu.cuda_allocate_arrays((size_t)p.GridX * p.GridY, (size_t)np);
            if (icm_scene_block(&p, &d, m->gpu.tmp_transfer_buffer, &np) != ICM_OK) {
                std::printf("scene: %s\n", icm_last_error());
                return 1;
            }
            m->gpu.transfer_ponts_to_device();
            m->Reset();
            m->Prepare();
            ens.add(*m);
            cases.push_back(std::move(m));
        }
        ens.set(4);
        ens.run(n);
        for (size_t i = 0; i < cases.size(); i++) {
            icy::Model &m = *cases[i];
            m.gpu.transfer_completion_callback = []() {};
            m.gpu.cuda_transfer_from_device();
            m.gpu.synchronize();
            const size_t count = (size_t)m.prms.nPtsPitch * ICM_N_PTS_ARRAYS;
            std::string path = std::string(argv[2]) + "." + std::to_string(i);
            FILE *f = std::fopen(path.c_str(), "wb");
            if (!f || std::fwrite(m.gpu.tmp_transfer_buffer, sizeof(double), count, f) != count) return 1;
            std::fclose(f);
            std::printf("case %zu step %d error %d\n", i, m.prms.SimulationStep, m.gpu.error_code);
        }
    } catch (const std::runtime_error &e) {
        std::printf("no device: %s\n", e.what());
        return 3;
    }
    std::printf("ensemble ok\n");
    return 0;
}
