// A program written against the reference's solver class (src/wrappers.cuh):
// only its include line differs.  Used by tests/test_drop_in.py, which builds
// it with g++ against include/rgrp_2d_cuda.hpp and libfvm2d.so.
//   drop_in_driver <n> <strategy> <out.bin> [record_dir]
// writes n, steps, the computation time and the final (n, n, 5) cells.
#include "rgrp_2d_cuda.hpp"

#include <cstdio>
#include <cstdlib>

int main(int argc, char **argv)
{
    if (argc < 4) return 2;
    const int n = std::atoi(argv[1]);
    const int strategy = std::atoi(argv[2]);
    RGRP_2D_CUDA solver;
    solver.setRPInitialData(vec5d(1.5, 1.5, 0.0, 0.0, 0.0), vec5d(0.5323, 0.3, 1.206, 0.0, 0.0),
                            vec5d(0.138, 0.029, 1.206, 1.206, 0.0), vec5d(0.5323, 0.3, 0.0, 1.206, 0.0), n, n);
    solver.setSpatialLayout(1.0, 1.0);
    solver.setTimeLayout(0.05, 0.45);
    solver.setAlpha(1.9);
    solver.setGamma(1.4);
    solver.setGhostCellStrategy(static_cast<ghostCellStrategy>(strategy));
    if (argc > 4) solver.setRecordModel(true, 10, argv[4]);
    std::vector<std::vector<vec5d>> U;
    try {
        U = solver.solve();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    FILE *f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    const int steps = solver.getTimeStagesCount();
    const double ms = solver.getComputationTime_ms();
    std::fwrite(&n, sizeof n, 1, f);
    std::fwrite(&steps, sizeof steps, 1, f);
    std::fwrite(&ms, sizeof ms, 1, f);
    for (const auto &row : U)
        for (const auto &c : row) std::fwrite(c.data, sizeof(double), 5, f);
    std::fclose(f);
    return 0;
}
