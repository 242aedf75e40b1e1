// txt_driver.cpp -- writes a given state with the C++ drop-in's
// writeFinalResultTo_txt (include/rgrp_2d_cuda.hpp), so its files can be
// compared with the reference's writeMatrixTo_txt (src/wrappers.cuh:370-397)
// without a GPU.  Usage: txt_driver IN DIR, IN as oracle/ref_txt.cu reads it.
#include "rgrp_2d_cuda.hpp"

#include <cstdio>

// The result and end time are protected members set by solve(); this test
// sets them directly.
struct TxtProbe : RGRP_2D_CUDA {
    void load(const std::vector<std::vector<vec5d>> &U, double t)
    {
        U_ = U;
        endTime_ = t;
    }
};

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int nx = 0, ny = 0;
    double t = 0.0;
    if (std::fread(&nx, 4, 1, f) != 1 || std::fread(&ny, 4, 1, f) != 1 || std::fread(&t, 8, 1, f) != 1) return 2;
    std::vector<std::vector<vec5d>> M(ny, std::vector<vec5d>(nx));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            double c[4];
            if (std::fread(c, 8, 4, f) != 4) return 2;
            M[j][i] = vec5d{c[0], c[1], c[2], c[3], 0.0};
        }
    std::fclose(f);
    TxtProbe p;
    p.load(M, t);
    p.writeFinalResultTo_txt(argv[2]);
    return 0;
}
