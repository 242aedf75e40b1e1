/*
 * ref_txt.cu -- the reference's own text writer, RGRP_2D_CUDA::writeMatrixTo_txt
 * (src/wrappers.cuh:370-397, reached by writeFinalResultTo_txt at
 * src/wrappers.cuh:318-321), compiled unchanged from the reference's header
 * with the OpenCV stand-in of oracle/opencv_stub (its PNG recorder is never
 * called).  Runs on the host only: no CUDA call is made.
 *
 * TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/ref_txt;
 * tests/test_txt_writer.py compares the library's C++ and Python writers with
 * it byte for byte.
 *
 * Usage: ref_txt IN DIR
 *   IN : int32 nx, ny; float64 t; then nx*ny*4 float64 (rho, p, u, v) row-major.
 *   Writes DIR/rho_<t>s.txt, p_, u_, v_ as the reference does.
 */
#include "wrappers.cuh"

#include <cstdio>

// writeMatrixTo_txt is a protected static member: a derived class names it.
struct TxtWriter : RGRP_2D_CUDA {
    using RGRP_2D_CUDA::writeMatrixTo_txt;
};

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: ref_txt IN DIR\n");
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    int nx = 0, ny = 0;
    double t = 0.0;
    if (fread(&nx, 4, 1, f) != 1 || fread(&ny, 4, 1, f) != 1 || fread(&t, 8, 1, f) != 1 || nx < 1 || ny < 1) return 2;
    vector<vector<vec5d>> M(ny, vector<vec5d>(nx));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            double c[4];
            if (fread(c, 8, 4, f) != 4) return 2;
            M[j][i] = vec5d{c[0], c[1], c[2], c[3], 0.0};
        }
    fclose(f);
    TxtWriter::writeMatrixTo_txt(argv[2], M, t);
    return 0;
}
