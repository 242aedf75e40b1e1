/*
 * ref_gpu.cu -- the reference's own CUDA kernels (src/basicFuns.cuh,
 * src/ghostCellPresets.cuh, compiled unchanged by nvcc for sm_100a) driven in
 * the exact launch sequence of RGRP_2D_CUDA::solve() (src/wrappers.cuh:154-306):
 * the same buffers, 16x16 blocks, cudaDeviceSynchronize after every kernel,
 * the thrust max reduction read back to the host every step, the device
 * copy, the memsets of the unused edited-flag buffers and the std::chrono
 * loop timer of wrappers.cuh:193,286-288.
 *
 * TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/ from
 * the reference sources; used by GPU parity tests and by bench.py to time the
 * reference's own CUDA build on the same B200.  wrappers.cuh itself includes
 * OpenCV (absent here) for its PNG recorder, so its loop is restated call for
 * call instead of compiled.
 *
 * Usage: ref_gpu IN OUT
 *   IN : int32 nx, ny, strategy, max_steps; float64 width, height, cfl,
 *        alpha, gamma, t_end; then nx*ny*4 float64 (rho, p, u, v) row-major.
 *   OUT: int32 steps, pad; float64 t, loop_ms, kernel_ms; then the state.
 * Only sizes that are multiples of 16 are accepted (set_ghost_cells has no
 * bounds check, ghostCellPresets.cuh:106-145).
 */
#include "basicFuns.cuh"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <vector>

#define CK(x)                                                                  \
    do {                                                                       \
        cudaError_t e_ = (x);                                                  \
        if (e_ != cudaSuccess) {                                               \
            fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            exit(3);                                                           \
        }                                                                      \
    } while (0)

int main(int argc, char **argv)
{
    if (argc != 3) { fprintf(stderr, "usage: ref_gpu IN OUT\n"); return 2; }
    FILE *f = fopen(argv[1], "rb");
    if (!f) { perror("open IN"); return 2; }
    int hdr[4];
    double par[6];
    if (fread(hdr, sizeof(int), 4, f) != 4 || fread(par, sizeof(double), 6, f) != 6) return 2;
    const int Nx = hdr[0], Ny = hdr[1], strategy = hdr[2], max_steps = hdr[3];
    const double width = par[0], height = par[1], CFL = par[2], alpha = par[3], gamma = par[4], endTime = par[5];
    if (Nx < 16 || Ny < 16 || Nx % 16 || Ny % 16 || strategy < 0 || strategy > 4) {
        fprintf(stderr, "unsupported size or strategy\n");
        return 2;
    }
    const int num_cells = Nx * Ny;
    std::vector<vec5d> U0(num_cells);
    std::vector<double> raw((size_t)num_cells * 4);
    if (fread(raw.data(), sizeof(double), raw.size(), f) != raw.size()) return 2;
    fclose(f);
    for (int k = 0; k < num_cells; ++k)
        U0[k] = vec5d(raw[4 * k], raw[4 * k + 1], raw[4 * k + 2], raw[4 * k + 3], 0.0);

    vec5d *u_dev, *u_dev_copy, *u_u_t_interface_dev, *u_lr_interface_dev, *u_y_dev;
    vec5d *u_u_t_y_interface_dev, *u_lr_y_interface_dev, *u_slope_dev, *u_slope_y_dev;
    double *speed;
    int *c_lr_interface_edited_dev, *c_lr_interface_y_edited_dev;
    CK(cudaMalloc(&u_dev, num_cells * sizeof(vec5d)));
    CK(cudaMalloc(&u_u_t_interface_dev, (num_cells + Ny) * 2 * sizeof(vec5d)));
    CK(cudaMalloc(&u_lr_interface_dev, (num_cells + Ny) * 2 * sizeof(vec5d)));
    CK(cudaMalloc(&u_u_t_y_interface_dev, (num_cells + Nx) * 2 * sizeof(vec5d)));
    CK(cudaMalloc(&u_y_dev, num_cells * sizeof(vec5d)));
    CK(cudaMalloc(&u_dev_copy, num_cells * sizeof(vec5d)));
    CK(cudaMalloc(&c_lr_interface_edited_dev, (num_cells + Ny) * 2 * sizeof(int)));
    CK(cudaMalloc(&c_lr_interface_y_edited_dev, (num_cells + Ny) * 2 * sizeof(int)));
    CK(cudaMalloc(&u_lr_y_interface_dev, (num_cells + Nx) * 2 * sizeof(vec5d)));
    CK(cudaMalloc(&u_slope_dev, num_cells * sizeof(vec5d)));
    CK(cudaMalloc(&u_slope_y_dev, num_cells * sizeof(vec5d)));
    CK(cudaMalloc(&speed, num_cells * sizeof(double)));
    CK(cudaMemset(u_slope_dev, 0, num_cells * sizeof(vec5d)));
    CK(cudaMemset(c_lr_interface_edited_dev, 0, (num_cells + Ny) * 2 * sizeof(int)));
    CK(cudaMemset(c_lr_interface_y_edited_dev, 0, (num_cells + Ny) * 2 * sizeof(int)));
    CK(cudaMemcpy(u_dev, U0.data(), num_cells * sizeof(vec5d), cudaMemcpyHostToDevice));

    dim3 blockSize(16, 16);
    dim3 gridSize((Nx + blockSize.x - 1) / blockSize.x, (Ny + blockSize.y - 1) / blockSize.y);
    dim3 gridSize_y((Ny + blockSize.y - 1) / blockSize.y, (Nx + blockSize.x - 1) / blockSize.x);

    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    double cTime = 0.0;
    int steps = 0;
    CK(cudaDeviceSynchronize());
    CK(cudaEventRecord(ev0));
    auto start = std::chrono::high_resolution_clock::now();
    while (cTime < endTime && (max_steps < 0 || steps < max_steps)) {
        maxPropagtingSpeed<<<gridSize, blockSize>>>(u_dev, speed, Nx, Ny, gamma);
        cudaDeviceSynchronize();
        thrust::device_ptr<double> p_speed = thrust::device_pointer_cast(speed);
        double max_speed = reduce(p_speed, p_speed + num_cells, -std::numeric_limits<double>::infinity(), thrust::maximum<double>());
        double h = std::min(width / double(Nx), height / double(Ny));
        double dt = std::min(CFL * h / max_speed, endTime - cTime);
        if (h / max_speed < 1e-20) break;

        cudaMemcpy(u_dev_copy, u_dev, num_cells * sizeof(vec5d), cudaMemcpyDeviceToDevice);

        MUSCL_rel_RP_GRP<<<gridSize, blockSize>>>(u_dev, u_slope_dev, Nx, Ny, alpha, width, u_lr_interface_dev);
        cudaDeviceSynchronize();
        rel_RP_posi_fix<<<gridSize, blockSize>>>(u_dev, u_slope_dev, u_lr_interface_dev, Nx, Ny, u_u_t_interface_dev, c_lr_interface_edited_dev, gamma);
        cudaDeviceSynchronize();
        forward_x_dir<<<gridSize, blockSize>>>(u_dev, u_u_t_interface_dev, Nx, Ny, width, dt, gamma);
        cudaDeviceSynchronize();
        rotate_and_flip_vertically<<<gridSize, blockSize>>>(u_dev, u_y_dev, Nx, Ny);
        cudaDeviceSynchronize();
        MUSCL_rel_RP_GRP<<<gridSize_y, blockSize>>>(u_y_dev, u_slope_y_dev, Ny, Nx, alpha, height, u_lr_y_interface_dev);
        cudaDeviceSynchronize();
        rel_RP_posi_fix<<<gridSize_y, blockSize>>>(u_y_dev, u_slope_y_dev, u_lr_y_interface_dev, Ny, Nx, u_u_t_y_interface_dev, c_lr_interface_y_edited_dev, gamma);
        cudaDeviceSynchronize();
        forward_x_dir<<<gridSize_y, blockSize>>>(u_y_dev, u_u_t_y_interface_dev, Ny, Nx, height, dt, gamma);
        cudaDeviceSynchronize();
        rotate_and_flip_vertically<<<gridSize_y, blockSize>>>(u_y_dev, u_dev, Ny, Nx);
        cudaDeviceSynchronize();

        cudaMemset(c_lr_interface_edited_dev, 0, (num_cells + Ny) * 2 * sizeof(int));
        cudaMemset(c_lr_interface_y_edited_dev, 0, (num_cells + Ny) * 2 * sizeof(int));

        rotate_and_flip_vertically<<<gridSize, blockSize>>>(u_dev_copy, u_y_dev, Nx, Ny);
        cudaDeviceSynchronize();
        MUSCL_rel_RP_GRP<<<gridSize_y, blockSize>>>(u_y_dev, u_slope_y_dev, Ny, Nx, alpha, height, u_lr_y_interface_dev);
        cudaDeviceSynchronize();
        rel_RP_posi_fix<<<gridSize_y, blockSize>>>(u_y_dev, u_slope_y_dev, u_lr_y_interface_dev, Ny, Nx, u_u_t_y_interface_dev, c_lr_interface_y_edited_dev, gamma);
        cudaDeviceSynchronize();
        forward_x_dir<<<gridSize_y, blockSize>>>(u_y_dev, u_u_t_y_interface_dev, Ny, Nx, height, dt, gamma);
        cudaDeviceSynchronize();
        rotate_and_flip_vertically<<<gridSize_y, blockSize>>>(u_y_dev, u_dev_copy, Ny, Nx);
        cudaDeviceSynchronize();
        MUSCL_rel_RP_GRP<<<gridSize, blockSize>>>(u_dev_copy, u_slope_dev, Nx, Ny, alpha, width, u_lr_interface_dev);
        cudaDeviceSynchronize();
        rel_RP_posi_fix<<<gridSize, blockSize>>>(u_dev_copy, u_slope_dev, u_lr_interface_dev, Nx, Ny, u_u_t_interface_dev, c_lr_interface_edited_dev, gamma);
        cudaDeviceSynchronize();
        forward_x_dir<<<gridSize, blockSize>>>(u_dev_copy, u_u_t_interface_dev, Nx, Ny, width, dt, gamma);
        cudaDeviceSynchronize();

        combineResults<<<gridSize, blockSize>>>(u_dev, u_dev_copy, Nx, Ny);

        cTime += dt;
        ++steps;

        if (strategy == 0)
            set_ghost_cells<<<gridSize, blockSize>>>(u_dev, Nx, Ny, width, height, cTime);
        else if (strategy == 2)
            set_ghost_cells_jet<<<gridSize, blockSize>>>(u_dev, Nx, Ny, width, height, cTime);
        else if (strategy == 3)
            set_ghost_cells_jet800<<<gridSize, blockSize>>>(u_dev, Nx, Ny, width, height, cTime);
        else
            set_ghost_cells_2Mach<<<gridSize, blockSize>>>(u_dev, Nx, Ny, width, height, cTime);
        cudaDeviceSynchronize();
        cudaMemset(c_lr_interface_edited_dev, 0, (num_cells + Ny) * 2 * sizeof(int));
        cudaMemset(c_lr_interface_y_edited_dev, 0, (num_cells + Ny) * 2 * sizeof(int));
    }
    auto end = std::chrono::high_resolution_clock::now();
    CK(cudaEventRecord(ev1));
    CK(cudaEventSynchronize(ev1));
    CK(cudaGetLastError());
    float kms = 0.f;
    CK(cudaEventElapsedTime(&kms, ev0, ev1));
    double loop_ms = std::chrono::duration_cast<std::chrono::microseconds>(end - start).count() / 1000.0;

    CK(cudaMemcpy(U0.data(), u_dev, num_cells * sizeof(vec5d), cudaMemcpyDeviceToHost));
    for (int k = 0; k < num_cells; ++k)
        for (int c = 0; c < 4; ++c) raw[4 * k + c] = U0[k][c];
    FILE *g = fopen(argv[2], "wb");
    if (!g) { perror("open OUT"); return 2; }
    int o[2] = {steps, 0};
    double d[3] = {cTime, loop_ms, (double)kms};
    fwrite(o, sizeof(int), 2, g);
    fwrite(d, sizeof(double), 3, g);
    fwrite(raw.data(), sizeof(double), raw.size(), g);
    fclose(g);
    cudaFree(u_dev); cudaFree(u_u_t_interface_dev); cudaFree(u_lr_interface_dev);
    cudaFree(u_u_t_y_interface_dev); cudaFree(u_y_dev); cudaFree(u_dev_copy);
    cudaFree(c_lr_interface_edited_dev); cudaFree(c_lr_interface_y_edited_dev);
    cudaFree(u_lr_y_interface_dev); cudaFree(u_slope_dev); cudaFree(u_slope_y_dev);
    cudaFree(speed);
    return 0;
}
