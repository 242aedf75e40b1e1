// rgrp_2d_cuda.hpp -- source-compatible replacement for the reference's
// src/wrappers.cuh (class RGRP_2D_CUDA, enum class ghostCellStrategy) and
// the vec5d type of src/ghostCellPresets.cuh, running on libfvm2d.so.
//
// A program written against the reference switches by replacing
//     #include "./src/wrappers.cuh"
// with
//     #include "rgrp_2d_cuda.hpp"
// and linking -lfvm2d.  It compiles with any C++17 host compiler (nvcc is not
// needed).  Differences from the reference, all at the edges of the hot path:
//  - failures throw std::runtime_error with the library's message (the
//    reference checks no CUDA call);
//  - setRecordModel frames are rendered on the GPU and written without
//    OpenCV; they show the state after each recorded step's ghost fill;
//  - ghostCellStrategy gains `periodic` and `reflective_tb`.
#pragma once

#include "fvm2d.h"

#include <array>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

// 5-double cell (rho, p, u, v, unused); arithmetic touches slots 0-3 only,
// as src/ghostCellPresets.cuh:4-45.
struct vec5d {
    vec5d() : data{0.0, 0.0, 0.0, 0.0, 0.0} {}
    vec5d(double x0, double x1, double x2, double x3, double x4) : data{x0, x1, x2, x3, x4} {}
    double &operator[](size_t i) { return data[i]; }
    const double &operator[](size_t i) const { return data[i]; }
    double &operator()(size_t i) { return data[i]; }
    const double &operator()(size_t i) const { return data[i]; }
    vec5d operator+(const vec5d &v) const
    {
        vec5d r;
        for (int i = 0; i < 4; ++i) r[i] = data[i] + v[i];
        return r;
    }
    vec5d operator-(const vec5d &v) const
    {
        vec5d r;
        for (int i = 0; i < 4; ++i) r[i] = data[i] - v[i];
        return r;
    }
    vec5d operator*(double a) const
    {
        vec5d r;
        for (int i = 0; i < 4; ++i) r[i] = data[i] * a;
        return r;
    }
    double data[5];
};

enum class ghostCellStrategy {
    outflow = FVM2D_OUTFLOW,
    reflective = FVM2D_REFLECTIVE,  // runs the double-Mach preset, as the reference does
    jet = FVM2D_JET,
    jet800 = FVM2D_JET800,
    doubleMach = FVM2D_DOUBLE_MACH,
    periodic = FVM2D_PERIODIC,
    reflective_tb = FVM2D_REFLECTIVE_TB
};

class RGRP_2D_CUDA {
public:
    explicit RGRP_2D_CUDA(const std::vector<std::vector<vec5d>> &U0)
    {
        for (const auto &row : U0)
            for (const auto &u : row) U0_.push_back(u);
        Nx_ = (int)U0[0].size();
        Ny_ = (int)U0.size();
    }
    RGRP_2D_CUDA() {}
    RGRP_2D_CUDA(const RGRP_2D_CUDA &) = delete;
    RGRP_2D_CUDA &operator=(const RGRP_2D_CUDA &) = delete;
    ~RGRP_2D_CUDA() { release(); }

    void setRPInitialData(const vec5d &U1, const vec5d &U2, const vec5d &U3, const vec5d &U4, int Nx, int Ny)
    {
        U0_.assign((size_t)Nx * Ny, vec5d());
        Nx_ = Nx;
        Ny_ = Ny;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i)
                U0_[(size_t)j * Nx + i] = (i < Nx / 2) ? (j < Ny / 2 ? U2 : U3) : (j < Ny / 2 ? U1 : U4);
    }
    void setSpatialLayout(double width, double height) { width_ = width, height_ = height; }
    void setTimeLayout(double endTime, double CFL) { endTime_ = endTime, CFL_ = CFL; }
    void setTimeLayout(double endTime) { endTime_ = endTime; }
    void setCFL(double CFL) { CFL_ = CFL; }
    void setAlpha(double alpha) { alpha_ = alpha; }
    void setGamma(double gamma) { gamma_ = gamma; }
    void setGhostCellStrategy(ghostCellStrategy strategy) { strategy_ = strategy; }
    // FVM2D_FP64 (default), FVM2D_FP64_STRICT, FVM2D_FP64_REFORDER, FVM2D_FP32 or FVM2D_FP32_RESIDUAL;
    // no reference counterpart.
    void setPrecision(int precision) { precision_ = precision; }
    void setRecordModel(bool on_off, int gapPerFrame = 10, const std::string &recordDir = ".")
    {
        record_ = on_off;
        gap_ = gapPerFrame;
        recordDir_ = recordDir;
    }

    std::vector<std::vector<vec5d>> solve()
    {
        if (U0_.empty()) throw std::runtime_error("no initial data");
        if (!h_ || hnx_ != Nx_ || hny_ != Ny_) {
            release();
            ok(fvm2d_create(&h_, Nx_, Ny_));
            hnx_ = Nx_;
            hny_ = Ny_;
        }
        ok(fvm2d_set_spatial_layout(h_, width_, height_));
        ok(fvm2d_set_time_layout(h_, endTime_, CFL_));
        ok(fvm2d_set_alpha(h_, alpha_));
        ok(fvm2d_set_gamma(h_, gamma_));
        ok(fvm2d_set_ghost_strategy(h_, (int)strategy_));
        ok(fvm2d_set_precision(h_, precision_));
        ok(fvm2d_set_record_model(h_, record_ ? 1 : 0, gap_, recordDir_.c_str()));
        ok(fvm2d_set_state(h_, U0_[0].data, 5));
        ok(fvm2d_solve(h_));
        ok(fvm2d_get_computation_time_ms(h_, &ms_));
        long long n = 0;
        ok(fvm2d_get_time_stages_count(h_, &n));
        stages_ = (int)n;
        // like src/wrappers.cuh:290, the result also becomes the next initial data
        ok(fvm2d_get_state(h_, U0_[0].data, 5));
        U_.assign(Ny_, std::vector<vec5d>(Nx_));
        for (int j = 0; j < Ny_; ++j)
            for (int i = 0; i < Nx_; ++i) U_[j][i] = U0_[(size_t)j * Nx_ + i];
        return U_;
    }
    double getComputationTime_ms() { return ms_; }
    int getTimeStagesCount() { return stages_; }
    // Mass, x momentum, y momentum and energy of the last result's interior
    // cells, summed in FP64 (fvm2d_get_conserved_totals; no reference
    // counterpart).
    std::array<double, 4> getConservedTotals()
    {
        if (!h_) throw std::runtime_error("no result: call solve() first");
        std::array<double, 4> t{};
        ok(fvm2d_get_conserved_totals(h_, t.data()));
        return t;
    }
    void writeFinalResultTo_txt(const std::string &dir)
    {
        // src/wrappers.cuh:370-397: one file per field, default stream formatting
        const char *names[4] = {"rho", "p", "u", "v"};
        for (int f = 0; f < 4; ++f) {
            std::ofstream out(dir + "/" + names[f] + "_" + std::to_string(endTime_) + "s.txt");
            if (!out.is_open()) continue;
            for (const auto &row : U_) {
                for (const auto &e : row) out << e(f) << " ";
                out << "\n";
            }
        }
    }
    void clear()
    {
        U0_.clear();
        U_.clear();
        release();
    }

protected:
    std::vector<vec5d> U0_;
    std::vector<std::vector<vec5d>> U_;
    double width_ = 1.0, height_ = 1.0, endTime_ = 0.0, CFL_ = 0.5;
    double alpha_ = 1.9, gamma_ = 1.4;
    int Nx_ = 100, Ny_ = 100;
    ghostCellStrategy strategy_ = ghostCellStrategy::outflow;
    int precision_ = FVM2D_FP64;
    bool record_ = false;
    int gap_ = 10;
    std::string recordDir_ = ".";
    double ms_ = 0.0;
    int stages_ = 0;
    fvm2d_solver *h_ = nullptr;
    int hnx_ = 0, hny_ = 0;

    static void ok(int rc)
    {
        if (rc != FVM2D_OK) throw std::runtime_error(std::string("libfvm2d: ") + fvm2d_last_error());
    }
    void release()
    {
        if (h_) fvm2d_destroy(h_);
        h_ = nullptr;
    }
};
