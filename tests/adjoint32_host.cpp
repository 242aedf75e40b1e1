// adjoint32_host.cpp -- the FP32 build's differentiation path compiled for
// the host: its taped forward step (PackedCompensated work items on FP32
// planes) and the adjoint step's kernels in single precision
// (2d_fvm_cuda_b200/csrc/fvm2d_adjoint.inc with FVM2D_REAL float, as
// fvm2d_adjoint32.cu builds them), so that the CPU tests can compare its
// vector-Jacobian product with the FP64 one of tests/kernels_host.cpp.
// tests/test_kernels_host.py builds it and calls it through ctypes.
#include "cuda_host_emu.h"

#define FVM2D_VARIANT host32
#define FVM2D_REAL float
#include "../2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_dual.cuh"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_adjoint.inc"
#include "../2d_fvm_cuda_b200/csrc/fvm2d_packed.cuh"

using namespace fvm2d::host32;
using fvm2d::ad::Dual;

#include "kernels_host_steps.h"

extern "C" {

// in_b = (d step at cells)^T out_b for the FP32 build's step: the taped
// forward in FP32, then the FP32 adjoint kernels in the launcher's order.
// Arrays are (ny, nx, 4) doubles; the state and cotangent are rounded to
// FP32 on the way in.
int k32_step_vjp(const double *cells, const double *out_b, int nx, int ny, int strategy, double t, double dt,
                 double width, double height, double alpha, double gamma, int T, double *in_b)
{
    if (nx < 6 || ny < 6) return 1;
    const double hx = width / nx, hy = height / ny;
    Planes<float> U(nx, ny), A1(nx, ny), B1(nx, ny), V(nx, ny);
    Planes<float> flux[4] = {Planes<float>(nx, ny), Planes<float>(nx, ny), Planes<float>(nx, ny),
                             Planes<float>(nx, ny)};
    cells_to(U, cells, nullptr);
    forward_step<float, true, PackedCompensated>(U, A1, B1, V, flux, strategy, t, dt, hx, hy, alpha, gamma, T);
    Planes<float> lb(nx, ny), H(nx, ny), T1(nx, ny), T2(nx, ny), out(nx, ny);
    cells_to(lb, out_b, nullptr);
    const GhostGeom gg{nx, ny, strategy};
    Field<float> lbf = lb.field(), Hf = H.field();
    emu::launch(dim3((nx + 31) / 32, (ny + 7) / 8), dim3(32, 8), false,
                [&] { ghost_adjoint_copy(lbf, Hf, gg, 0.5f); });
    const int ring = 4 * nx + 4 * (ny - 4);
    emu::launch(dim3((ring + 255) / 256), dim3(256), false, [&] { ghost_adjoint_scatter(lbf, Hf, gg, 0.5f); });
    transpose(1, A1, flux[2], H, T1, nullptr, hy, dt, alpha, gamma);
    transpose(0, U, flux[0], T1, T2, nullptr, hx, dt, alpha, gamma);
    transpose(0, B1, flux[3], H, T1, nullptr, hx, dt, alpha, gamma);
    transpose(1, U, flux[1], T1, out, &T2, hy, dt, alpha, gamma);
    for (long long c = 0; c < out.plane; ++c)
        for (int f = 0; f < 4; ++f) in_b[4 * c + f] = double(out.v[f * out.plane + c]);
    return 0;
}

} // extern "C"
