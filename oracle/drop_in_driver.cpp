/*
 * drop_in_driver.cpp -- the reference's time loop with the GPU adapters dropped in.
 *
 * TEST INFRASTRUCTURE (built into oracle/_ref by `make dropin`).  A
 * kielflow.cpp-shaped driver (kielflow.cpp:156-286) that builds the reference's
 * own grid, parameters and fields, then advances the same initial state twice:
 *   1. with the reference's objects: solver_poisson_jacobi_nlin +
 *      solver_poisson_multigrid (the plan of kielflow.cpp:197-217),
 *      rhs_standard and Runge_kutta_O4;
 *   2. with kf_gpu_rhs / kf_gpu_rk4 from include/kf_adapters.hpp in their place,
 *      the loop body unchanged.
 * Usage: drop_in_driver <dir> <n> <M> <tau> <theta> <dt> <nsteps> [m]; with m
 * the axes are axis_CoSiSt(-L/2, L, n, m) (the frontend's grid); <dir> holds
 * state.bin (4 half spectra, interleaved doubles), nd.bin, mask.bin (n^3
 * doubles); writes ref_state.bin and gpu_state.bin.
 */
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "RKO4.hpp"
#include "axis_EqSt.hpp"
#include "axis_SiSt.hpp"
#include "field.hpp"
#include "grid.hpp"
#include "interface_ODE_solver.hpp"
#include "interface_poisson_solver.hpp"
#include "interface_rhs.hpp"
#include "masks.hpp"
#include "parameters.hpp"
#include "rhs_standard.hpp"
#include "solver_poisson_jacobi_nlin.hpp"
#include "solver_poisson_multigrid.hpp"

#include "kf_adapters.hpp"

static bool read_bin(const std::string &p, double *dst, size_t count) {
    FILE *f = std::fopen(p.c_str(), "rb");
    if (!f) return false;
    size_t got = std::fread(dst, sizeof(double), count, f);
    std::fclose(f);
    return got == count;
}

static bool write_bin(const std::string &p, const double *src, size_t count) {
    FILE *f = std::fopen(p.c_str(), "wb");
    if (!f) return false;
    size_t put = std::fwrite(src, sizeof(double), count, f);
    std::fclose(f);
    return put == count;
}

int main(int argc, char **argv) {
    if (argc != 8 && argc != 9) {
        std::fprintf(stderr, "usage: %s dir n M tau theta dt nsteps [m]\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int n = std::atoi(argv[2]);
    const double M = std::atof(argv[3]), tau = std::atof(argv[4]), theta = std::atof(argv[5]);
    const double dt = std::atof(argv[6]);
    const int nsteps = std::atoi(argv[7]);
    const double L = 2. * acos(-1.) * 4.;
    const double m = argc == 9 ? std::atof(argv[8]) : 0.;
    axis_CoEqSt axe(-0.5 * L, L, n);
    axis_CoSiSt axs(-0.5 * L, L, n, m);
    const axis &ax = m != 0. ? static_cast<const axis &>(axs) : static_cast<const axis &>(axe);
    grid Omega(ax, ax, ax);
    parameters Params(M, tau, theta, 0., 0.);
    field_imag FUx(Omega), FUy(Omega), FUz(Omega), Fni(Omega);
    field_real nd(Omega), mask(Omega);
    const size_t Nc = (size_t)FUx.N, N = (size_t)nd.N;
    std::vector<double> st(8 * Nc);
    if (!read_bin(dir + "/state.bin", st.data(), st.size()) || !read_bin(dir + "/nd.bin", nd.val, N) ||
        !read_bin(dir + "/mask.bin", mask.val, N)) {
        std::fprintf(stderr, "cannot read inputs in %s\n", dir.c_str());
        return 3;
    }
    field_imag *F[4] = {&FUx, &FUy, &FUz, &Fni};
    auto load = [&]() {
        for (int q = 0; q < 4; ++q)
            for (size_t i = 0; i < Nc; ++i) {
                F[q]->val[i][0] = st[2 * (q * Nc + i)];
                F[q]->val[i][1] = st[2 * (q * Nc + i) + 1];
            }
    };
    auto store = [&](const std::string &name) {
        std::vector<double> out(8 * Nc);
        for (int q = 0; q < 4; ++q)
            for (size_t i = 0; i < Nc; ++i) {
                out[2 * (q * Nc + i)] = F[q]->val[i][0];
                out[2 * (q * Nc + i) + 1] = F[q]->val[i][1];
            }
        return write_bin(dir + "/" + name, out.data(), out.size());
    };
    try {
        /* 1. the reference's objects (kielflow.cpp:197-240) */
        load();
        {
            fkt3d_const boundary_shape(0.), boundary_value(0.);
            solver_poisson_jacobi_nlin NLJ(boundary_shape, boundary_value, .8);
            NLJ.set_max_iterations(80);
            NLJ.set_limit_NormMax(.5e-5);
            NLJ.set_limit_NormSum(.5e-7);
            solver_poisson_multigrid MG(NLJ);
            int steps[4] = {0, -1, -1, -1};
            MG_lvl_control shape[4] = {lvl_down3, lvl_up, lvl_up, lvl_up};
            double tol[4] = {0.01, 0.0005, 0.0001, 0.0001};
            MG.set_level_control(4, steps, shape, tol);
            field_real Ph(Omega);
            for (size_t i = 0; i < N; ++i) Ph.val[i] = 0.;
            rhs_standard rhs(Params, MG, Ph, nd, mask, Omega);
            Runge_kutta_O4 time_integrator(rhs, dt);
            for (int step = 0; step < nsteps; ++step) time_integrator.solve(FUx, FUy, FUz, Fni);
        }
        if (!store("ref_state.bin")) return 4;
        /* 2. the same loop with the GPU adapters in their place */
        load();
        {
            kf_gpu_rhs rhs(Params, nd, mask, Omega, KF_PS_CASCADIC, KF_T_SHIPPED);
            kf_gpu_rk4 time_integrator(rhs, dt);
            for (int step = 0; step < nsteps; ++step) time_integrator.solve(FUx, FUy, FUz, Fni);
        }
        if (!store("gpu_state.bin")) return 4;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 5;
    } catch (const char *e) {
        std::fprintf(stderr, "error: %s\n", e);
        return 5;
    }
    std::printf("ok\n");
    return 0;
}
