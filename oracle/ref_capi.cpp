/*
 * ref_capi.cpp -- C entry points over the reference's own hot-path classes.
 *
 * TEST INFRASTRUCTURE (oracle/_ref).  Compiled together with the reference's
 * unmodified sources (RKO4.cpp, rhs_standard.cpp, OP_*.cpp, operations.cpp,
 * field_*.cpp, field_interpolation.cpp, axis_EqSt.cpp, axis_SiSt.cpp, grid_base.cpp,
 * solver_poisson_jacobi_nlin.cpp, solver_poisson_multigrid.cpp, parameters.cpp,
 * effect_penalization.cpp, effect_diffusion.cpp)
 * so that the Python tests can drive the reference exactly as its driver does
 * (kielflow.cpp:156-286) on seeded in-memory inputs instead of HDF5 files.
 * This file only wires objects together; every number comes from reference code.
 */
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "RKO4.hpp"
#include "axis_EqSt.hpp"
#include "axis_SiSt.hpp"
#include "effect_diffusion.hpp"
#include "effect_penalization.hpp"
#include "field.hpp"
#include "grid.hpp"
#include "masks.hpp"
#include "operations.hpp"
#include "OP_FFT.hpp"
#include "OP_iFFT.hpp"
#include "OP_dealiasing.hpp"
#include "OP_partial_derivative.hpp"
#include "field_interpolation.hpp"
#include "parameters.hpp"
#include "rhs_standard.hpp"
#include "solver_poisson_jacobi_nlin.hpp"
#include "solver_poisson_multigrid.hpp"

namespace {

grid make_grid(int n, double L, double m = 0.) {
    if (m != 0.) {
        axis_CoSiSt ax(-0.5 * L, L, n, m);
        return grid(ax, ax, ax);
    }
    axis_CoEqSt ax(-0.5 * L, L, n);
    return grid(ax, ax, ax);
}

/* rhs_standard keeps its spectral-viscosity table protected; expose it. */
struct rhs_probe : public rhs_standard {
    using rhs_standard::rhs_standard;
    const double *sv() const { return field_SV; }
};

std::string g_err;
int g_rk4_n = -1; /* Runge_kutta_O4 keeps function-static buffers (RKO4.cpp:68-72) */

}  // namespace

struct kfref_ctx {
    int n;
    double L;
    grid omega;
    parameters params;
    field_imag FUx, FUy, FUz, Fni;
    field_real nd, mask, Phi;
    fkt3d_const bshape, bvalue;
    solver_poisson_jacobi_nlin nlj;
    solver_poisson_multigrid mg;
    std::unique_ptr<rhs_probe> rhs;
    kfref_ctx(int n_, double L_, double M, double tau, double theta, double m)
        : n(n_), L(L_), omega(make_grid(n_, L_, m)), params(M, tau, theta, 0., 0.),
          FUx(omega), FUy(omega), FUz(omega), Fni(omega), nd(omega), mask(omega), Phi(omega),
          bshape(0.), bvalue(0.), nlj(bshape, bvalue, .8), mg(nlj) {
        for (int i = 0; i < nd.N; ++i) nd.val[i] = mask.val[i] = Phi.val[i] = 0.;
        for (int i = 0; i < FUx.N; ++i)
            FUx.val[i][0] = FUx.val[i][1] = FUy.val[i][0] = FUy.val[i][1] = FUz.val[i][0] =
                FUz.val[i][1] = Fni.val[i][0] = Fni.val[i][1] = 0.;
    }
};

extern "C" {

const char *kfref_last_error(void) { return g_err.c_str(); }

/* poisson_mode 0: the nonlinear Jacobi solver used directly as the RHS's
 * interface_poisson_solver (max_it sweeps, relative-update limit);
 * poisson_mode 1: the cascadic multigrid plan of kielflow.cpp:199-217.
 * m: 0 for axis_CoEqSt axes, else axis_CoSiSt(-L/2, L, n, m) axes (the
 * frontend's grid, frontend.cpp:285-287). */
kfref_ctx *kfref_create(int n, double L, double M, double tau, double theta, int poisson_mode,
                        int nlj_max_it, double nlj_limit_max, double m) {
    try {
        kfref_ctx *c = new kfref_ctx(n, L, M, tau, theta, m);
        c->nlj.set_max_iterations(nlj_max_it);
        c->nlj.set_limit_NormMax(nlj_limit_max);
        c->nlj.set_limit_NormSum(.5e-7);
        interface_poisson_solver *ps = &c->nlj;
        if (poisson_mode == 1) {
            int steps[4] = {0, -1, -1, -1};
            MG_lvl_control shape[4] = {lvl_down3, lvl_up, lvl_up, lvl_up};
            double tol[4] = {0.01, 0.0005, 0.0001, 0.0001};
            c->mg.set_level_control(4, steps, shape, tol);
            ps = &c->mg;
        }
        c->rhs.reset(new rhs_probe(c->params, *ps, c->Phi, c->nd, c->mask, c->omega));
        return c;
    } catch (const char *e) {
        g_err = e;
    } catch (const std::string &e) {
        g_err = e;
    } catch (...) {
        g_err = "unknown exception";
    }
    return nullptr;
}

void kfref_destroy(kfref_ctx *c) { delete c; }

static void put_c(field_imag &f, const double *src) {
    std::memcpy(f.val, src, sizeof(double) * 2 * f.N);
}
static void get_c(const field_imag &f, double *dst) {
    std::memcpy(dst, f.val, sizeof(double) * 2 * f.N);
}

void kfref_set_state(kfref_ctx *c, const double *ux, const double *uy, const double *uz,
                     const double *ni) {
    put_c(c->FUx, ux); put_c(c->FUy, uy); put_c(c->FUz, uz); put_c(c->Fni, ni);
}

void kfref_get_state(kfref_ctx *c, double *ux, double *uy, double *uz, double *ni) {
    get_c(c->FUx, ux); get_c(c->FUy, uy); get_c(c->FUz, uz); get_c(c->Fni, ni);
}

void kfref_set_real(kfref_ctx *c, int which, const double *src) {
    field_real &f = which == 0 ? c->nd : (which == 1 ? c->mask : c->Phi);
    std::memcpy(f.val, src, sizeof(double) * f.N);
}

void kfref_get_real(kfref_ctx *c, int which, double *dst) {
    field_real &f = which == 0 ? c->nd : (which == 1 ? c->mask : c->Phi);
    std::memcpy(dst, f.val, sizeof(double) * f.N);
}

void kfref_get_sv(kfref_ctx *c, double *dst) {
    std::memcpy(dst, c->rhs->sv(), sizeof(double) * c->FUx.N);
}

/* rhs_standard::solve in place on the context's state (rhs_standard.cpp:89-566). */
int kfref_rhs(kfref_ctx *c, double t) {
    try {
        c->rhs->solve(t, c->FUx, c->FUy, c->FUz, c->Fni);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* nsteps calls of Runge_kutta_O4::solve (RKO4.cpp:50-241). */
int kfref_rk4(kfref_ctx *c, double dt, int nsteps) {
    if (g_rk4_n >= 0 && g_rk4_n != c->n) {
        g_err = "Runge_kutta_O4 keeps static buffers: one grid size per process";
        return -2;
    }
    g_rk4_n = c->n;
    try {
        Runge_kutta_O4 rk(*c->rhs, dt);
        for (int s = 0; s < nsteps; ++s) rk.solve(c->FUx, c->FUy, c->FUz, c->Fni);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* ------------------------------------------------------- standalone operators */

void kfref_fft_r2c(int n, double L, const double *in, double *out) {
    grid g = make_grid(n, L);
    field_real r(g);
    field_imag f(g);
    std::memcpy(r.val, in, sizeof(double) * r.N);
    OP_FFT op(g);
    op(r, f);
    get_c(f, out);
}

void kfref_fft_c2r(int n, double L, const double *in, double *out) {
    grid g = make_grid(n, L);
    field_real r(g);
    field_imag f(g);
    put_c(f, in);
    OP_iFFT op(g);
    op(f, r);
    std::memcpy(out, r.val, sizeof(double) * r.N);
}

void kfref_dealias(int n, double L, double *F) {
    grid g = make_grid(n, L);
    field_imag f(g);
    put_c(f, F);
    OP_dealiasing op(g, [](const double &k) { return k < (2. / 3.) ? 1. : 0.; });
    op(f);
    get_c(f, F);
}

void kfref_phi_filter(int n, double L, double *F) {
    grid g = make_grid(n, L);
    field_imag f(g);
    put_c(f, F);
    dealiasing_undesignated(f, [](double k) { return exp(-2000. * pow(k, 15.)); });
    get_c(f, F);
}

void kfref_deriv(int n, double L, int dir, const double *in, double *out) {
    grid g = make_grid(n, L);
    field_imag a(g), b(g);
    put_c(a, in);
    OP_partial_derivative op(g, dir == 0 ? e_x : (dir == 1 ? e_y : e_z));
    op(a, b);
    get_c(b, out);
}

/* solver_poisson_jacobi_nlin::solve on (phi_io, rho) (solver_poisson_jacobi_nlin.cpp:50-108). */
int kfref_nlj_solve(int n, double L, double *phi_io, const double *rho, int max_it,
                    double limit_max) {
    try {
        grid g = make_grid(n, L);
        field_real phi(g), r(g);
        std::memcpy(phi.val, phi_io, sizeof(double) * phi.N);
        std::memcpy(r.val, rho, sizeof(double) * r.N);
        fkt3d_const bs(0.), bv(0.);
        solver_poisson_jacobi_nlin nlj(bs, bv, .8);
        nlj.set_max_iterations(max_it);
        nlj.set_limit_NormMax(limit_max);
        nlj.solve(phi, r);
        std::memcpy(phi_io, phi.val, sizeof(double) * phi.N);
        return nlj.converged() ? 1 : 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* The cascadic multigrid plan of kielflow.cpp:199-217 on (phi_io, rho). */
int kfref_mg_solve(int n, double L, double *phi_io, const double *rho) {
    try {
        grid g = make_grid(n, L);
        field_real phi(g), r(g);
        std::memcpy(phi.val, phi_io, sizeof(double) * phi.N);
        std::memcpy(r.val, rho, sizeof(double) * r.N);
        fkt3d_const bs(0.), bv(0.);
        solver_poisson_jacobi_nlin nlj(bs, bv, .8);
        nlj.set_max_iterations(80);
        nlj.set_limit_NormMax(.5e-5);
        nlj.set_limit_NormSum(.5e-7);
        solver_poisson_multigrid mg(nlj);
        int steps[4] = {0, -1, -1, -1};
        MG_lvl_control shape[4] = {lvl_down3, lvl_up, lvl_up, lvl_up};
        double tol[4] = {0.01, 0.0005, 0.0001, 0.0001};
        mg.set_level_control(4, steps, shape, tol);
        mg.solve(phi, r);
        std::memcpy(phi_io, phi.val, sizeof(double) * phi.N);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* Inter-grid transfer (field_interpolation.cpp): kind 0 = OP_hto2h (n -> 2n),
 * 1 = OP_2htoh_lvl0 (n -> n/2), 2 = OP_4htoh, 3 = OP_8htoh.  n is the input size. */
int kfref_transfer(int kind, int n, double L, const double *in, double *out) {
    try {
        grid g = make_grid(n, L);
        field_real a(g), b(g);
        std::memcpy(a.val, in, sizeof(double) * a.N);
        if (kind == 0) OP_hto2h(a, b);
        else if (kind == 1) OP_2htoh_lvl0(a, b);
        else if (kind == 2) OP_4htoh(a, b);
        else OP_8htoh(a, b);
        std::memcpy(out, b.val, sizeof(double) * b.N);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* Stretched-grid (axis_CoSiSt, m != 0) forms of the entries above. */
void kfref_positions(int n, double L, double m, double *out) {
    grid g = make_grid(n, L, m);
    for (int i = -1; i <= n; ++i) out[i + 1] = g.x_axis->val_at(i);
}

void kfref_deriv_m(int n, double L, double m, int dir, const double *in, double *out) {
    grid g = make_grid(n, L, m);
    field_imag a(g), b(g);
    put_c(a, in);
    OP_partial_derivative op(g, dir == 0 ? e_x : (dir == 1 ? e_y : e_z));
    op(a, b);
    get_c(b, out);
}

int kfref_mg_solve_m(int n, double L, double m, double *phi_io, const double *rho) {
    try {
        grid g = make_grid(n, L, m);
        field_real phi(g), r(g);
        std::memcpy(phi.val, phi_io, sizeof(double) * phi.N);
        std::memcpy(r.val, rho, sizeof(double) * r.N);
        fkt3d_const bs(0.), bv(0.);
        solver_poisson_jacobi_nlin nlj(bs, bv, .8);
        nlj.set_max_iterations(80);
        nlj.set_limit_NormMax(.5e-5);
        nlj.set_limit_NormSum(.5e-7);
        solver_poisson_multigrid mg(nlj);
        int steps[4] = {0, -1, -1, -1};
        MG_lvl_control shape[4] = {lvl_down3, lvl_up, lvl_up, lvl_up};
        double tol[4] = {0.01, 0.0005, 0.0001, 0.0001};
        mg.set_level_control(4, steps, shape, tol);
        mg.solve(phi, r);
        std::memcpy(phi_io, phi.val, sizeof(double) * phi.N);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

void kfref_gauss_m(int n, double L, double m, double Q, double sigma, double *out) {
    grid g = make_grid(n, L, m);
    field_real f(g);
    fkt3d_Gauss fk(Q, sigma, sigma, sigma);
    f.fill(fk);
    std::memcpy(out, f.val, sizeof(double) * f.N);
}

/* effect_penalization::execute (effect_penalization.cpp:21-44) on an n^3
 * equidistant grid: out <- FFT((1 - H) iFFT(out) + H eta (iFFT(in) - fix)).
 * The constructor's guard (:7-12) refuses eta > 0: -1 and kfref_last_error. */
int kfref_penalize(int n, double L, double eta, double fix, const double *H, const double *in,
                   double *out) {
    try {
        grid g = make_grid(n, L);
        field_real mask(g);
        field_imag a(g), b(g);
        std::memcpy(mask.val, H, sizeof(double) * mask.N);
        put_c(a, in);
        put_c(b, out);
        effect_penalization pen(eta, mask, fix);
        pen.execute(a, b);
        get_c(b, out);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* effect_diffusion::execute (effect_diffusion.cpp:16-44) as written: out -=
 * nu * (the three second derivatives of in).  Its derivative operators are
 * function-static (built on the first call's grid), so one grid size per
 * process: -2 for another size. */
int kfref_diffuse(int n, double L, double nu, const double *in, double *out) {
    static int first_n = -1;
    if (first_n >= 0 && first_n != n) {
        g_err = "effect_diffusion keeps static derivative operators: one grid size per process";
        return -2;
    }
    first_n = n;
    try {
        static grid g = make_grid(n, L);
        field_imag a(g), b(g);
        put_c(a, in);
        put_c(b, out);
        effect_diffusion diff(nu);
        diff.execute(a, b);
        get_c(b, out);
        return 0;
    } catch (const char *e) { g_err = e; } catch (const std::string &e) { g_err = e; }
    catch (...) { g_err = "unknown exception"; }
    return -1;
}

/* fkt3d_Gauss (masks.hpp:351-366) sampled on the grid through field_real::fill. */
void kfref_gauss(int n, double L, double Q, double sigma, double *out) {
    grid g = make_grid(n, L);
    field_real f(g);
    fkt3d_Gauss fk(Q, sigma, sigma, sigma);
    f.fill(fk);
    std::memcpy(out, f.val, sizeof(double) * f.N);
}

}  // extern "C"
