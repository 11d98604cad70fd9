/*
 * kf_adapters.hpp -- drop-in adapters: the reference's interfaces on the C ABI.
 *
 * Include after the reference's own headers (interface_rhs.hpp,
 * interface_ODE_solver.hpp, interface_poisson_solver.hpp, field.hpp,
 * parameters.hpp) and link libkf.so.  Each class implements one interface of
 * the reference, with its argument meaning and in-place behaviour, and throws
 * std::runtime_error where the reference throws:
 *
 *   kf_gpu_rhs     : interface_rhs           (rhs_standard, rhs_standard.cpp:7-566)
 *   kf_gpu_rk4     : interface_ode_solver    (Runge_kutta_O4, RKO4.cpp:41-241)
 *   kf_gpu_poisson : interface_poisson_solver (solver_poisson_multigrid /
 *                    solver_poisson_jacobi_nlin, kielflow.cpp:197-217)
 *
 * field_imag::val is fftw_complex[] = interleaved doubles, field_real::val is
 * double[], both in the layouts the C ABI expects (field_base.hpp:23-24).
 */
#ifndef KF_ADAPTERS_HPP_
#define KF_ADAPTERS_HPP_

#include <stdexcept>
#include <string>

#include "kielflow_b200.h"

namespace kf_adapt {

inline void check(kf_ctx *c, int rc) {
    if (rc) throw std::runtime_error(std::string("kielflow_b200: ") + kf_last_error(c));
}

/* kf_config for a cubic reference grid and parameters (the shipped physics by
 * default: rhs_standard.hpp:22-30 term set, SV amplitude 0.5, theta from params).
 * The three axes must be alike: axis_CoEqSt (type_id 1) or axis_CoSiSt
 * (type_id 3, its m becomes stretch_m); axis_CoHySt has no dS and cannot take
 * derivatives in the reference either (axis_base.cpp:17-23). */
template <typename Grid, typename Params>
kf_config config_from(const Grid &g, const Params &p, int poisson_mode, int terms = KF_T_SHIPPED) {
    if (g.Nx != g.Ny || g.Nx != g.Nz) throw std::runtime_error("kielflow_b200: cubic grids only");
    const auto *ax = g.x_axis;
    for (const auto *a : {g.y_axis, g.z_axis})
        if (a->type_id != ax->type_id || a->L != ax->L || a->l0 != ax->l0 || (ax->type_id == 3 && a->m != ax->m))
            throw std::runtime_error("kielflow_b200: the three axes must be alike");
    if (ax->type_id != 1 && ax->type_id != 3)
        throw std::runtime_error("kielflow_b200: axis_CoEqSt or axis_CoSiSt axes only");
    if (ax->l0 != -0.5 * ax->L) throw std::runtime_error("kielflow_b200: the box must be centred (l0 = -L/2)");
    kf_config c = {};
    c.n = g.Nx;
    c.L = ax->L;
    c.stretch_m = ax->type_id == 3 ? ax->m : 0.;
    c.M = p.M;
    c.tau = p.tau;
    c.theta = p.theta;
    c.sv_eps = 0.5;
    c.terms = terms;
    c.poisson_mode = poisson_mode;
    c.nlj_max_it = 80;       /* kielflow.cpp:201 */
    c.nlj_limit = .5e-5;     /* kielflow.cpp:202 */
    c.res_tol = 1e-10;
    c.mg_levels = 4;
    c.mg_pre = 2;
    c.mg_post = 2;
    c.coarse_tol = 1e-13;
    c.max_cycles = 100;
    c.phi_extrap = 0;
    c.precision = KF_FP64;
    return c;
}

}  // namespace kf_adapt

/* interface_rhs: solve(t, FUx, FUy, FUz, Fni) replaces the fields by their time
 * derivative (rhs_standard.cpp:89-566).  The potential persists on the device
 * between calls as the warm start, as rhs_standard keeps a reference to Phi. */
class kf_gpu_rhs : public interface_rhs {
public:
    template <typename Grid>
    kf_gpu_rhs(parameters &P, field_real &nd, field_real &mask, const Grid &g,
               int poisson_mode = KF_PS_CASCADIC, int terms = KF_T_SHIPPED) {
        kf_config c = kf_adapt::config_from(g, P, poisson_mode, terms);
        kf_adapt::check(nullptr, kf_ctx_create(&c, &ctx_));
        kf_adapt::check(ctx_, kf_set_sources(ctx_, nd.val, mask.val));
    }
    ~kf_gpu_rhs() { kf_ctx_destroy(ctx_); }
    void solve(const double &t, field_imag &FUx, field_imag &FUy, field_imag &FUz, field_imag &Fni) {
        kf_adapt::check(ctx_, kf_set_state(ctx_, &FUx.val[0][0], &FUy.val[0][0], &FUz.val[0][0], &Fni.val[0][0]));
        kf_adapt::check(ctx_, kf_rhs_eval(ctx_, t));
        kf_adapt::check(ctx_, kf_get_state(ctx_, &FUx.val[0][0], &FUy.val[0][0], &FUz.val[0][0], &Fni.val[0][0]));
    }
    void get_phi(field_real &Phi) { kf_adapt::check(ctx_, kf_get_phi(ctx_, Phi.val)); }
    kf_ctx *context() { return ctx_; }

private:
    kf_ctx *ctx_ = nullptr;
};

/* interface_ode_solver: solve(FUx, FUy, FUz, Fni) advances the fields by one
 * fixed dt (RKO4.cpp:50-241) on the right-hand side of a kf_gpu_rhs. */
class kf_gpu_rk4 : public interface_ode_solver {
public:
    kf_gpu_rk4(kf_gpu_rhs &rhs, double dt = 0.01) : ctx_(rhs.context()), dt_(dt) {}
    void solve(field_imag &FUx, field_imag &FUy, field_imag &FUz, field_imag &Fni) {
        kf_adapt::check(ctx_, kf_step_host(ctx_, 1, dt_, &FUx.val[0][0], &FUy.val[0][0], &FUz.val[0][0],
                                           &Fni.val[0][0]));
    }

private:
    kf_ctx *ctx_;
    double dt_;
};

/* interface_poisson_solver: solve(Phi_IO, rho), Phi_IO the initial guess and
 * the result (interface_poisson_solver.hpp:18). */
class kf_gpu_poisson : public interface_poisson_solver {
public:
    template <typename Grid>
    explicit kf_gpu_poisson(const Grid &g, int mode = KF_PS_FAS) {
        parameters p;
        kf_config c = kf_adapt::config_from(g, p, mode);
        c.theta = 1.;
        kf_adapt::check(nullptr, kf_ctx_create(&c, &ctx_));
    }
    ~kf_gpu_poisson() { kf_ctx_destroy(ctx_); }
    void solve(field_real &Phi_IO, field_real &rho) {
        kf_adapt::check(ctx_, kf_poisson_solve(ctx_, Phi_IO.val, rho.val));
    }

private:
    kf_ctx *ctx_ = nullptr;
};

#endif
