"""include/kf_adapters.hpp on the CPU: kf_adapt::config_from maps the
reference's own grid (axis type_id and m) and parameters onto kf_config.
Compiled with the host C++ compiler against minimal stand-ins for the
reference's types (the members the adapter reads), no GPU call is made."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include <cstdio>
#include <stdexcept>
typedef double fftw_complex[2];
struct axis { unsigned int type_id; int N; double l0, L, m; };
struct grid { int Nx, Ny, Nz; axis *x_axis, *y_axis, *z_axis; };
struct parameters { double M = 0., tau = 0., theta = 0.; };
struct field_imag { fftw_complex *val; };
struct field_real { double *val; };
struct interface_rhs {
    virtual ~interface_rhs() {}
    virtual void solve(const double &, field_imag &, field_imag &, field_imag &, field_imag &) = 0;
};
struct interface_ode_solver {
    virtual ~interface_ode_solver() {}
    virtual void solve(field_imag &, field_imag &, field_imag &, field_imag &) = 0;
};
struct interface_poisson_solver {
    virtual ~interface_poisson_solver() {}
    virtual void solve(field_real &, field_real &) = 0;
};
#include "kf_adapters.hpp"

static int rejects(grid &g, parameters &p) {
    try {
        kf_adapt::config_from(g, p, KF_PS_CASCADIC);
    } catch (const std::runtime_error &) {
        return 1;
    }
    return 0;
}

int main() {
    const double L = 25.132741228718345, m = L * 0.7 / (2. * 3.141592653589793);
    axis eq{1, 32, -0.5 * L, L, 0.}, si{3, 32, -0.5 * L, L, m}, hy{2, 32, -0.5 * L, L, 3.};
    parameters p;
    p.M = 1.2; p.tau = 0.1; p.theta = 30.;
    grid ge{32, 32, 32, &eq, &eq, &eq}, gs{32, 32, 32, &si, &si, &si};
    kf_config c = kf_adapt::config_from(ge, p, KF_PS_CASCADIC);
    std::printf("eq %d %.17g %.17g %.17g %.17g %.17g %d\n", c.n, c.L, c.M, c.tau, c.theta, c.stretch_m, c.poisson_mode);
    c = kf_adapt::config_from(gs, p, KF_PS_FAS);
    std::printf("si %.17g %d %.17g\n", c.stretch_m, c.poisson_mode, c.mg_omega);
    grid gh{32, 32, 32, &hy, &hy, &hy}, gm{32, 32, 32, &eq, &si, &eq}, gn{32, 32, 16, &eq, &eq, &eq};
    axis off{1, 32, 0., L, 0.};
    grid go{32, 32, 32, &off, &off, &off};
    std::printf("rejects %d %d %d %d\n", rejects(gh, p), rejects(gm, p), rejects(gn, p), rejects(go, p));
    return 0;
}
'''


def test_config_from_reads_the_reference_grid(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "adapters.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "adapters"
    subprocess.run([cxx, "-std=c++11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    eq = out[0].split()
    assert eq[0] == "eq" and int(eq[1]) == 32 and float(eq[2]) == 25.132741228718345
    assert (float(eq[3]), float(eq[4]), float(eq[5]), float(eq[6])) == (1.2, 0.1, 30.0, 0.0)
    si = out[1].split()
    assert float(si[1]) == 25.132741228718345 * 0.7 / (2.0 * 3.141592653589793)
    assert float(si[3]) == 0.0  # the plain Newton step unless the caller asks for more
    assert out[2].split() == ["rejects", "1", "1", "1", "1"]  # HySt, unlike axes, non-cubic, off-centre
