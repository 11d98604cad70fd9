"""kielflow_b200 -- the B200 (sm_100a) time-step hot path of kielflow.

The CUDA work lives in ``libkf.so`` (C ABI: include/kielflow_b200.h).  This
package is the host-side mirror of the reference's operator interfaces for
that path, so that a driver shaped like the reference's ``kielflow.cpp`` can
swap its objects one for one:

=============================  ==============================================
reference (C++)                here
=============================  ==============================================
``grid`` / ``axis_CoEqSt``     :class:`Grid`
``parameters``                 :class:`Parameters`
``rhs_standard``               :class:`RhsStandard`  (``interface_rhs``)
``Runge_kutta_O4``             :class:`RungeKuttaO4` (``interface_ode_solver``)
``solver_poisson_multigrid`` / :class:`PoissonSolver`
``solver_poisson_jacobi_nlin``  (``interface_poisson_solver``)
=============================  ==============================================

Fields are numpy arrays in the reference's layouts: real fields
``float64[n, n, n]`` (``field_real``), spectral fields
``complex128[n, n, n//2+1]`` (``field_imag``, FFTW r2c layout).  There is no
CPU fallback: without the CUDA library or a B200 every call raises.
"""
from ._lib import (  # noqa: F401
    KF_FP32_BULK, KF_FP64, KF_PS_CASCADIC, KF_PS_FAS, KF_PS_JACOBI_REF, KF_PS_JACOBI_RES, KF_T_ADVECTION,
    KF_T_CONTINUITY, KF_T_DIFFUSION, KF_T_DISSIPATION, KF_T_E_EXT, KF_T_E_INT, KF_T_PENALIZATION,
    KF_T_POISSON, KF_T_PRESSURE, KF_T_SHIPPED, KF_T_SVISCOSITY, KF_T_ALL, KF_ADJ_J_ONLY, KF_ADJ_STORE_PHI, Config,
    Context, GradOut, TuneOut, KfError, batch_rk4, file_info, load_library, library_path, KF_FILE_SLICE, KF_FILE_BACKUP,
    KF_OUT_SLICE, KF_OUT_BACKUP,
)
from .interfaces import Grid, Parameters, PoissonSolver, RhsStandard, RungeKuttaO4  # noqa: F401
from . import inputs  # noqa: F401
from . import kfh  # noqa: F401
