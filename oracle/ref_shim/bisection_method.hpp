/* bisection_method.hpp -- placeholder (oracle build only).  Included by
 * solver_poisson_jacobi_nlin.hpp:15 but absent from the reference; the solver
 * uses nothing from it (its bisection calls are commented out, :174,209-210). */
#ifndef BISECTION_METHOD_HPP_
#define BISECTION_METHOD_HPP_
#endif
