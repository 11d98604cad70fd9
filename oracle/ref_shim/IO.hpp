/*
 * IO.hpp -- stand-in for the reference's include/IO.hpp (oracle build only).
 *
 * The reference header pulls in echelon/HDF5 (IO.hpp:40), which are absent.
 * The hot-path sources only need its transitive includes and the declaration
 * of save_2d (RKO4.cpp:36, reached only under _MONITOR_EVOLUTION), so this
 * stand-in provides those and a no-op save_2d.  File I/O is off the hot path.
 */
#ifndef IO_HPP
#define IO_HPP

#include <cmath>
#include <string>
#include <sstream>
#include <fstream>
#include <iostream>
#include <vector>
#include <ctime>
#include <iomanip>
#include <omp.h>
#include "fftw3.h"
#include "parameters.hpp"
#include "field.hpp"
#include "grid.hpp"
#include "axis.hpp"
#include "axis_EqSt.hpp"
#include "operations.hpp"
#include "subdim.hpp"
#include "o_math.hpp"

inline void save_2d(const field_real &, subdim &, const std::string & = "") {}

#endif
