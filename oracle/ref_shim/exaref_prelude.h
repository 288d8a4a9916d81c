// Force-included before the reference headers (g++ -include). The reference kernels call
// std::abs<double> as a function object (3d/riemannSolverNonlinear.cpph:66) and use
// std::numeric_limits without including <limits> (3d/stableTimeStepSize.cpph:31); g++ 13 needs
// both declared. Test infrastructure for oracle/_ref only.
#pragma once
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>
namespace std {
template <class T>
T abs(T x) { return std::fabs(x); }
}
