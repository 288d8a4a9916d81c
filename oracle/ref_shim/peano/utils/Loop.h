// dfor / dLinearisedWithoutLookup stand-ins (row-major d-dimensional loop, first index fastest),
// used by the reference's GaussLegendreBasis.cpp interpolation helper.
#pragma once
#include "peano/utils/Globals.h"
#include "tarch/la/Vector.h"
namespace peano { namespace utils {
inline int dLinearisedWithoutLookup(const tarch::la::Vector<DIMENSIONS, int>& c, int n) {
  int r = 0; for (int d = DIMENSIONS - 1; d >= 0; d--) r = r * n + c[d]; return r;
}
inline bool dforNext(tarch::la::Vector<DIMENSIONS, int>& c, int n) {
  for (int d = 0; d < DIMENSIONS; d++) { c[d]++; if (c[d] < n) return true; c[d] = 0; }
  return false;
}
}}
#define dfor(counter, max) \
  for (tarch::la::Vector<DIMENSIONS, int> counter(0), *counter##_once = &counter; counter##_once; \
       counter##_once = peano::utils::dforNext(counter, (max)) ? &counter : nullptr)
