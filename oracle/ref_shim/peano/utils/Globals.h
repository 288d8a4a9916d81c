// DIMENSIONS comes from the compiler command line (-DDIMENSIONS=2|3).
#pragma once
#ifndef DIMENSIONS
#error "compile with -DDIMENSIONS=2 or -DDIMENSIONS=3"
#endif
// number of faces of a cell, as Peano's Globals.h names it (read by limiter/generic/c/Limiter.cpph)
#define DIMENSIONS_TIMES_TWO (2 * DIMENSIONS)
