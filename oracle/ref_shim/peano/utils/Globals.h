// DIMENSIONS comes from the compiler command line (-DDIMENSIONS=2|3).
#pragma once
#ifndef DIMENSIONS
#error "compile with -DDIMENSIONS=2 or -DDIMENSIONS=3"
#endif
