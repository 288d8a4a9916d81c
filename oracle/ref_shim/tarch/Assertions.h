// Assertion macros of Peano's tarch, compiled out (the reference builds its kernels the
// same way when -DAsserts is absent). Test infrastructure for oracle/_ref only.
#pragma once
#define assertion(...) ((void)0)
#define assertion1(...) ((void)0)
#define assertion2(...) ((void)0)
#define assertion3(...) ((void)0)
#define assertion4(...) ((void)0)
#define assertion5(...) ((void)0)
#define assertion6(...) ((void)0)
#define assertion7(...) ((void)0)
#define assertion8(...) ((void)0)
#define assertionMsg(...) ((void)0)
#define assertionEquals(...) ((void)0)
#define assertionEquals1(...) ((void)0)
#define assertionEquals2(...) ((void)0)
#define assertionNumericalEquals(...) ((void)0)
#define assertionNumericalEquals1(...) ((void)0)
