#pragma once
#include "tarch/la/Vector.h"
