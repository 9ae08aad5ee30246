// Included by the reference's BiCGStab2.h; its solve uses the vector type's
// own methods, so nothing more is needed for the parity checker.
#pragma once

#include "BelosSolverManager.hpp"
