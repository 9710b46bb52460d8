// Same-named stand-in for the reference header liquid_closure.h: the whole reference API comes from
// mpcd_b200.hpp, so a caller written against the reference compiles unchanged.
#pragma once
#include "../mpcd_b200.hpp"
