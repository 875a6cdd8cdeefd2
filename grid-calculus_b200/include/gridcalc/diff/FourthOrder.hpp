// Drop-in for the reference header of the same path: everything lives in
// gridcalc/b200.hpp (see there for what each function maps to).
#pragma once
#include <gridcalc/b200.hpp>
