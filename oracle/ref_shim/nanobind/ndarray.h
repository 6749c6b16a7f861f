// Stand-in for <nanobind/ndarray.h>: everything lives in nanobind.h.
#pragma once
#include "nanobind.h"
