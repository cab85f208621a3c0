// Oracle test infrastructure, not product code.
// source/TabulatedLteH.hpp includes YAKL's NetCDF header for its table
// loader; the stand-in reader lives in the shim's YAKL.h.
#pragma once

#include "YAKL.h"
