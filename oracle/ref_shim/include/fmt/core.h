// Oracle test infrastructure, not product code.
// Empty stand-in for fmt's header: the hydro hot-path sources include it
// (source/Boundaries.hpp) but call nothing from it.
#pragma once
