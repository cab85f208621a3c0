// Oracle test infrastructure, not product code.
// Stand-in for DexRT's CascadeState (see State.hpp in this directory).
#pragma once
struct CascadeState {};
