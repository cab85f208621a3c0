// Oracle test infrastructure, not product code.
// Stand-in for the DexRT radiative-transfer state type that
// source/DexInterface.hpp names as a member of the Simulation aggregate.
// The radiative-transfer coupling is outside the hydro hot path, so an empty
// type is enough for the hot-path sources to compile.
#pragma once
namespace Dex {
using fp_t = double;
}
struct State {};
