// Test infrastructure only.  The reference's basis library exports its interface
// for uint32 strings alone (src/extern/basis.cpp:3); its operator library also
// exports the uint64 operators (_ui64_f64, _ui64_c64: src/extern/otf_native.cpp:5-6),
// which take a BasisManager<uint64>.  This file instantiates the reference's own
// basis interface macro (basis/declare.hpp) for uint64 with the suffix _ui64, so
// that the parity tests can drive those operators.  It is compiled against the
// reference headers where they lie (oracle/Makefile) into oracle/_ref/.
#include "basis/declare.hpp"

DECLARE_BASIS_INTERFACES(uint64, _ui64)
