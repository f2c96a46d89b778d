// Stand-in for OWL's owl/common/math/vec/functors.h: the functors (dot, cross,
// normalize, sqrt, abs, clamp) are defined together with the types in
// owl/common/math/vec.h of this shim.  Test infrastructure (oracle/_ref) only.
#pragma once
#include <owl/common/math/vec.h>
