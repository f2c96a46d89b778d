// Stand-in for OWL's owl/owl.h: the reference kernel headers include it only
// for the vector types, which live in owl/common/math/vec.h here.
// Test infrastructure (oracle/_ref build) only.
#pragma once
#include <owl/common/math/vec.h>
