// Forced-include prelude for compiling the reference's host+device headers
// with g++ (oracle/_ref only).  SpectralCore.h calls isfinite() unqualified.
#pragma once
#include <cmath>
using std::isfinite;
