// Host stand-in for <curand_kernel.h>, used ONLY when the reference's
// device-side integrator headers are compiled for the host (oracle/_ref).
//
// The reference draws every random number through curand_init/curand_uniform
// (PathTracerLib/src/Sampling/RandCore.h:7-23).  On the host there is no
// cuRAND device API, so this stand-in replays a "tape": a row of uniforms that
// the GPU produced by calling the real cuRAND for the same seed, or that a test
// produced with any other generator.  curand_init() selects the row that the
// harness registered for the calling thread; curand_uniform() pops from it.
// Nothing here restates cuRAND's own algorithm.
#pragma once

#include <cstdint>

struct RefTapeState {
    const float* row;     // uniforms for this (pixel, sample)
    int cursor;           // next value to return
    int length;           // values available in the row
    unsigned int seed;    // seed handed to curand_init (checked by the harness)
};

typedef RefTapeState curandState;
typedef RefTapeState curandStateXORWOW;

void curand_init(unsigned long long seed, unsigned long long subsequence,
                 unsigned long long offset, curandState* state);
float curand_uniform(curandState* state);
