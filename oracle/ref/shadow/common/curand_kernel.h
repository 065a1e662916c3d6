/*
 * Host stand-in for <curand_kernel.h> (oracle/_ref build only).  A curandState replays a
 * caller-supplied sequence of uniforms in (0,1], so the reference's control/duration draws
 * (statePropagatorSpatialHash.cu:74-77, 141-144, 236-241) consume exactly the values the
 * oracle and the CUDA kernels are given.  No cuRAND algorithm is reproduced.
 */
#pragma once
typedef struct curandStateReplay {
    const float* draws;
    int pos;
} curandState;
static inline float curand_uniform(curandState* s) { return s->draws[s->pos++]; }
