/*
 * Force-included prelude for compiling the reference's device functions on the host
 * (oracle/_ref, test infrastructure only).  CUDA qualifiers become plain C++; int min/max
 * stand in for the CUDA device overloads used by worldToGrid (spatialHash.cuh:236-246).
 */
#pragma once
#include <math.h>
#include <cmath>
#include <stdio.h>
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
typedef unsigned int uint;
