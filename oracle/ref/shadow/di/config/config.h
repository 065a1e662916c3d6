/* 6D double integrator benchmark configuration (oracle/_ref build only):
 * h 0.1 s, steps U{1..10}, |v| <= 1, a in [-1,1]^3, workspace [0,100]^3, R1 8^3, R2 2^3. */
#pragma once
#include "kref_prelude.h"
#define MODEL 1
#define MAX_TREE_SIZE (1 << 20)
#define MAX_ITER 300
#define STEP_SIZE 0.1f
#define MAX_PROPAGATION_DURATION 10
#define GOAL_THRESH 5.0f
#define STATE_DIM 6
#define CONTROL_DIM 3
#define W_DIM 3
#define C_DIM 0
#define V_DIM 3
#define W_MIN 0.0f
#define W_MAX 100.0f
#define W_SIZE 100.0f
#define C_MIN -M_PI
#define C_MAX M_PI
#define V_MIN -1.0f
#define V_MAX 1.0f
#define A_MIN -1.0f
#define A_MAX 1.0f
#define W_R1_LENGTH 8
#define C_R1_LENGTH 1
#define V_R1_LENGTH 1
#define W_R2_LENGTH 2
#define C_R2_LENGTH 1
#define V_R2_LENGTH 1
#define EPSILON 1e-2f
#include "kref_config_derived.h"
