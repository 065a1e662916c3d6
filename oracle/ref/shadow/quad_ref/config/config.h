/* 12D quadrotor with the values of the reference's active configuration block (oracle/_ref build
 * only): h 0.1 s, up to 10 steps, Zc in [0, 30], torques in [-pi, pi] (from kref_config_derived.h),
 * |u,v,w| <= 30, regions R1 8^3 x 2^3 x 2^3, R2 2^3 x 1 x 2^3, capacity 400000. */
#pragma once
#include "kref_prelude.h"
#define MODEL 3
#define MAX_TREE_SIZE 400000
#define MAX_ITER 300
#define STEP_SIZE 0.1f
#define MAX_PROPAGATION_DURATION 10
#define GOAL_THRESH 5.0f
#define STATE_DIM 12
#define CONTROL_DIM 4
#define W_DIM 3
#define C_DIM 3
#define V_DIM 3
#define W_MIN 0.0f
#define W_MAX 100.0f
#define W_SIZE 100.0f
#define C_MIN -M_PI
#define C_MAX M_PI
#define V_MIN -30.0f
#define V_MAX 30.0f
#define A_MIN -30.0f
#define A_MAX 30.0f
#define W_R1_LENGTH 8
#define C_R1_LENGTH 2
#define V_R1_LENGTH 2
#define W_R2_LENGTH 2
#define C_R2_LENGTH 1
#define V_R2_LENGTH 2
#define EPSILON 1e-2f
#include "kref_config_derived.h"
