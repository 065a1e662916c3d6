/* 12D quadrotor with the values of the reference's active configuration block: h 0.1 s,
 * steps = 1 + (int)(u * 10), Zc in [0, 30], torques in [-pi, pi], |u,v,w| <= 30, regions
 * R1 8^3 x 2^3 x 2^3, R2 2^3 x 1 x 2^3, with a tree capacity of 2^22 in place of its 400000 (room for
 * the frontier it grows before its capacity branch). */
#pragma once
#define MODEL 3
#define MAX_TREE_SIZE (1 << 22)
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
#include "../../../kref_cuda_common.h"
