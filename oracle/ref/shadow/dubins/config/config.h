/* Dubins airplane benchmark configuration (oracle/_ref build only): h 0.05 s, up to 20 steps,
 * v in [0.5,2], a in [-1,1], yaw/pitch rates in [-0.5,0.5], pitch within +-pi/3,
 * regions as the reference's Dubins block (R1 8^3 x 8^2, R2 2^3 x 3^2). */
#pragma once
#include "kref_prelude.h"
#define MODEL 2
#define MAX_TREE_SIZE (1 << 20)
#define MAX_ITER 300
#define STEP_SIZE 0.05f
#define MAX_PROPAGATION_DURATION 20
#define GOAL_THRESH 5.0f
#define STATE_DIM 6
#define CONTROL_DIM 3
#define W_DIM 3
#define C_DIM 2
#define V_DIM 1
#define W_MIN 0.0f
#define W_MAX 100.0f
#define W_SIZE 100.0f
#define C_MIN -M_PI
#define C_MAX M_PI
#define V_MIN 0.5f
#define V_MAX 2.0f
#define A_MIN -1.0f
#define A_MAX 1.0f
#define DUBINS_AIRPLANE_MIN_PR -0.5f
#define DUBINS_AIRPLANE_MAX_PR 0.5f
#define DUBINS_AIRPLANE_MIN_YR -0.5f
#define DUBINS_AIRPLANE_MAX_YR 0.5f
#define W_R1_LENGTH 8
#define C_R1_LENGTH 8
#define V_R1_LENGTH 1
#define W_R2_LENGTH 2
#define C_R2_LENGTH 3
#define V_R2_LENGTH 1
#define EPSILON 1e-2f
#include "kref_config_derived.h"
