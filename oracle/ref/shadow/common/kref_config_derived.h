/*
 * Derived macros and constants of the models that a configuration does not select
 * (oracle/_ref build only).  The names are the ones the reference's sources read
 * (include/config/config.h); the per-configuration values come from the benchmark
 * configurations in the sibling di/, dubins/, quad/ directories.
 */
#pragma once
#define SAMPLE_DIM (STATE_DIM + CONTROL_DIM + 1)
#define W_R1_SIZE ((W_MAX - W_MIN) / W_R1_LENGTH)
#define C_R1_SIZE ((C_MAX - C_MIN) / C_R1_LENGTH)
#define V_R1_SIZE ((V_MAX - V_MIN) / V_R1_LENGTH)
#define W_R1_VOL (W_R1_SIZE * W_R1_SIZE * W_R1_SIZE)
#define KREF_IPOW(b, e) ((e) == 0 ? 1 : (e) == 1 ? (b) : (e) == 2 ? (b) * (b) : (b) * (b) * (b))
#define NUM_R1_REGIONS \
    (W_R1_LENGTH * W_R1_LENGTH * W_R1_LENGTH * KREF_IPOW(C_R1_LENGTH, C_DIM) * KREF_IPOW(V_R1_LENGTH, V_DIM))
#define NUM_R2_PER_R1 \
    (W_R2_LENGTH * W_R2_LENGTH * W_R2_LENGTH * KREF_IPOW(C_R2_LENGTH, C_DIM) * KREF_IPOW(V_R2_LENGTH, V_DIM))
#define NUM_R2_REGIONS (NUM_R1_REGIONS * NUM_R2_PER_R1)
#define NUM_R1_REGIONS_KERNEL1 1024
#define NUM_PARTIAL_SUMS 1024
#define MAX_ITER_REKINO 20000
#define VERBOSE 0

/* unicycle (model 0) is compiled but never selected */
#define UNI_MIN_STEERING -M_PI / 2
#define UNI_MAX_STEERING M_PI / 2
#define UNI_MIN_DT 0.1f
#define UNI_MAX_DT 2.0f
#define UNI_LENGTH 1.0f

#ifndef DUBINS_AIRPLANE_MIN_PR
#define DUBINS_AIRPLANE_MIN_PR (-M_PI / 4)
#define DUBINS_AIRPLANE_MAX_PR (M_PI / 4)
#define DUBINS_AIRPLANE_MIN_YR (-M_PI / 4)
#define DUBINS_AIRPLANE_MAX_YR (M_PI / 4)
#endif
#define DUBINS_AIRPLANE_MIN_YAW -M_PI
#define DUBINS_AIRPLANE_MAX_YAW M_PI
#define DUBINS_AIRPLANE_MIN_PITCH -M_PI / 3
#define DUBINS_AIRPLANE_MAX_PITCH M_PI / 3

#ifndef QUAD_MIN_Zc
#define QUAD_MIN_Zc 0.0f
#define QUAD_MAX_Zc 30.0f
#define QUAD_MIN_Lc -M_PI
#define QUAD_MAX_Lc M_PI
#define QUAD_MIN_Mc -M_PI
#define QUAD_MAX_Mc M_PI
#define QUAD_MIN_Nc -M_PI
#define QUAD_MAX_Nc M_PI
#endif
#define QUAD_MIN_YAW -M_PI
#define QUAD_MAX_YAW M_PI
#define QUAD_MIN_PITCH -M_PI
#define QUAD_MAX_PITCH M_PI
#define QUAD_MIN_ROLL -M_PI
#define QUAD_MAX_ROLL M_PI
#define QUAD_MIN_ANGLE_RATE -30.0f
#define QUAD_MAX_ANGLE_RATE 30.0f
#define NU 10e-3f
#define MU 2e-6f
#define KM 0.03f
#define IX 1.0f
#define IY 1.0f
#define IZ 2.0f
#define GRAVITY -9.81f
#define MASS 1.0f
#define MASS_INV 1.0f / MASS
