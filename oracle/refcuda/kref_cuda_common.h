/*
 * Shared part of the configuration headers of the reference's CUDA build (TEST INFRASTRUCTURE:
 * the reference planner compiled unmodified from its own sources for sm_100a, timed beside this
 * library; nothing in the product links it).
 *
 * The reference reads its configuration from include/config/config.h; each directory under cfg/
 * holds one config/config.h that is found ahead of it on the include path.  Names are the
 * reference's macros.  Two choices differ from a plain configuration:
 *  - MAX_ITER expands to a call of kref_iteration_bound(), a host function of the harness
 *    (ref_plan.cu).  The reference evaluates MAX_ITER in its constructor (the sizes of the path
 *    buffers, Planner.cu:9, 22) and before every iteration of its plan loop
 *    (`while(h_itr_ < MAX_ITER)`, KPAX.cu:94).  At the loop test the harness reads the
 *    frontier's repeat total and ends the plan before an iteration whose full expansion would not
 *    fit in the tree (the branch of KPAX.cu:323-341, whose writes can pass the end of the tree
 *    buffers), and after its iteration cap.
 *  - VERBOSE is 0 (from kref_config_derived.h).
 */
#pragma once
#include "../ref/shadow/common/kref_config_derived.h"

int kref_iteration_bound(void);
#define MAX_ITER kref_iteration_bound()
