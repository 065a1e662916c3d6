/* Host stand-in for the reference's helper/helper.cuh (oracle/_ref build only): the
 * propagation sources include it but use none of its thrust/CSV helpers. */
#pragma once
#include "../kref_prelude.h"
#include "config/config.h"
inline int iDivUp(int a, int b) { return (a + b - 1) / b; }
