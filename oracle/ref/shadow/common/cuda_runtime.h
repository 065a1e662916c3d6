/* Host stand-in for <cuda_runtime.h> (oracle/_ref build only). */
#pragma once
#include "kref_prelude.h"
