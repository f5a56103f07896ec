// ref_gpu_compat.h -- TEST INFRASTRUCTURE ONLY: force-included when the
// reference's GPU sources are recompiled for sm_100a (oracle/build.py).
// The reference's shuffle reduction (GPU_Solver/CUPOT_ShuffleReduction.cu:28,
// used at POT_GHOST_SIZE 5) calls the pre-Volta __shfl_down, which sm_70 and
// later only offer as __shfl_down_sync with an explicit lane mask; every lane
// of the warp takes part there, so the full mask keeps its meaning.
#pragma once
#define __shfl_down(v, offset, width) __shfl_down_sync(0xffffffffu, (v), (offset), (width))
