// configs.h -- the tile configurations (warps across WX, warps down WY) the kernels are
// instantiated for.  A warp covers 16 x 16 output pixels (8 per thread), so a CTA covers
// (16*WX) x (16*WY) pixels with 32*WX*WY threads.  The autotuner picks among these per kernel set
// and device; configurations whose shared memory does not fit a kernel set are skipped.
#pragma once

// X(index, WX, WY)
#define LPAICI_TILE_CONFIGS(X) \
    X(0, 4, 4)                 \
    X(1, 8, 2)                 \
    X(2, 2, 8)                 \
    X(3, 4, 2)                 \
    X(4, 2, 4)

#define LPAICI_NUM_TILE_CONFIGS 5
#define LPAICI_DEFAULT_TILE_CONFIG 0
