// configs.h -- the tile configurations (pixels per thread P, warps across WX, warps down WY) the
// forward kernels are instantiated for.  A warp covers 8 rows x 4P columns, so a CTA covers
// (WX*4*P) x (WY*8) output pixels with 32*WX*WY threads.  P is odd (bank-conflict-free window
// loads).  The autotuner picks among these per kernel set and device.
#pragma once

// X(index, P, WX, WY)
#define LPAICI_TILE_CONFIGS(X) \
    X(0, 9, 2, 4)              \
    X(1, 7, 2, 4)              \
    X(2, 9, 2, 2)              \
    X(3, 11, 2, 4)             \
    X(4, 5, 2, 4)

#define LPAICI_NUM_TILE_CONFIGS 5
#define LPAICI_DEFAULT_TILE_CONFIG 0
