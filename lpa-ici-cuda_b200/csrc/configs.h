// configs.h -- the tile configurations the kernels are instantiated for: warps across WX, warps
// down WY, column pairs per thread Q (4 or 8).  A warp covers 16 rows x 4Q columns (2Q pixels per
// thread), so a CTA covers (4Q*WX) x (16*WY) pixels with 32*WX*WY threads.  The autotuner picks among
// these per kernel set and device; configurations whose shared memory does not fit a kernel set are
// skipped.  The adjoint's selection pass runs the configuration the forward uses.
#pragma once

// X(index, WX, WY, Q)
#define LPAICI_TILE_CONFIGS(X) \
    X(0, 4, 4, 4)              \
    X(1, 8, 2, 4)              \
    X(2, 2, 8, 4)              \
    X(3, 2, 4, 8)              \
    X(4, 4, 2, 8)              \
    X(5, 1, 8, 8)              \
    X(6, 4, 2, 4)              \
    X(7, 5, 4, 4)              \
    X(8, 4, 5, 4)              \
    X(9, 6, 4, 4)              \
    X(10, 4, 6, 4)

#define LPAICI_NUM_TILE_CONFIGS 11
#define LPAICI_DEFAULT_TILE_CONFIG 0

// Without autotuning, the first of these whose shared memory fits is used: the configurations in
// order of their B200 time on the 4096^2 benchmark image (16x7 symmetric kernels), fastest first.
#define LPAICI_TILE_PREFERENCE {10, 9, 8, 7, 0, 1, 2, 6, 3, 4, 5}
