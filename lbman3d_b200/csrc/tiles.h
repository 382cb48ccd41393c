// tiles.h -- the compiled z-marching tile shapes (cells per x-y plane of one
// block) of the Q+force, fused and ensemble kernels.  A shape whose shared
// memory does not fit one block for a precision is skipped for it.
#pragma once

#define LBMAN_TILES(X) X(30, 6) X(32, 6) X(14, 14) X(30, 14) X(62, 6) X(32, 8) X(32, 14) X(64, 6)
// tiles of the two-points-per-thread FP32 Q+force kernel (qpair.cuh)
#define LBMAN_PAIR_TILES(X) X(30, 6) X(30, 10) X(30, 14)

namespace lbman {
#define LBMAN_TILE_PAIR(x, y) {x, y},
constexpr int kTileList[][2] = {LBMAN_TILES(LBMAN_TILE_PAIR)};
#undef LBMAN_TILE_PAIR
constexpr int kNumTiles = sizeof(kTileList) / sizeof(kTileList[0]);
#define LBMAN_TILE_PAIR(x, y) {x, y},
constexpr int kPairTileList[][2] = {LBMAN_PAIR_TILES(LBMAN_TILE_PAIR)};
#undef LBMAN_TILE_PAIR
}  // namespace lbman
