// Sizes and launch shapes shared by the host orchestration and the kernels.

#pragma once

namespace b200fe {

constexpr int kMaxDims = 8;
constexpr int kMaxLarge = 2;
constexpr int kMaxSmall = 4;
constexpr int kSmallLevels = 64;   // a non-primary dim with <= 64 levels is "small"
constexpr int kMaxSmallRows = 128; // total levels over all small dims
constexpr int kPassThreads = 128;  // long-segment pass CTA size (4 warps)
constexpr int kTileThreads = 256;  // tile pass CTA size (8 warps)
constexpr int kRowThreads = 256;   // alpha-space row kernels
constexpr int kTileObs = 448;      // observations staged per tile
constexpr int kTileStride = 320;   // tiles start within windows of this many obs
constexpr int kLongSeg = kTileObs - kTileStride;  // longer segments take the long path

}  // namespace b200fe
