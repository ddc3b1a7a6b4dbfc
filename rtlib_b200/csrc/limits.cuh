// Compile-time capacities of rtlib_b200.
#pragma once
#include <stdint.h>

namespace rtpg {
// Nodes per directional quadtree.  RTLib stores children as uint16 and stops a reset at
// 65535 nodes (OPX7UtilsPathGuiding.h:934-939); here a reset builds each tree breadth first
// in shared memory (8 bytes per node), so the cap is 16384 nodes.  With RTLib's defaults
// (split fraction 0.01, depth 20) a tree never exceeds 1 + 19 * 100 nodes.
constexpr uint32_t kDTreeNodeCap = 16384;
// Deepest quadtree level (RTLib's default maximum depth is 20, PG.h:1352).
constexpr uint32_t kMaxDTreeDepth = 31;
// Hash-grid bucket size (RTLIB_EXT_OPX7_TEST_HASH_GRID_BLOCK_SIZE, OPX7/CMakeLists.txt:104).
constexpr uint32_t kHashBlock = 32;
}  // namespace rtpg
