// ss_internal.h -- library-internal entry points shared between translation
// units (not part of the C ABI).
#pragma once

#include <cstddef>
#include <cstdint>

namespace ss {

// Workspace bytes the route needs for `tiles` tiles of edge `tile`; false if
// the size does not fit the workspace's index ranges.
bool workspace_bytes_for_tiles(int64_t tiles, int tile, size_t* bytes);

}  // namespace ss
