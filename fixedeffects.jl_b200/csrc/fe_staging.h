// fe_staging.h -- pageable host columns staged through a pinned ring owned by
// the plan (fe_staging.cu).
#pragma once

#include <stdint.h>

#include <vector>

struct fe_plan;

namespace fe {

constexpr int kRingSlots = 4;                    // pinned slots per direction
constexpr size_t kRingSlotBytes = (size_t)16 << 20;  // bytes per slot
// host-buffer solves below this many bytes copy pageable columns directly
constexpr size_t kStageMinBytes = (size_t)8 << 20;

struct PageableStager;

// Starts staging the columns cols[j] (col_bytes each) of all tiles
// (tile0: first column of each tile, then the column count) into the device
// buffer dev (column j at dev + j * col_bytes).
int stager_begin(fe_plan* pl, void* const* cols, size_t col_bytes, const std::vector<int64_t>& tile0,
                 char* dev, PageableStager** out);
// Before a tile's first launch: its columns are uploaded (the plan's stream
// waits for them).
int stager_before_tile(PageableStager* x, size_t tile);
// After a tile's last launch: its columns go back to the caller's buffers.
int stager_after_tile(PageableStager* x, size_t tile);
// Waits for every download, releases the helpers; returns the first error.
int stager_end(PageableStager* x);

}  // namespace fe
