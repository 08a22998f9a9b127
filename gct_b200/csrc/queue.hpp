// Work-queue backprojection on the host side: tile configurations, queue items and the on-device
// autotuner shared by the batch engine (batch.cu) and the serving loop (server.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "plan.hpp"

namespace gct {

// Tile of one block of the queue kernel: zpt voxels along z per thread, bx x by threads
// (bx * by = kQueueThreads) over x and y, vps views of coefficients staged per block barrier.
struct TileConfig {
    int zpt = 8, bx = 8, by = 32, vps = 32;
};

struct Tuned {
    TileConfig cfg;
    double ups = 0.0;  // measured voxel-view updates per second of cfg
};

bool vol3d(const gct_fdk_plan *p);
// Queue item of a prepared stack (all views; work entries pick the view range and write mode).
// Fails unless bx * by == kQueueThreads and zpt is a queue shape: every thread of a block owns
// one column of its tile, and tiles must not overlap (accumulating entries would add twice).
// A stack in the quarter-turn layout (st.quarter > 0) makes a quarter-turn item: tiles over the
// first quadrant of columns, 8 voxels deep (1 for 2D images), views counted in base views.
BpItem make_item(const gct_fdk_plan *p, const StackRef &st, float *vol, const TileConfig &c);
long long item_tiles(const BpItem &it);
// Views that work entries of the item count (base views for quarter-turn items) and its queue
// depth class.
int item_views(const gct_fdk_plan *p, const StackRef &st);
int item_class(const StackRef &st, const TileConfig &c);
// Work entries for every tile of queue item `item` over views [vb, vb + vc).
std::vector<BpWork> tile_entries(int item, long long tiles, int vb, int vc, int mode);
// The fixed shape used when autotuning is off: 8 x 32 x 8 voxels (3D and quarter-turn items) or
// 32 x 8 pixels (2D).
TileConfig default_config(const gct_fdk_plan *p, bool quarter_turn = false);
// Best tile shape for the plan's kind, storage and sizes: every candidate is timed with its depth
// class's queue kernel over all tiles and the first 64 views (writing into `vol`), once per
// process, device and shape; later calls return the cached choice.
Tuned autotune(const gct_fdk_plan *p, const StackRef &st, float *vol, int num_sms, cudaStream_t s);

}  // namespace gct
