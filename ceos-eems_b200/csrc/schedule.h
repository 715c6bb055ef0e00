// schedule.h -- work queue of the fused element loop + CSR assembly (mixed precision).
//
// Host-only planning, kept free of CUDA so that its properties (every wait targets an earlier
// queue position; the ring slots of a tile are released before the tile reduces into them) can be
// checked on the CPU.  The kernel side is element_assemble_kernel in element_kernel.cuh.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace ceos {

struct ConvItem {  // same layout as the kernel's int4
    int n0, n1;    // CSR rows of nodes [n0, n1)
    int t0, t1;    // tiles [t0, t1] contain those nodes
};
struct TileWait {  // same layout as the kernel's int2
    int x, y;      // conversion items [x, y) that last used the tile's ring slots
};

struct SchedulePlan {
    std::vector<int> queue;        // >= 0 tile, < 0 conversion item -(j+1)
    std::vector<int> slab_q;       // [n_slabs + 1] queue position where slab c starts
    std::vector<ConvItem> conv;
    std::vector<TileWait> tile_wait;
    int n_tiles = 0;
    long long ring_blocks = 0;     // power of two
    std::string err;
};

// Tiles are tile_elems consecutive elements.  Node n owns the node-pair blocks
// [bb(n), bb(n) + 1 + nup[n]) with bb(n) = n + (rs[n] - 6n)/9 (rs[n]: CSR position of row 3n).
// slab_e [n_slabs + 1] are element boundaries (multiples of tile_elems, last = n_elem); after slab
// c the rows of nodes [0, slab_node_end[c]) are final.  An item holds at most stage_max - 1 K values
// and at most max_nodes nodes.  Returns 0 or a negative code with out.err set.
int plan_schedule(int n_nodes, int n_elem, const int* conn0, const long long* rs, const int* nup, long long n_blocks,
                  const std::vector<int>& slab_e, const std::vector<int>& slab_node_end, int tile_elems, int slack,
                  long long stage_max, int max_nodes, SchedulePlan& out);

}  // namespace ceos
