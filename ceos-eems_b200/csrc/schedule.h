// schedule.h -- plans of the mixed-precision K assembly: the work queue of the fused element loop +
// CSR assembly, and the bands of the banded two-pass assembly.
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

// Banded two-pass assembly (mixed precision): the element pass runs in bands of band_elems elements
// (whole tiles), consecutive bands on alternating streams; after band c the rows of nodes
// [0, node_end[c]) are final and the conversion of band c (its own stream, after element bands c
// and c-1) turns rows [node_end[c-1], node_end[c]) into CSR.  Element band c starts after the
// conversion of band c - depth, so at any time at most two element bands run and every row below
// node_end[c - depth] is converted and its blocks zeroed.  The live blocks then lie in
// [bb(node_end[c - depth]), M(c + 1)) with M(k) the largest block end of bands <= k, and a ring of
// R > max_c of that span (a power of two) never gives two live blocks one slot.
struct BandPlan {
    std::vector<int> band_e;       // [n_bands + 1] element boundaries (multiples of tile_elems)
    std::vector<int> node_end;     // [n_bands] final node-row prefix after band c
    std::vector<ConvItem> conv;    // conversion items (t0 = t1 = band), cut at node_end
    std::vector<int> band_conv;    // [n_bands + 1] items of band c: [band_conv[c], band_conv[c + 1])
    long long ring_blocks = 0;     // power of two
    long long max_span = 0;        // the largest live block span
    std::string err;
};
int plan_bands(int n_nodes, int n_elem, const int* conn0, const long long* rs, const int* nup, long long n_blocks,
               int band_elems, int tile_elems, long long stage_max, int max_nodes, int depth, BandPlan& out);

}  // namespace ceos
