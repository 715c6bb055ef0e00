// schedule.cpp -- work queue of the fused element loop + CSR assembly (see schedule.h).
//
//  - Tiles: tile t = elements [t*tile_elems, (t+1)*tile_elems).
//  - Conversion items: runs of at most max_nodes consecutive nodes whose CSR rows hold at most
//    stage_max - 1 values, cut at the node prefixes the host-buffer slabs finish.  Item j waits for the tiles [t0, t1]
//    that contain its nodes, and is queued `slack` tiles after t1 (so those tiles are normally
//    done when it starts) but never after the end of t1's slab.
//  - Ring: block b occupies slot b & (R - 1).  Before tile t reduces, the previous occupants of its
//    slots, blocks [minb(t) - R, maxb(t) - R), must have been converted: tile_wait[t] lists the items
//    that hold them.  Occupants further back were converted before those by the same rule (the
//    tiles that wrote the previous occupants waited for them, and the items converting the previous
//    occupants waited for those tiles).  R is a power of two for which every item a tile waits for
//    is queued before the tile (at most the power of two >= n_blocks, which never wraps): the
//    smallest such R0, enlarged up to 4 R0 so that those items are normally two grids of queue
//    positions ahead of the tile.
// Every wait of the kernel therefore targets an earlier queue position, and the earliest unfinished
// queue entry never waits for anything unfinished: the queue always drains.
#include "schedule.h"

#include <algorithm>

#include "../../include/ceos_gpu.h"

namespace ceos {

int plan_schedule(int n_nodes, int n_elem, const int* conn0, const long long* rs, const int* nup, long long n_blocks,
                  const std::vector<int>& slab_e, const std::vector<int>& slab_node_end, int tile_elems, int slack,
                  long long stage_max, int max_nodes, SchedulePlan& out) {
    const int E = n_elem, N = n_nodes;
    const int n_slabs = (int)slab_node_end.size();
    if (E < 1 || N < 1 || tile_elems < 1 || max_nodes < 1 || (int)slab_e.size() != n_slabs + 1 ||
        slab_e[n_slabs] != E) {
        out.err = "schedule: bad arguments";
        return CEOS_E_ARG;
    }
    const int T = (E + tile_elems - 1) / tile_elems;
    out.n_tiles = T;
    std::vector<long long> bb(N + 1);
    for (int n = 0; n < N; ++n) bb[n] = (long long)n + (rs[n] - 6LL * n) / 9;
    bb[N] = n_blocks;
    std::vector<int> ftile(N, T), ltile(N, -1);
    std::vector<long long> tminb(T, n_blocks), tmaxb(T, 0);
    for (int e = 0; e < E; ++e) {
        const int t = e / tile_elems;
        for (int k = 0; k < 8; ++k) {
            const int n = conn0[(size_t)8 * e + k];
            ftile[n] = std::min(ftile[n], t);
            ltile[n] = std::max(ltile[n], t);
            tminb[t] = std::min(tminb[t], bb[n]);
            tmaxb[t] = std::max(tmaxb[t], bb[n] + 1 + nup[n]);
        }
    }
    for (int n = 0; n < N; ++n)
        if (ltile[n] < 0) {
            out.err = "schedule: node " + std::to_string(n + 1) + " belongs to no element";
            return CEOS_E_MESH;
        }
    // conversion items
    std::vector<char> cut(N + 1, 0);
    for (int c = 0; c < n_slabs; ++c) cut[slab_node_end[c]] = 1;
    out.conv.clear();
    std::vector<long long> item_b0;
    {
        auto push = [&](int a0, int a1) {
            int z = T, w = -1;
            for (int n = a0; n < a1; ++n) {
                z = std::min(z, ftile[n]);
                w = std::max(w, ltile[n]);
            }
            out.conv.push_back(ConvItem{a0, a1, z, w});
            item_b0.push_back(bb[a0]);
        };
        int n0 = 0;
        long long len = 0;
        for (int n = 0; n < N; ++n) {
            const long long ln = 6 + 9LL * nup[n];
            if (ln > stage_max - 1) {
                out.err = "schedule: the CSR rows of node " + std::to_string(n + 1) + " exceed the staging buffer";
                return CEOS_E_MESH;
            }
            if (n > n0 && (cut[n] || len + ln > stage_max - 1 || n - n0 >= max_nodes)) {
                push(n0, n);
                n0 = n;
                len = 0;
            }
            len += ln;
        }
        push(n0, N);
    }
    const int J = (int)out.conv.size();
    // queue: tiles in order, item j after tile min(t1_j + slack, last tile of t1_j's slab)
    std::vector<int> tile_slab(T, 0);
    for (int c = 0; c < n_slabs; ++c)
        for (int t = slab_e[c] / tile_elems; t < (slab_e[c + 1] + tile_elems - 1) / tile_elems; ++t) tile_slab[t] = c;
    std::vector<std::vector<int>> after(T);
    for (int j = 0; j < J; ++j) {
        const int w = out.conv[j].t1;
        const int slab_last = (slab_e[tile_slab[w] + 1] + tile_elems - 1) / tile_elems - 1;
        after[std::min(w + std::max(0, slack), slab_last)].push_back(j);
    }
    out.queue.clear();
    out.queue.reserve((size_t)T + J);
    out.slab_q.assign(n_slabs + 1, 0);
    std::vector<int> pos_tile(T), pos_item(J);
    for (int t = 0; t < T; ++t) {
        if ((long long)t * tile_elems == slab_e[tile_slab[t]]) out.slab_q[tile_slab[t]] = (int)out.queue.size();
        pos_tile[t] = (int)out.queue.size();
        out.queue.push_back(t);
        for (int j : after[t]) {
            pos_item[j] = (int)out.queue.size();
            out.queue.push_back(-(j + 1));
        }
    }
    out.slab_q[n_slabs] = (int)out.queue.size();
    for (int j = 0; j < J; ++j)
        if (pos_tile[out.conv[j].t1] >= pos_item[j]) {
            out.err = "schedule: conversion item queued before its tiles";
            return CEOS_E_MESH;
        }
    // ring size: the smallest power of two R0 for which every item a tile waits for is queued before the
    // tile; then, up to 4 R0, a larger ring that keeps those items at least two grids of queue positions
    // ahead of the tile, so that a tile rarely waits for a conversion that has only just started
    long long span = 1LL << 16;
    for (int t = 0; t < T; ++t) span = std::max(span, tmaxb[t] - tminb[t]);
    long long Rmax = 1;
    while (Rmax < n_blocks) Rmax <<= 1;
    auto fill_waits = [&](long long R, long long dist) {
        bool ok = true;
        for (int t = 0; t < T && ok; ++t) {
            const long long hi = tmaxb[t] - R;
            if (R >= Rmax || hi <= 0) {
                out.tile_wait[t] = TileWait{0, 0};
                continue;
            }
            const long long lo = std::max(0LL, tminb[t] - R);
            const int x = (int)(std::upper_bound(item_b0.begin(), item_b0.end(), lo) - item_b0.begin()) - 1;
            const int y = (int)(std::upper_bound(item_b0.begin(), item_b0.end(), hi - 1) - item_b0.begin());
            out.tile_wait[t] = TileWait{x, y};
            for (int j = x; j < y && ok; ++j) ok = pos_item[j] + dist < pos_tile[t];
        }
        return ok;
    };
    out.tile_wait.assign(T, TileWait{0, 0});
    long long R0 = 1;
    while (R0 < span) R0 <<= 1;
    while (R0 < Rmax && !fill_waits(R0, 0)) R0 <<= 1;
    const long long dist = 2LL * std::max(1, slack);
    long long R = R0;
    while (R < Rmax && R < 4 * R0 && !fill_waits(R, dist)) R <<= 1;
    if (!fill_waits(R, 0)) {  // a larger ring is never needed for correctness; keep the minimal one then
        R = R0;
        fill_waits(R, 0);
    }
    out.ring_blocks = std::min(R, Rmax);
    return 0;
}

int plan_bands(int n_nodes, int n_elem, const int* conn0, const long long* rs, const int* nup, long long n_blocks,
               int band_elems, int tile_elems, long long stage_max, int max_nodes, int depth, BandPlan& out) {
    const int E = n_elem, N = n_nodes;
    if (E < 1 || N < 1 || tile_elems < 1 || band_elems < tile_elems || band_elems % tile_elems || max_nodes < 1 ||
        depth < 1) {
        out.err = "bands: bad arguments";
        return CEOS_E_ARG;
    }
    const int nb = (E + band_elems - 1) / band_elems;
    out.band_e.assign(nb + 1, 0);
    for (int c = 0; c < nb; ++c) out.band_e[c] = c * band_elems;
    out.band_e[nb] = E;
    std::vector<long long> bb(N + 1);
    for (int n = 0; n < N; ++n) bb[n] = (long long)n + (rs[n] - 6LL * n) / 9;
    bb[N] = n_blocks;
    // last band touching each node, and the largest block end each band touches
    std::vector<int> last(N, -1);
    std::vector<long long> maxb(nb, 0);
    for (int c = 0; c < nb; ++c)
        for (int e = out.band_e[c]; e < out.band_e[c + 1]; ++e)
            for (int k = 0; k < 8; ++k) {
                const int n = conn0[(size_t)8 * e + k];
                last[n] = c;
                maxb[c] = std::max(maxb[c], bb[n] + 1 + nup[n]);
            }
    for (int n = 0; n < N; ++n)
        if (last[n] < 0) {
            out.err = "bands: node " + std::to_string(n + 1) + " belongs to no element";
            return CEOS_E_MESH;
        }
    // final prefixes: a running maximum over the last bands of the nodes in row order
    out.node_end.assign(nb, 0);
    {
        int run = 0, n = 0;
        for (int c = 0; c < nb; ++c) {
            while (n < N && std::max(run, last[n]) <= c) run = std::max(run, last[n++]);
            out.node_end[c] = n;
        }
        out.node_end[nb - 1] = N;
    }
    // conversion items: runs of at most max_nodes nodes and stage_max - 1 values, cut at the prefixes
    out.conv.clear();
    out.band_conv.assign(nb + 1, 0);
    int n0 = 0;
    for (int c = 0; c < nb; ++c) {
        out.band_conv[c] = (int)out.conv.size();
        const int n_end = out.node_end[c];
        long long len = 0;
        int a = n0;
        for (int n = n0; n < n_end; ++n) {
            const long long ln = 6 + 9LL * nup[n];
            if (ln > stage_max - 1) {
                out.err = "bands: the CSR rows of node " + std::to_string(n + 1) + " exceed the staging buffer";
                return CEOS_E_MESH;
            }
            if (n > a && (len + ln > stage_max - 1 || n - a >= max_nodes)) {
                out.conv.push_back(ConvItem{a, n, c, c});
                a = n;
                len = 0;
            }
            len += ln;
        }
        if (n_end > a) out.conv.push_back(ConvItem{a, n_end, c, c});
        n0 = std::max(n0, n_end);
    }
    out.band_conv[nb] = (int)out.conv.size();
    // ring: the largest span of live blocks [bb(node_end[c - depth]), M(c + 1))
    long long Rmax = 1;
    while (Rmax < n_blocks) Rmax <<= 1;
    long long span = 1, M = 0;
    std::vector<long long> Mk(nb);
    for (int c = 0; c < nb; ++c) Mk[c] = M = std::max(M, maxb[c]);
    for (int c = 0; c < nb; ++c) {
        const long long lo = c - depth >= 0 ? bb[out.node_end[c - depth]] : 0;
        const long long hi = Mk[std::min(c + 1, nb - 1)];
        span = std::max(span, hi - lo);
    }
    out.max_span = span;
    long long R = 1;
    while (R < span + 1) R <<= 1;
    out.ring_blocks = std::min(R, Rmax);
    return 0;
}

}  // namespace ceos

#ifdef CEOS_SCHEDULE_TEST
// Flat entry for the CPU tests of the plan (built only into the test library).  Output arrays are
// sized by the caller: queue [n_elem/tile_elems + 1 + n_nodes], conv [4 n_nodes], wait [2 n_tiles],
// slab_q [n_slabs + 1]; counts [n_queue, n_conv, n_tiles].
extern "C" int ceos_test_plan_schedule(int n_nodes, int n_elem, const int* conn0, const long long* rs, const int* nup,
                                       long long n_blocks, int n_slabs, const int* slab_e, const int* slab_node_end,
                                       int tile_elems, int slack, long long stage_max, int max_nodes, int* queue,
                                       int* conv, int* wait, int* slab_q, int* counts, long long* ring_blocks) {
    ceos::SchedulePlan p;
    std::vector<int> se(slab_e, slab_e + n_slabs + 1), sn(slab_node_end, slab_node_end + n_slabs);
    const int rc = ceos::plan_schedule(n_nodes, n_elem, conn0, rs, nup, n_blocks, se, sn, tile_elems, slack, stage_max, max_nodes,
                                        p);
    if (rc) return rc;
    std::copy(p.queue.begin(), p.queue.end(), queue);
    for (size_t j = 0; j < p.conv.size(); ++j) {
        conv[4 * j] = p.conv[j].n0;
        conv[4 * j + 1] = p.conv[j].n1;
        conv[4 * j + 2] = p.conv[j].t0;
        conv[4 * j + 3] = p.conv[j].t1;
    }
    for (size_t t = 0; t < p.tile_wait.size(); ++t) {
        wait[2 * t] = p.tile_wait[t].x;
        wait[2 * t + 1] = p.tile_wait[t].y;
    }
    std::copy(p.slab_q.begin(), p.slab_q.end(), slab_q);
    counts[0] = (int)p.queue.size();
    counts[1] = (int)p.conv.size();
    counts[2] = p.n_tiles;
    *ring_blocks = p.ring_blocks;
    return 0;
}
#endif

#ifdef CEOS_SCHEDULE_TEST
// Flat entry for the CPU tests of the band plan.  Output arrays sized by the caller: band_e
// [n_elem/band_elems + 2], node_end [n_elem/band_elems + 1], conv [4 n_nodes], band_conv
// [n_elem/band_elems + 2]; counts [n_bands, n_conv]; ring [ring_blocks, max_span].
extern "C" int ceos_test_plan_bands(int n_nodes, int n_elem, const int* conn0, const long long* rs, const int* nup,
                                    long long n_blocks, int band_elems, int tile_elems, long long stage_max,
                                    int max_nodes, int depth, int* band_e, int* node_end, int* conv, int* band_conv,
                                    int* counts, long long* ring) {
    ceos::BandPlan p;
    const int rc = ceos::plan_bands(n_nodes, n_elem, conn0, rs, nup, n_blocks, band_elems, tile_elems, stage_max,
                                    max_nodes, depth, p);
    if (rc) return rc;
    const int nb = (int)p.node_end.size();
    std::copy(p.band_e.begin(), p.band_e.end(), band_e);
    std::copy(p.node_end.begin(), p.node_end.end(), node_end);
    std::copy(p.band_conv.begin(), p.band_conv.end(), band_conv);
    for (size_t j = 0; j < p.conv.size(); ++j) {
        conv[4 * j] = p.conv[j].n0;
        conv[4 * j + 1] = p.conv[j].n1;
        conv[4 * j + 2] = p.conv[j].t0;
        conv[4 * j + 3] = p.conv[j].t1;
    }
    counts[0] = nb;
    counts[1] = (int)p.conv.size();
    ring[0] = p.ring_blocks;
    ring[1] = p.max_span;
    return 0;
}
#endif
