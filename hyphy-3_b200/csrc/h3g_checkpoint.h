// h3g_checkpoint.h — subtree checkpointing plan (host only).
//
// The reference keeps the inside, outside and message partials of every node for
// all patterns (likelihood.hpp:314-340).  When that does not fit the device, the
// tree is cut into blocks: a block is a checkpoint node r with every descendant
// reachable from r without passing another checkpoint.  Checkpoint nodes (the
// root always among them) own persistent partial slots [0, ncp); every other node
// gets a scratch slot numbered inside its block, so all blocks share one scratch
// region of max-block size.  Evaluation order:
//   inside:  blocks in post-order (a block after the blocks below it), each over its
//            internal nodes by height; a checkpoint's message and exponents stay in
//            its persistent slot for the block above;
//   outside: blocks in reverse post-order; each first recomputes its inside partials
//            below r (r's own are persistent; the root's block is still in scratch
//            from the inside pass), then walks its internal nodes by depth writing
//            the outside vectors of their children (a child that roots another block
//            gets them in its persistent slot), then accumulates the gradient
//            operands of its branches.
// Block sizes stay within 1 + (children per node) x (target - 1) nodes.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace h3g {

struct CkBlock {
    int root = -1;
    std::vector<int> in_nodes;      // internal nodes by increasing height, the block root last
    std::vector<int> in_lv;         // level offsets into in_nodes (one level per height)
    std::vector<int> out_kids;      // children of the block's internal nodes by increasing parent depth
    std::vector<int> out_lv;        // level offsets into out_kids
    std::vector<int> acc;           // branches accumulated with this block (its nodes but the tree root)
};

struct CkPlan {
    int target = 0;
    int ncp = 0, scratch_int = 0, scratch_all = 0;
    std::vector<uint8_t> is_ckpt;   // [n]
    std::vector<int> block_of;      // [n] block computing the node
    std::vector<int> iidx, vidx;    // [n] partial slot (internal nodes, else -1) and gradient-operand slot
    std::vector<CkBlock> blocks;    // post-order, the root's block last
};

// kids[u] in increasing id order; order = BFS order from the root (parents before children).
inline CkPlan plan_checkpoints(int n, int root, const std::vector<std::vector<int>>& kids, const uint8_t* is_leaf,
                               const std::vector<int>& order, const std::vector<int>& depth,
                               const std::vector<int>& height, int target) {
    CkPlan pl;
    pl.target = std::max(target, 2);
    pl.is_ckpt.assign(n, 0);
    pl.block_of.assign(n, -1);
    pl.iidx.assign(n, -1);
    pl.vidx.assign(n, -1);
    std::vector<int> open(n, 0);
    for (int q = n - 1; q >= 0; --q) {
        const int u = order[q];
        if (is_leaf[u]) continue;
        int s = 1;
        for (int c : kids[u]) s += is_leaf[c] ? 1 : (pl.is_ckpt[c] ? 0 : open[c]);
        open[u] = s;
        if (u != root && s >= pl.target) pl.is_ckpt[u] = 1;
    }
    pl.is_ckpt[root] = 1;
    // blocks in post-order: checkpoint nodes in reverse BFS order (a block root is deeper than
    // the root of the block above it)
    for (int q = n - 1; q >= 0; --q)
        if (pl.is_ckpt[order[q]]) {
            pl.blocks.emplace_back();
            pl.blocks.back().root = order[q];
        }
    for (size_t bi = 0; bi < pl.blocks.size(); ++bi) pl.iidx[pl.blocks[bi].root] = pl.vidx[pl.blocks[bi].root] = int(bi);
    pl.ncp = int(pl.blocks.size());
    std::vector<int> members, stack;
    for (size_t bi = 0; bi < pl.blocks.size(); ++bi) {
        CkBlock& B = pl.blocks[bi];
        members.clear();
        stack.assign(1, B.root);
        while (!stack.empty()) {
            const int u = stack.back();
            stack.pop_back();
            members.push_back(u);
            pl.block_of[u] = int(bi);
            if (is_leaf[u]) continue;
            for (int c : kids[u])
                if (is_leaf[c] || !pl.is_ckpt[c]) stack.push_back(c);
        }
        std::sort(members.begin(), members.end());
        int li = 0, lv = 0;
        for (int u : members) {
            if (u == B.root) continue;
            if (!is_leaf[u]) pl.iidx[u] = pl.ncp + li++;
            pl.vidx[u] = pl.ncp + lv++;
        }
        pl.scratch_int = std::max(pl.scratch_int, li);
        pl.scratch_all = std::max(pl.scratch_all, lv);
        // inside levels by height, outside levels by the parent's depth
        std::vector<int> internal;
        for (int u : members)
            if (!is_leaf[u]) internal.push_back(u);
        std::stable_sort(internal.begin(), internal.end(), [&](int a, int b) { return height[a] < height[b]; });
        B.in_lv.assign(1, 0);
        for (size_t k = 0; k < internal.size(); ++k) {
            B.in_nodes.push_back(internal[k]);
            if (k + 1 == internal.size() || height[internal[k + 1]] != height[internal[k]]) B.in_lv.push_back(int(k + 1));
        }
        std::stable_sort(internal.begin(), internal.end(), [&](int a, int b) { return depth[a] < depth[b]; });
        B.out_lv.assign(1, 0);
        for (size_t k = 0; k < internal.size(); ++k) {
            for (int c : kids[internal[k]]) B.out_kids.push_back(c);
            if (k + 1 == internal.size() || depth[internal[k + 1]] != depth[internal[k]])
                B.out_lv.push_back(int(B.out_kids.size()));
        }
        for (int u : members)
            if (u != root) B.acc.push_back(u);
    }
    return pl;
}

}  // namespace h3g
