// gg_rtree.cpp -- the initial comparison lists in the reference's R-tree order (host).
//
// grainhdl::find_neighbors (grainhdl.cpp:1029-1054) inserts every existing grain's box,
// in ascending ID order, into an R-tree (the vendored RTree.h: Guttman's R-tree with the
// quadratic split, at most 8 and at least 4 branches per node, node volumes measured as
// the volume of the box's circumscribed sphere in float), then each grain searches the
// tree with its own box (LSbox::computeDirectNeighbours, box.cpp:2871-2887) and keeps
// the hits other than itself in the order the depth-first search meets them.  That
// order is the comparison tie-break of every later step, so a run from these lists is
// bit-exact with the reference's.  The tree is restated here from that published
// algorithm: insertion descends to the child whose sphere volume grows least (ties to
// the smaller volume), a full node splits by picking the two most wasteful seeds and
// then assigning the branch with the largest growth difference first (ties to the group
// with fewer entries), and boxes overlap when they overlap or touch on every axis.  The
// float arithmetic is evaluated as the reference evaluates it.  Init-only work on the
// host: one tree of G boxes.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/gg_b200.h"

namespace {

constexpr int kMax = 8, kMin = 4;
constexpr float kUnitSphere3 = 4.188790f;  // the volume of the unit sphere in 3D

struct Rect {
    int lo[3], hi[3];
};

struct Branch {
    Rect r;
    int child;     // node index (internal nodes)
    uint32_t id;   // grain (leaves)
};

struct Node {
    int count = 0, level = -1;
    Branch b[kMax];
};

Rect combine(const Rect& a, const Rect& b) {
    Rect c;
    for (int d = 0; d < 3; d++) {
        c.lo[d] = a.lo[d] < b.lo[d] ? a.lo[d] : b.lo[d];
        c.hi[d] = a.hi[d] > b.hi[d] ? a.hi[d] : b.hi[d];
    }
    return c;
}

// The circumscribed sphere's volume, in float as the reference computes it.
float volume(const Rect& r) {
    float sum = 0.0f;
    for (int d = 0; d < 3; d++) {
        const float half = ((float)r.hi[d] - (float)r.lo[d]) * 0.5f;
        sum += half * half;
    }
    const float radius = (float)std::sqrt((double)sum);
    return radius * radius * radius * kUnitSphere3;
}

bool overlap(const Rect& a, const Rect& b) {
    for (int d = 0; d < 3; d++)
        if (a.lo[d] > b.hi[d] || b.lo[d] > a.hi[d]) return false;
    return true;
}

class Tree {
  public:
    Tree() { root_ = alloc(0); }

    void insert(const Rect& r, uint32_t id) {
        Branch br{r, -1, id};
        int split = -1;
        if (insert_rec(br, root_, &split, 0)) {  // the root split: a new root above both
            const int nr = alloc(nodes_[root_].level + 1);
            add(Branch{cover(root_), root_, 0}, nr, nullptr);
            add(Branch{cover(split), split, 0}, nr, nullptr);
            root_ = nr;
        }
    }

    void search(const Rect& r, std::vector<uint32_t>& out) const { search_rec(root_, r, out); }

  private:
    std::vector<Node> nodes_;
    int root_ = -1;

    int alloc(int level) {
        nodes_.push_back(Node());
        nodes_.back().level = level;
        return (int)nodes_.size() - 1;
    }

    Rect cover(int n) const {
        const Node& node = nodes_[n];
        Rect r = node.b[0].r;
        for (int i = 1; i < node.count; i++) r = combine(r, node.b[i].r);
        return r;
    }

    // Adds br to node n; returns true (and the new node in *split) when n had to split.
    bool add(const Branch& br, int n, int* split) {
        if (nodes_[n].count < kMax) {
            nodes_[n].b[nodes_[n].count++] = br;
            return false;
        }
        split_node(n, br, split);
        return true;
    }

    int pick_branch(const Rect& r, int n) const {
        const Node& node = nodes_[n];
        int best = 0;
        float best_incr = -1.0f, best_area = 0.0f;
        for (int i = 0; i < node.count; i++) {
            const float area = volume(node.b[i].r);
            const float incr = volume(combine(r, node.b[i].r)) - area;
            if (incr < best_incr || i == 0) {
                best = i;
                best_area = area;
                best_incr = incr;
            } else if (incr == best_incr && area < best_area) {
                best = i;
                best_area = area;
                best_incr = incr;
            }
        }
        return best;
    }

    bool insert_rec(const Branch& br, int n, int* split, int level) {
        if (nodes_[n].level > level) {
            const int i = pick_branch(br.r, n);
            int other = -1;
            const int child = nodes_[n].b[i].child;
            if (!insert_rec(br, child, &other, level)) {
                nodes_[n].b[i].r = combine(br.r, nodes_[n].b[i].r);
                return false;
            }
            nodes_[n].b[i].r = cover(child);
            return add(Branch{cover(other), other, 0}, n, split);
        }
        if (nodes_[n].level == level) return add(br, n, split);
        return false;
    }

    struct Partition {
        Branch buf[kMax + 1];
        int part[kMax + 1];
        bool taken[kMax + 1];
        int count[2] = {0, 0};
        Rect cov[2];
        float area[2] = {0.0f, 0.0f};
        float cover_area = 0.0f;
    };

    static void classify(Partition& p, int i, int g) {
        p.part[i] = g;
        p.taken[i] = true;
        p.cov[g] = p.count[g] == 0 ? p.buf[i].r : combine(p.buf[i].r, p.cov[g]);
        p.area[g] = volume(p.cov[g]);
        p.count[g]++;
    }

    void split_node(int n, const Branch& extra, int* split) {
        Partition p;
        const int total = kMax + 1;
        for (int i = 0; i < kMax; i++) p.buf[i] = nodes_[n].b[i];
        p.buf[kMax] = extra;
        Rect all = p.buf[0].r;
        for (int i = 1; i < total; i++) all = combine(all, p.buf[i].r);
        p.cover_area = volume(all);
        const int level = nodes_[n].level;
        nodes_[n].count = 0;
        for (int i = 0; i < total; i++) {
            p.taken[i] = false;
            p.part[i] = -1;
        }
        // the seeds: the pair whose combined box wastes the most volume
        float area[kMax + 1];
        for (int i = 0; i < total; i++) area[i] = volume(p.buf[i].r);
        float worst = -p.cover_area - 1;
        int s0 = 0, s1 = 1;
        for (int a = 0; a < total - 1; a++)
            for (int b = a + 1; b < total; b++) {
                const float waste = volume(combine(p.buf[a].r, p.buf[b].r)) - area[a] - area[b];
                if (waste > worst) {
                    worst = waste;
                    s0 = a;
                    s1 = b;
                }
            }
        classify(p, s0, 0);
        classify(p, s1, 1);
        while (p.count[0] + p.count[1] < total && p.count[0] < total - kMin && p.count[1] < total - kMin) {
            float biggest = -1.0f;
            int chosen = 0, better = 0;
            for (int i = 0; i < total; i++) {
                if (p.taken[i]) continue;
                const float g0 = volume(combine(p.buf[i].r, p.cov[0])) - p.area[0];
                const float g1 = volume(combine(p.buf[i].r, p.cov[1])) - p.area[1];
                float diff = g1 - g0;
                int group = 0;
                if (diff < 0) {
                    group = 1;
                    diff = -diff;
                }
                if (diff > biggest) {
                    biggest = diff;
                    chosen = i;
                    better = group;
                } else if (diff == biggest && p.count[group] < p.count[better]) {
                    chosen = i;
                    better = group;
                }
            }
            classify(p, chosen, better);
        }
        if (p.count[0] + p.count[1] < total) {
            const int group = p.count[0] >= total - kMin ? 1 : 0;
            for (int i = 0; i < total; i++)
                if (!p.taken[i]) classify(p, i, group);
        }
        const int other = alloc(level);
        *split = other;
        nodes_[n].level = level;
        for (int i = 0; i < total; i++) add(p.buf[i], p.part[i] == 0 ? n : other, nullptr);
    }

    void search_rec(int n, const Rect& r, std::vector<uint32_t>& out) const {
        const Node& node = nodes_[n];
        for (int i = 0; i < node.count; i++) {
            if (!overlap(r, node.b[i].r)) continue;
            if (node.level > 0) search_rec(node.b[i].child, r, out);
            else out.push_back(node.b[i].id);
        }
    }
};

}  // namespace

extern "C" int64_t gg_rtree_lists_from_boxes(int32_t n_grains, const int32_t* boxes, const uint8_t* valid,
                                             int64_t* offsets, uint32_t* ids, int64_t cap) {
    if (n_grains < 0 || !boxes || !valid || !offsets) return GG_ERR_INVALID;
    Tree tree;
    auto rect_of = [&](int g) {
        const int32_t* b = boxes + 6 * (int64_t)g;
        return Rect{{b[0], b[2], b[4]}, {b[1], b[3], b[5]}};
    };
    for (int g = 1; g <= n_grains; g++)
        if (valid[g]) tree.insert(rect_of(g), (uint32_t)g);
    std::vector<uint32_t> hits;
    int64_t total = 0;
    offsets[0] = offsets[1] = 0;
    for (int g = 1; g <= n_grains; g++) {
        if (valid[g]) {
            hits.clear();
            tree.search(rect_of(g), hits);
            for (uint32_t h : hits) {
                if (h == (uint32_t)g) continue;
                if (ids && total < cap) ids[total] = h;
                total++;
            }
        }
        offsets[g + 1] = total;
    }
    return total;
}
