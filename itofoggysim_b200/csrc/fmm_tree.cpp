// Octree lists of the ML-FMM, built on the host from the device-sorted level-21 keys.
//
// Levels l_min..l_max hold the boxes that contain spheres (the reference's hierarchy of X/XY
// boxes, lib_ml_fmm_hf_create_hierarchy, libmlfmm/src/lib/lib_ml_fmm_helper_functions.f90:366-457).
// Because the spheres are sorted by key, the spheres of any box are one contiguous run of the
// sorted order, so
//   E1(box)  = the run of the box (lib_tree_get_domain_e1, libtree/src/lib/lib_tree.f90:492-609),
//   E2(box)  = the runs of the box and of its existing neighbours at distance 1
//              (lib_tree_get_domain_e2, :611-724, neighbours lib_tree_hf_get_neighbour_all_xD,
//              libtree/src/lib/lib_tree_helper_functions.f90:914-997),
//   I4(box)  = children of the parent's I2 minus the box's own I2, I2 = the box and its
//              neighbours (lib_tree_get_domain_i4, lib_tree.f90:994-1143), kept where they exist.
// Box indices are Morton codes with dimension 1 most significant in each 3-bit group, as the
// universal index (lib_tree_hf_get_universal_index, lib_tree_helper_functions.f90:202-364).
// Lists are in ascending Morton order, which is the reference's order wherever it does not go
// through its hash table (the order only changes the rounding of sums).
#include <algorithm>
#include <cmath>
#include <unordered_map>

#include "foggy_internal.h"

namespace foggy {

void morton_deinterleave(int64_t n, int l, int64_t c[3]) {
    c[0] = c[1] = c[2] = 0;
    for (int b = 0; b < l; ++b)
        for (int d = 0; d < 3; ++d) c[d] |= ((n >> (3 * b + (2 - d))) & 1) << b;
}

int64_t morton_interleave(const int64_t c[3], int l) {
    int64_t n = 0;
    for (int b = 0; b < l; ++b)
        for (int d = 0; d < 3; ++d) n |= ((c[d] >> b) & 1) << (3 * b + (2 - d));
    return n;
}

// normalised centre of box n at level l (lib_tree_hf_get_centre_of_box, :774-799)
void box_centre(int64_t n, int l, double out[3]) {
    int64_t c[3];
    morton_deinterleave(n, l, c);
    for (int d = 0; d < 3; ++d) out[d] = std::ldexp(1.0, -l) * ((double)c[d] + 0.5);
}

// the box and its neighbours at distance 1 that lie inside [0, 2^l)^3, own box first
void tree_i2(int64_t n, int l, std::vector<int64_t>& out) {
    out.clear();
    out.push_back(n);
    int64_t c[3], q[3];
    morton_deinterleave(n, l, c);
    const int64_t hi = ((int64_t)1 << l) - 1;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (!dx && !dy && !dz) continue;
                q[0] = c[0] + dx;
                q[1] = c[1] + dy;
                q[2] = c[2] + dz;
                if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] > hi || q[1] > hi || q[2] > hi) continue;
                out.push_back(morton_interleave(q, l));
            }
}

void tree_i4(int64_t n, int l, std::vector<int64_t>& out) {
    out.clear();
    if (l == 0) return;
    std::vector<int64_t> own, par;
    tree_i2(n, l, own);
    tree_i2(n >> 3, l - 1, par);
    std::sort(own.begin(), own.end());
    for (int64_t q : par)
        for (int c = 0; c < 8; ++c) {
            const int64_t b = (q << 3) | c;
            if (!std::binary_search(own.begin(), own.end(), b)) out.push_back(b);
        }
    std::sort(out.begin(), out.end());
}

void build_fmm_tree(int n, const uint64_t* key21_sorted, const int* order, int lmin, int lmax, FmmTree& t) {
    t = FmmTree();
    if (lmax < lmin) lmin = lmax;
    t.lmin = lmin;
    t.lmax = lmax;
    const int nlev = lmax - lmin + 1;
    t.level_base.assign(nlev + 1, 0);
    std::vector<std::unordered_map<int64_t, int>> id(nlev);
    std::vector<int> run_start, run_end;   // sorted-sphere run of each box (global id)
    for (int li = 0; li < nlev; ++li) {
        const int l = lmin + li;
        t.level_base[li] = (int)t.box_n.size();
        const int sh = 3 * (21 - l);
        for (int i = 0; i < n; ++i) {
            const int64_t b = (int64_t)(key21_sorted[i] >> sh);
            if (i == 0 || (int64_t)(key21_sorted[i - 1] >> sh) != b) {
                id[li][b] = (int)t.box_n.size();
                t.box_n.push_back(b);
                t.box_level.push_back(l);
                run_start.push_back(i);
                run_end.push_back(i + 1);
            } else {
                run_end.back() = i + 1;
            }
        }
    }
    const int nbox = (int)t.box_n.size();
    t.level_base[nlev] = nbox;
    // parents and children
    t.parent.assign(nbox, -1);
    std::vector<std::vector<int>> kids(nbox);
    for (int li = 1; li < nlev; ++li)
        for (int b = t.level_base[li]; b < t.level_base[li + 1]; ++b) {
            const int p = id[li - 1].at(t.box_n[b] >> 3);
            t.parent[b] = p;
            kids[p].push_back(b);
        }
    t.child_ptr.assign(nbox + 1, 0);
    for (int b = 0; b < nbox; ++b) {
        std::sort(kids[b].begin(), kids[b].end());
        t.child_ptr[b + 1] = t.child_ptr[b] + (int)kids[b].size();
        t.child_idx.insert(t.child_idx.end(), kids[b].begin(), kids[b].end());
    }
    // interaction lists
    t.i4_ptr.assign(nbox + 1, 0);
    std::vector<int64_t> own, cand;
    for (int li = 0; li < nlev; ++li) {
        const int l = lmin + li;
        for (int b = t.level_base[li]; b < t.level_base[li + 1]; ++b) {
            const int64_t nb = t.box_n[b];
            std::vector<int> list;
            tree_i4(nb, l, cand);
            for (int64_t q : cand) {
                auto it = id[li].find(q);
                if (it != id[li].end()) list.push_back(it->second);
            }
            t.i4_ptr[b + 1] = (int)t.i4_idx.size() + (int)list.size();
            t.i4_idx.insert(t.i4_idx.end(), list.begin(), list.end());
        }
    }
    // leaf lists (E1, E2) and the leaf box of each sphere
    const int lb0 = t.level_base[nlev - 1], nleaf = nbox - lb0;
    t.leaf_of.assign(n, -1);
    t.e1_ptr.assign(nleaf + 1, 0);
    t.e2_ptr.assign(nleaf + 1, 0);
    for (int q = 0; q < nleaf; ++q) {
        const int b = lb0 + q;
        for (int i = run_start[b]; i < run_end[b]; ++i) {
            t.e1_idx.push_back(order[i]);
            t.leaf_of[order[i]] = b;
        }
        t.e1_ptr[q + 1] = (int)t.e1_idx.size();
        tree_i2(t.box_n[b], lmax, own);
        std::sort(own.begin(), own.end());
        for (int64_t nb : own) {
            auto it = id[nlev - 1].find(nb);
            if (it == id[nlev - 1].end()) continue;
            for (int i = run_start[it->second]; i < run_end[it->second]; ++i) t.e2_idx.push_back(order[i]);
        }
        t.e2_ptr[q + 1] = (int)t.e2_idx.size();
    }
}

}  // namespace foggy
