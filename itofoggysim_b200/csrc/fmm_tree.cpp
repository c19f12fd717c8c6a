// libtree box arithmetic on the host: de-/interleaving of Morton codes, box centres, the I2
// neighbourhood and the I4 interaction list of a box (every candidate inside the domain).  These
// serve the handle-less box entries and the domain queries of the ABI; the ML-FMM's hierarchy and
// pass lists are built on the device (k_tree.cu).
//
//   I2(box)  = the box and its neighbours at distance 1 (lib_tree_hf_get_neighbour_all_xD,
//              libtree/src/lib/lib_tree_helper_functions.f90:914-997),
//   I4(box)  = children of the parent's I2 minus the box's own I2 (lib_tree_get_domain_i4,
//              libtree/src/lib/lib_tree.f90:994-1143).
// Box indices are Morton codes with dimension 1 most significant in each 3-bit group, as the
// universal index (lib_tree_hf_get_universal_index, lib_tree_helper_functions.f90:202-364).
#include <algorithm>
#include <cmath>

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

}  // namespace foggy
