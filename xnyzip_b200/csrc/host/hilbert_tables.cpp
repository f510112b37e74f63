// Builds the Hilbert state machines used by the kernels.
//
// The curve is the one of the reference (quantizer/hilbert-curves-cpp/hilbert.cpp): base
// Gray-code pattern {0,1,3,2,6,7,5,4} mapping Hilbert index to Morton octant (:33,44), the 24
// cube rotations as octant permutations enumerated from 90-degree Euler angles and ordered
// lexicographically (:197-238), and a depth-first search choosing, for each child in curve
// order, the first rotation whose entry corner touches the previous child's exit corner
// (:269-337).  The resulting per-octant child orientations define the curve; the reference
// applies them digit by digit with an O(levels^2) loop (:412-464), here they are folded
// into state machines whose state is the accumulated orientation, so a code is transformed
// with one table lookup per 3-bit level.
#include "hilbert_tables.h"

#include <algorithm>
#include <map>
#include <set>
#include <stdexcept>
#include <vector>

namespace xnyz {
namespace {

using Perm = std::array<uint8_t, 8>;
constexpr Perm kH2M = {0, 1, 3, 2, 6, 7, 5, 4};

Perm inverse(const Perm& p) {
    Perm r{};
    for (int i = 0; i < 8; ++i) r[p[i]] = static_cast<uint8_t>(i);
    return r;
}

// (p o q)(x) = p[q[x]]
Perm compose(const Perm& p, const Perm& q) {
    Perm r{};
    for (int i = 0; i < 8; ++i) r[i] = p[q[i]];
    return r;
}

std::array<int, 3> octant_corner(int v) { return {(v >> 2) & 1, (v >> 1) & 1, v & 1}; }

std::vector<Perm> rotations() {
    static const int sn[4] = {0, 1, 0, -1}, cs[4] = {1, 0, -1, 0};
    std::set<Perm> all;
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
            for (int c = 0; c < 4; ++c) {
                const int sx = sn[a], sy = sn[b], sz = sn[c], cx = cs[a], cy = cs[b], cz = cs[c];
                const int m[3][3] = {{cx * cy, sx * sz - cx * cz * sy, cz * sx + cx * sy * sz},
                                     {sy, cy * cz, -cy * sz},
                                     {-cy * sx, cx * sz + cz * sx * sy, cx * cz - sx * sy * sz}};
                Perm p{};
                for (int i = 0; i < 8; ++i) {
                    const int v[3] = {((i >> 2) & 1) * 2 - 1, ((i >> 1) & 1) * 2 - 1, (i & 1) * 2 - 1};
                    int r[3];
                    for (int k = 0; k < 3; ++k) r[k] = (m[k][0] * v[0] + m[k][1] * v[1] + m[k][2] * v[2] + 1) / 2;
                    p[i] = static_cast<uint8_t>((r[0] << 2) | (r[1] << 1) | r[2]);
                }
                all.insert(p);
            }
    return std::vector<Perm>(all.begin(), all.end());
}

bool search(const std::vector<Perm>& rots, Perm child[8], int i, std::array<int, 3> prev_exit) {
    const auto pos = [](int idx) { return octant_corner(kH2M[idx]); };
    std::array<int, 3> first{}, last{}, here{};
    for (int k = 0; k < 3; ++k) {
        first[k] = pos(0)[k] * 3;
        last[k] = pos(7)[k] * 3;
        here[k] = pos(i)[k] * 2;
    }
    for (const Perm& r : rots) {
        const auto b = octant_corner(r[kH2M[0]]);
        const std::array<int, 3> entry{b[0] + here[0], b[1] + here[1], b[2] + here[2]};
        if (i == 0) {
            if (entry != first) continue;
        } else {
            int d2 = 0;
            for (int k = 0; k < 3; ++k) d2 += (entry[k] - prev_exit[k]) * (entry[k] - prev_exit[k]);
            if (d2 != 1) continue;
        }
        const auto e = octant_corner(r[kH2M[7]]);
        const std::array<int, 3> exit{e[0] + here[0], e[1] + here[1], e[2] + here[2]};
        if (i != 7) {
            if (!search(rots, child, i + 1, exit)) continue;
        } else if (exit != last) {
            continue;
        }
        child[kH2M[i]] = r;
        return true;
    }
    return false;
}

// BFS over states reachable from the identity; step(state perm, digit) -> (out, next perm).
template <typename Step>
int build_machine(std::array<uint8_t, 256>& tab, Step step) {
    std::map<Perm, int> index;
    std::vector<Perm> states;
    Perm id{};
    for (int i = 0; i < 8; ++i) id[i] = static_cast<uint8_t>(i);
    index[id] = 0;
    states.push_back(id);
    for (size_t s = 0; s < states.size(); ++s) {
        for (int d = 0; d < 8; ++d) {
            Perm next;
            const int out = step(states[s], d, next);
            auto it = index.find(next);
            int ni;
            if (it == index.end()) {
                ni = static_cast<int>(states.size());
                index[next] = ni;
                states.push_back(next);
            } else {
                ni = it->second;
            }
            if (ni >= 32) throw std::runtime_error("Hilbert state machine exceeds 32 states");
            tab[s * 8 + d] = static_cast<uint8_t>(out | (ni << 3));
        }
    }
    return static_cast<int>(states.size());
}

HilbertMachines make() {
    const auto rots = rotations();
    Perm child_h2m[8];
    if (!search(rots, child_h2m, 0, {0, 0, 0})) throw std::runtime_error("Hilbert child search failed");
    Perm child_m2h[8];
    for (int i = 0; i < 8; ++i) child_m2h[i] = inverse(child_h2m[i]);
    const Perm m2h = inverse(kH2M);
    HilbertMachines hm{};
    hm.fwd.fill(0);
    hm.inv.fill(0);
    // Forward: digit d of the current level is first moved by the accumulated orientation A,
    // emitted through the base pattern, and the child orientation of that octant is
    // composed onto A for the lower levels.
    hm.fwd_states = build_machine(hm.fwd, [&](const Perm& A, int d, Perm& next) {
        const int md = A[d];
        next = compose(child_m2h[md], A);
        return static_cast<int>(m2h[md]);
    });
    // Inverse: the Morton octant of Hilbert digit h is h2m[h] seen through the orientation B
    // accumulated from the higher levels; the child orientation of that octant composes
    // on the right.
    hm.inv_states = build_machine(hm.inv, [&](const Perm& B, int h, Perm& next) {
        const int md = kH2M[h];
        next = compose(B, child_h2m[md]);
        return static_cast<int>(B[md]);
    });
    uint32_t s = 0, t = 0;
    for (int level = 20; level >= 6; --level) {
        if ((hm.fwd[s * 8] & 7) != 0 || (hm.inv[t * 8] & 7) != 0)
            throw std::runtime_error("Hilbert zero digit does not map to zero");
        s = hm.fwd[s * 8] >> 3;
        t = hm.inv[t * 8] >> 3;
    }
    hm.fwd_block_start = s;
    hm.inv_block_start = t;
    return hm;
}

}  // namespace

const HilbertMachines& hilbert_machines() {
    static const HilbertMachines hm = make();
    return hm;
}

uint64_t hilbert_apply_host(const std::array<uint8_t, 256>& tab, uint64_t code, int top, uint32_t state) {
    uint64_t out = top >= 21 ? 0 : (top >= 20 ? (code & (1ull << 63)) : (code & (~0ull << (3 * (top + 1)))));
    for (int l = top; l >= 0; --l) {
        const uint32_t d = static_cast<uint32_t>(code >> (3 * l)) & 7u;
        const uint32_t e = tab[state * 8 + d];
        out |= static_cast<uint64_t>(e & 7u) << (3 * l);
        state = e >> 3;
    }
    return out;
}

}  // namespace xnyz
