// Table-driven form of the digit-permutation Hilbert transform of the reference
// (quantizer/hilbert-curves-cpp/hilbert.cpp:33-464).
#pragma once

#include <array>
#include <cstdint>

namespace xnyz {

// State machines over curve orientations.  Entry [state * 8 + digit] = out_digit | next << 3;
// state 0 is the identity orientation.
struct HilbertMachines {
    std::array<uint8_t, 256> fwd;   // Morton -> Hilbert (mortonToHilbert3)
    std::array<uint8_t, 256> inv;   // Hilbert -> Morton (hilbertToMorton3)
    uint32_t fwd_block_start;       // state after levels 20..6 of zero digits (18-bit local codes)
    uint32_t inv_block_start;
    int fwd_states;
    int inv_states;
};

const HilbertMachines& hilbert_machines();

// Host evaluation of the machines (used to cross-check the tables).
uint64_t hilbert_apply_host(const std::array<uint8_t, 256>& tab, uint64_t code, int top, uint32_t state);

}  // namespace xnyz
