// Host-side Huffman / exp-Golomb codebooks of the XnYZip container streams.
//
// The reference builds its codes with std::unordered_map / std::priority_queue
// (encoder/huffman_encoder.hpp:33-147): the code bits, the tie-breaking between equal
// frequencies and the order of the entries in the serialized meta all follow libstdc++'s
// container order, which depends only on the sequence of distinct symbols inserted (the
// order of first occurrence in the data) and the final frequencies.  The kernels therefore
// return, per symbol, its frequency and first-occurrence index, and this file re-runs the
// same container operations on them to obtain byte-identical codes and metas.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace xnyz {

struct CodeEntry {
    uint32_t bits;  // code value (the low 32 bits of longer codes, which are zero-extended)
    uint8_t len;
};

struct SymbolStat {
    uint64_t symbol;    // symbol value (two's complement for signed types)
    uint64_t count;     // frequency
    uint64_t first;     // index of its first occurrence in the data
};

// Result of building one stream's code.
struct StreamCode {
    bool exp_golomb = false;
    uint8_t eg_k = 0;
    std::vector<uint8_t> meta;                 // serialized meta (get_meta)
    std::vector<uint64_t> symbols;             // coded symbols (Huffman mode)
    std::vector<CodeEntry> codes;              // their codes, parallel to `symbols`
    uint64_t encoded_bits = 0;                 // total bits of the encoded stream
};

// Symbol type of the stream (the template argument of HuffmanEncoder<T> in the reference).
enum class SymType { U64, U8, I32 };

// One build() + get_meta() of a fresh HuffmanEncoder<T> (used for the repos / SFC-delta and
// quad symbol streams).  `stats` in any order; `total` = number of symbols.
StreamCode build_stream_code(SymType type, std::vector<SymbolStat> stats, uint64_t total);

// The -rle count stream (composer/block_compressor_rle.hpp:290-303): build, measure, switch
// to exp-Golomb when the meta exceeds a quarter of the data, build again on the same object.
StreamCode build_count_code(std::vector<SymbolStat> stats, uint64_t total);

// HuffmanEncoder<T>::build_complete (huffman_encoder.hpp:70-85), the shared-codebook fit:
// the data's symbols in first-occurrence order, then every value of [0, alphabet_max] the data
// lacks with frequency 1, built without the exp-Golomb switch.
StreamCode build_complete_code(SymType type, std::vector<SymbolStat> stats, uint64_t total, uint64_t alphabet_max);

// A fresh HuffmanEncoder<T> given `meta` by load_meta (huffman_encoder.hpp:172-203), then
// get_meta + encode: the meta written back lists the loaded table in its own iteration
// order.  Fails when the meta is malformed or a symbol of `stats` has no code.
bool loaded_stream_code(SymType type, const uint8_t* meta, uint64_t len, std::vector<SymbolStat> stats,
                        StreamCode& out, std::string& err);

// Parsed meta of a stream for decoding (load_meta, huffman_encoder.hpp:172-203).
struct ParsedMeta {
    bool exp_golomb = false;
    uint8_t eg_k = 0;
    std::vector<uint64_t> symbols;
    std::vector<CodeEntry> codes;
    int distinct = 0;  // distinct symbols (code_table size)
};
// Returns false with a message on malformed input.
bool parse_meta(SymType type, const uint8_t* meta, uint64_t len, ParsedMeta& out, std::string& err);

// Golomb-Rice parameter (golomb_rice_encoder.hpp:157-183).
uint8_t golomb_rice_k(uint64_t sum, uint64_t count, bool all_zero);

}  // namespace xnyz
