// Replays HuffmanEncoder<T>::build / build_from_freq / build_code / get_meta
// (encoder/huffman_encoder.hpp:33-147,250-309) from per-symbol statistics.
//
// The container operations are the ones the reference performs, in the same order:
//   * freq: std::unordered_map<T, uint64_t>, distinct symbols inserted in order of first
//     occurrence (what `for (v : data) freq[v]++` does), final counts assigned;
//   * the entropy sum and the priority-queue pushes iterate freq in its own order;
//   * priority_queue with comparator `a.freq > b.freq`, pop two, push the merged node;
//   * code_table: std::unordered_map<T, Code> filled by a left-first walk of the tree, and
//     (for the -rle count stream) reused after clear(), which keeps its bucket array;
//   * the meta lists code_table in its iteration order.
#include "codebook.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <queue>
#include <unordered_map>

namespace xnyz {
namespace {

template <typename T>
uint64_t to_unsigned(T v) {
    if constexpr (std::is_signed<T>::value) {
        const int64_t s = static_cast<int64_t>(v);
        return (static_cast<uint64_t>(s) << 1) ^ static_cast<uint64_t>(s >> 63);
    } else {
        return static_cast<uint64_t>(v);
    }
}

int bit_length_min1(uint64_t v) {
    int l = v ? 64 - __builtin_clzll(v) : 0;
    return l ? l : 1;
}

template <typename T>
class Replay {
public:
    struct Code {
        uint32_t bits;
        uint8_t length;
    };

    bool use_eg = false;
    uint8_t eg_k = 0;
    std::unordered_map<T, Code> code_table;

    // `ordered` = distinct symbols in first-occurrence order with their frequencies.
    void build(const std::vector<std::pair<T, uint64_t>>& ordered, uint64_t total) {
        code_table.clear();
        if (total == 0) return;
        std::unordered_map<T, uint64_t> freq;
        for (const auto& sc : ordered) freq[sc.first] = sc.second;
        double entropy = 0.0;
        for (auto& kv : freq) {
            const double p = double(kv.second) / total;
            entropy -= p * std::log2(p);
        }
        if (entropy > 10.0 || use_eg) {
            use_eg = true;
            eg_k = best_exp_golomb_k(freq);
            return;
        }
        from_freq(freq);
    }

    // build_complete (:70-85): fresh freq map, then the missing values of [0, amax].
    void build_complete(const std::vector<std::pair<T, uint64_t>>& ordered, T amax) {
        code_table.clear();
        use_eg = false;
        eg_k = 0;
        std::unordered_map<T, uint64_t> freq;
        for (const auto& sc : ordered) freq[sc.first] = sc.second;
        for (T s = 0; s <= amax; ++s) {
            if (freq.find(s) == freq.end()) freq[s] = 1;
            if (s == std::numeric_limits<T>::max()) break;
        }
        from_freq(freq);
    }

    // load_meta (:172-203) on a fresh encoder: entries inserted in the meta's order (a
    // repeated symbol keeps its last code).
    bool load(const uint8_t* m, uint64_t len, std::string& err) {
        code_table.clear();
        use_eg = false;
        eg_k = 0;
        uint64_t p = 0;
        if (len >= 4 && m[0] == 0xE1 && m[1] == 0xC1 && m[2] == 0x01) {
            p = 4;
            if (m[3] == 0x01) {
                eg_k = len > 4 ? m[4] : 0;
                use_eg = true;
                return true;
            }
        }
        if (p + 4 > len) {
            err = "truncated Huffman meta in the profile";
            return false;
        }
        const uint32_t count =
            (uint32_t(m[p]) << 24) | (uint32_t(m[p + 1]) << 16) | (uint32_t(m[p + 2]) << 8) | uint32_t(m[p + 3]);
        p += 4;
        const uint64_t entry = sizeof(T) + 1 + 4;
        if (count > (len - p) / entry) {
            err = "truncated Huffman meta in the profile";
            return false;
        }
        for (uint32_t i = 0; i < count; ++i) {
            T sym;
            if constexpr (sizeof(T) == 8) {
                uint64_t v = 0;
                for (int k = 0; k < 8; ++k) v = (v << 8) | m[p++];
                sym = static_cast<T>(v);
            } else {
                std::memcpy(&sym, m + p, sizeof(T));
                p += sizeof(T);
            }
            const uint8_t l = m[p++];
            const uint32_t b =
                (uint32_t(m[p]) << 24) | (uint32_t(m[p + 1]) << 16) | (uint32_t(m[p + 2]) << 8) | uint32_t(m[p + 3]);
            p += 4;
            code_table[sym] = Code{b, l};
        }
        return true;
    }

    std::vector<uint8_t> meta() const {
        if (use_eg) return {0xE1, 0xC1, 0x01, 0x01, eg_k};
        std::vector<uint8_t> out;
        put_be32(out, static_cast<uint32_t>(code_table.size()));
        for (auto& kv : code_table) {
            if constexpr (sizeof(T) == 8) {
                for (int s = 56; s >= 0; s -= 8) out.push_back(static_cast<uint8_t>(static_cast<uint64_t>(kv.first) >> s));
            } else {
                T v = kv.first;
                uint8_t b[sizeof(T)];
                std::memcpy(b, &v, sizeof(T));
                out.insert(out.end(), b, b + sizeof(T));
            }
            out.push_back(kv.second.length);
            put_be32(out, kv.second.bits);
        }
        return out;
    }

    uint64_t encoded_bits(const std::vector<std::pair<T, uint64_t>>& ordered) const {
        uint64_t bits = 0;
        for (const auto& sc : ordered) {
            if (use_eg) {
                const uint64_t n = to_unsigned(sc.first);
                const uint64_t n1 = (n >> eg_k) + 1;
                bits += sc.second * static_cast<uint64_t>(2 * bit_length_min1(n1) - 1 + eg_k);
            } else {
                bits += sc.second * code_table.at(sc.first).length;
            }
        }
        return bits;
    }

private:
    static void put_be32(std::vector<uint8_t>& o, uint32_t v) {
        o.push_back(static_cast<uint8_t>(v >> 24));
        o.push_back(static_cast<uint8_t>(v >> 16));
        o.push_back(static_cast<uint8_t>(v >> 8));
        o.push_back(static_cast<uint8_t>(v));
    }

    // select_best_exp_golomb_k (:344-363): the cost only depends on the value, so it is
    // summed over distinct symbols weighted by their frequency.
    static uint8_t best_exp_golomb_k(const std::unordered_map<T, uint64_t>& freq) {
        uint64_t best = std::numeric_limits<uint64_t>::max();
        uint8_t bk = 0;
        for (uint8_t k = 0; k <= 16; ++k) {
            uint64_t cost = 0;
            for (auto& kv : freq) {
                const uint64_t n1 = (to_unsigned(kv.first) >> k) + 1;
                cost += kv.second * static_cast<uint64_t>(2 * bit_length_min1(n1) - 1 + k);
            }
            if (cost < best) {
                best = cost;
                bk = k;
            }
        }
        return bk;
    }

    struct Node {
        T symbol{};
        uint64_t freq = 0;
        int left = -1, right = -1;
    };

    void from_freq(const std::unordered_map<T, uint64_t>& freq) {
        if (freq.empty()) return;
        std::vector<Node> nodes;
        nodes.reserve(2 * freq.size());
        auto cmp = [&nodes](int a, int b) { return nodes[a].freq > nodes[b].freq; };
        std::priority_queue<int, std::vector<int>, decltype(cmp)> pq(cmp);
        for (auto& kv : freq) {
            nodes.push_back(Node{kv.first, kv.second, -1, -1});
            pq.push(static_cast<int>(nodes.size()) - 1);
        }
        while (pq.size() > 1) {
            const int a = pq.top();
            pq.pop();
            const int b = pq.top();
            pq.pop();
            nodes.push_back(Node{T{}, nodes[a].freq + nodes[b].freq, a, b});
            pq.push(static_cast<int>(nodes.size()) - 1);
        }
        walk(nodes, pq.top(), 0u, 0);
    }

    void walk(const std::vector<Node>& nodes, int n, uint32_t prefix, uint8_t len) {
        const Node& nd = nodes[n];
        if (nd.left < 0 && nd.right < 0) {
            code_table[nd.symbol] = len == 0 ? Code{0, 1} : Code{prefix, len};
            return;
        }
        walk(nodes, nd.left, prefix << 1, static_cast<uint8_t>(len + 1));
        walk(nodes, nd.right, (prefix << 1) | 1u, static_cast<uint8_t>(len + 1));
    }
};

template <typename T>
std::vector<std::pair<T, uint64_t>> ordered_stats(std::vector<SymbolStat>& stats) {
    std::sort(stats.begin(), stats.end(), [](const SymbolStat& a, const SymbolStat& b) { return a.first < b.first; });
    std::vector<std::pair<T, uint64_t>> out;
    out.reserve(stats.size());
    for (const auto& s : stats)
        if (s.count) out.emplace_back(static_cast<T>(s.symbol), s.count);
    return out;
}

template <typename T>
StreamCode finish(const Replay<T>& r, const std::vector<std::pair<T, uint64_t>>& ordered) {
    StreamCode sc;
    sc.exp_golomb = r.use_eg;
    sc.eg_k = r.eg_k;
    sc.meta = r.meta();
    sc.encoded_bits = r.encoded_bits(ordered);
    if (!r.use_eg) {
        for (auto& kv : r.code_table) {
            sc.symbols.push_back(static_cast<uint64_t>(static_cast<int64_t>(kv.first)));
            sc.codes.push_back(CodeEntry{kv.second.bits, kv.second.length});
        }
    }
    return sc;
}

template <typename T>
StreamCode build_one(std::vector<SymbolStat>& stats, uint64_t total) {
    auto ordered = ordered_stats<T>(stats);
    Replay<T> r;
    r.build(ordered, total);
    return finish(r, ordered);
}

template <typename T>
T read_symbol(const uint8_t* m, uint64_t& p) {
    if constexpr (sizeof(T) == 8) {
        uint64_t v = 0;
        for (int k = 0; k < 8; ++k) v = (v << 8) | m[p++];
        return static_cast<T>(v);
    } else {
        T v;
        std::memcpy(&v, m + p, sizeof(T));
        p += sizeof(T);
        return v;
    }
}

template <typename T>
bool parse_meta_t(const uint8_t* meta, uint64_t len, ParsedMeta& out, std::string& err) {
    out = ParsedMeta{};
    if (len >= 4 && meta[0] == 0xE1 && meta[1] == 0xC1 && meta[2] == 0x01) {
        if (meta[3] == 0x01) {
            out.exp_golomb = true;
            out.eg_k = len > 4 ? meta[4] : 0;
            return true;
        }
        // header with Huffman mode: the reference then parses from offset 4
    }
    uint64_t p = (len >= 4 && meta[0] == 0xE1 && meta[1] == 0xC1 && meta[2] == 0x01) ? 4 : 0;
    if (p + 4 > len) {
        err = "truncated Huffman meta";
        return false;
    }
    const uint32_t count = (uint32_t(meta[p]) << 24) | (uint32_t(meta[p + 1]) << 16) | (uint32_t(meta[p + 2]) << 8) |
                           uint32_t(meta[p + 3]);
    p += 4;
    const uint64_t entry = sizeof(T) + 1 + 4;
    if (count > (len - p) / entry) {
        err = "truncated Huffman meta";
        return false;
    }
    // code_table[sym] = {bits, len}: a repeated symbol keeps its last entry.
    std::unordered_map<T, size_t> where;
    for (uint32_t i = 0; i < count; ++i) {
        const T s = read_symbol<T>(meta, p);
        const uint8_t l = meta[p++];
        const uint32_t b = (uint32_t(meta[p]) << 24) | (uint32_t(meta[p + 1]) << 16) | (uint32_t(meta[p + 2]) << 8) |
                           uint32_t(meta[p + 3]);
        p += 4;
        auto it = where.find(s);
        if (it == where.end()) {
            where[s] = out.symbols.size();
            out.symbols.push_back(static_cast<uint64_t>(static_cast<int64_t>(s)));
            out.codes.push_back(CodeEntry{b, l});
        } else {
            out.codes[it->second] = CodeEntry{b, l};
        }
    }
    out.distinct = static_cast<int>(out.symbols.size());
    return true;
}

}  // namespace

StreamCode build_stream_code(SymType type, std::vector<SymbolStat> stats, uint64_t total) {
    switch (type) {
        case SymType::U64: return build_one<uint64_t>(stats, total);
        case SymType::U8: return build_one<uint8_t>(stats, total);
        default: return build_one<int>(stats, total);
    }
}

StreamCode build_complete_code(SymType type, std::vector<SymbolStat> stats, uint64_t total, uint64_t alphabet_max) {
    (void)total;
    switch (type) {
        case SymType::U64: {
            auto ordered = ordered_stats<uint64_t>(stats);
            Replay<uint64_t> r;
            r.build_complete(ordered, alphabet_max);
            return finish(r, ordered);
        }
        case SymType::U8: {
            auto ordered = ordered_stats<uint8_t>(stats);
            Replay<uint8_t> r;
            r.build_complete(ordered, static_cast<uint8_t>(std::min<uint64_t>(alphabet_max, 255)));
            return finish(r, ordered);
        }
        default: {
            auto ordered = ordered_stats<int>(stats);
            Replay<int> r;
            r.build_complete(ordered, static_cast<int>(std::min<uint64_t>(alphabet_max, 0x7fffffff)));
            return finish(r, ordered);
        }
    }
}

namespace {
template <typename T>
bool loaded_one(const uint8_t* meta, uint64_t len, std::vector<SymbolStat>& stats, StreamCode& out, std::string& err) {
    auto ordered = ordered_stats<T>(stats);
    Replay<T> r;
    if (!r.load(meta, len, err)) return false;
    if (!r.use_eg)
        for (const auto& sc : ordered)
            if (!r.code_table.count(sc.first)) {
                err = "a symbol of the stream has no code in the profile";
                return false;
            }
    out = finish(r, ordered);
    return true;
}
}  // namespace

bool loaded_stream_code(SymType type, const uint8_t* meta, uint64_t len, std::vector<SymbolStat> stats,
                        StreamCode& out, std::string& err) {
    switch (type) {
        case SymType::U64: return loaded_one<uint64_t>(meta, len, stats, out, err);
        case SymType::U8: return loaded_one<uint8_t>(meta, len, stats, out, err);
        default: return loaded_one<int>(meta, len, stats, out, err);
    }
}

StreamCode build_count_code(std::vector<SymbolStat> stats, uint64_t total) {
    auto ordered = ordered_stats<int>(stats);
    Replay<int> r;
    r.build(ordered, total);
    const auto meta5 = r.meta();
    const uint64_t bytes5 = (r.encoded_bits(ordered) + 7) / 8;
    if (static_cast<double>(meta5.size()) > static_cast<double>(bytes5) * 0.25) r.use_eg = true;
    r.build(ordered, total);
    return finish(r, ordered);
}

bool parse_meta(SymType type, const uint8_t* meta, uint64_t len, ParsedMeta& out, std::string& err) {
    switch (type) {
        case SymType::U64: return parse_meta_t<uint64_t>(meta, len, out, err);
        case SymType::U8: return parse_meta_t<uint8_t>(meta, len, out, err);
        default: return parse_meta_t<int>(meta, len, out, err);
    }
}

uint8_t golomb_rice_k(uint64_t sum, uint64_t count, bool all_zero) {
    uint8_t k = 0;
    if (!all_zero && count) {
        const double average = static_cast<double>(sum) / count;
        k = average < 1.0 ? 0 : static_cast<uint8_t>(std::floor(std::log2(average)));
    }
    if (k >= 63) k = 62;
    return k;
}

}  // namespace xnyz
