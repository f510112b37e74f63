// Launchers of the sm_100a kernels (implemented in k_*.cu), called by the host pipeline.
// All pointers are device pointers unless named *_host; every launcher is asynchronous on
// `st`.  Plain C++ types only, so host .cpp files include this without CUDA headers.
#pragma once

#include <cstddef>
#include <cstdint>

typedef struct CUstream_st* cudaStream_t;

namespace xnyz {
namespace dev {

struct QuantParams {
    int quantizer;  // 0 cube, 1 truncated octahedron, 2 adaptive
    float div;      // float(double(2*l2)/sqrt(3|5))
    float s;        // l2 as float
    float rdiv;     // float(sqrt(3|5))
    float step[3];  // adaptive: per-axis steps (decompression: from the container)
    const float* step_dev;  // adaptive compression: the steps in device memory (PointStats::step)
};

// Results of the bounding-box / quantization sweeps (one struct in device memory).
struct PointStats {
    unsigned long long minkey[3];  // per axis: (order key << 32) | first index of the minimum
    int max_cell[3];               // max lattice index per axis (>= 0: starts at 0 like the reference)
    int min_cell[3];               // min lattice index per axis (starts at INT_MAX)
    unsigned int nonfinite;        // inputs that are NaN or +-inf
    unsigned int mse_max_bits;     // max per-point squared error (float bits)
    double mse_sum;                // sum of per-point squared errors
    unsigned int err;              // device error bits
    float offset[3];               // shift offset (written by quantize_range)
    unsigned int maxkey[3];        // per axis: largest order key (bbox, for the adaptive steps)
    float step[3];                 // adaptive quantizer steps (launch_adaptive_steps)
};

// Key layout of block mode.  Normal cells: key = id << 21 | quad << 18 | sfc18.  Cells with
// z = -1 (the truncated-octahedron edge case) carry `defect_flag` and the id minus
// `defect_base` so that they sort after all other cells in the reference's id order.
struct BlockKeyParams {
    unsigned long long nx, ny;
    unsigned long long defect_flag;  // 0 if no z = -1 cells
    unsigned long long defect_base;  // ((2^64-1)/64/2) * nx * ny  (mod 2^64)
    int hilbert;
    unsigned int hstart;  // Hilbert state after levels 20..6 (all zero digits)
};

// Key layout of direct mode: key = sfc, or defect_flag | (sfc & (defect_flag - 1)) for z = -1
// cells whose high sfc bits equal `defect_high`.
struct DirectKeyParams {
    int bits;      // hilbert_bits = bit length of the max range (>= 1)
    int hilbert;
    unsigned long long defect_flag;
    unsigned long long defect_high;
};

// Unit (unique cell, or point for -normal) outputs of the segment kernels.
struct UnitOutputs {
    uint8_t* rep_sym;               // PFor symbol of repos / sfc delta per unit
    uint8_t* quad_sym;              // PFor symbol of the quad delta per unit (block mode)
    unsigned long long* patches;    // PFor patches in order
    unsigned long long* blk_id;     // block mode: id of each block
    uint32_t* blk_unit;             // block mode: first unit of each block
    uint32_t* unit_pos;             // -rle: sorted position of each unit's first point
    unsigned long long* hist_rep;   // [256]
    uint32_t* first_rep;            // [256]
    unsigned long long* hist_quad;  // [256]
    uint32_t* first_quad;           // [256]
    unsigned long long* counters;   // [0] units, [1] patches, [2] blocks, [3] sum of patches
    unsigned long long* rep_val;    // optional: repos / sfc delta value per unit (extended container)
};

struct LookBackState {
    uint32_t* flag;
    unsigned long long* agg;
    unsigned long long* inc;
};

// Count-stream statistics (-rle).
constexpr int kCountDense = 4096;
struct CountStats {
    unsigned long long* hist;   // [kCountDense]
    uint32_t* first;            // [kCountDense]
    uint32_t* over_val;         // counts >= kCountDense: value
    uint32_t* over_unit;        //   ... and unit index
    uint32_t* over_n;           // number of such counts
};

// Huffman code table for uint8 symbols, and for int counts (dense part + sorted sparse part).
struct ByteCodes {
    uint32_t bits[256];
    uint8_t len[256];
};

struct EncodeTotals {
    unsigned long long bits[8];  // total bits per stream (see Stream enum in pipeline.cpp)
};

// --- points ---------------------------------------------------------------------------
void launch_bbox(const float* xyz, uint64_t n, PointStats* stats, cudaStream_t st);
// AdaptiveQuantizer steps from the bounding box (after launch_bbox) into stats->step.
void launch_adaptive_steps(const float* xyz, float l2, PointStats* stats, cudaStream_t st);
// cells (optional, 3 n int32): each finite point's lattice cell, for launch_keys_cells.
void launch_quantize_range(const float* xyz, uint64_t n, QuantParams q, PointStats* stats, int with_error_stats,
                           cudaStream_t st, int32_t* cells = nullptr);
void launch_keys_block(const float* xyz, uint64_t n, QuantParams q, const PointStats* stats, BlockKeyParams kp,
                       const uint8_t* hilbert_tab, unsigned long long* keys, uint32_t* payload, int passes,
                       uint32_t* hist, cudaStream_t st);
void launch_keys_direct(const float* xyz, uint64_t n, QuantParams q, const PointStats* stats, DirectKeyParams kp,
                        const uint8_t* hilbert_tab, unsigned long long* keys, uint32_t* payload, int passes,
                        uint32_t* hist, cudaStream_t st);
// Cell tables: block keys from int32 cells; per-axis min / max of cells (stats->min_cell /
// max_cell, initialised by the caller); dst[i] = src[idx[i]]; expansion + recover + unshift
// (lb: flag, agg, inc of ceil(n / 4096) tiles; *total receives the point count).
void launch_keys_cells(const int32_t* cells, uint64_t n, BlockKeyParams kp, const uint8_t* hilbert_tab,
                       unsigned long long* keys, uint32_t* payload, int passes, uint32_t* hist, cudaStream_t st);
void launch_cells_stats(const int32_t* cells, uint64_t n, PointStats* stats, cudaStream_t st);
void launch_gather_i32(const int32_t* src, const uint32_t* idx, uint64_t n, int32_t* dst, cudaStream_t st);
void launch_expand_cells(const int32_t* cells, const int32_t* counts, uint64_t n, QuantParams q, const float* off3,
                         LookBackState lb, uint32_t* tile_counter, float* out, uint64_t cap,
                         unsigned long long* total, uint32_t* err, cudaStream_t st);
void launch_quantize_cells(const float* xyz, uint64_t n, QuantParams q, const PointStats* stats, int32_t* cells,
                           cudaStream_t st);
void launch_recover_cells(const int32_t* cells, uint64_t n, QuantParams q, const float* offset3_dev, float* xyz,
                          cudaStream_t st);
void launch_hilbert(const unsigned long long* in, uint64_t n, const uint8_t* tab, int top, unsigned int state,
                    unsigned long long* out, cudaStream_t st);

// --- sort -----------------------------------------------------------------------------
constexpr int kSortTile = 4096;
void launch_sort_histogram(const unsigned long long* keys, uint64_t n, int passes, uint32_t* hist, cudaStream_t st);
void launch_sort_offsets(uint32_t* hist, int passes, cudaStream_t st);  // in place: counts -> exclusive offsets
void launch_sort_pass(const unsigned long long* kin, unsigned long long* kout, const uint32_t* vin, uint32_t* vout,
                      uint64_t n, int shift, const uint32_t* offsets, unsigned long long* status, uint32_t epoch,
                      uint32_t* tile_counter, uint32_t* err, cudaStream_t st);

// --- compress segments + encoders -------------------------------------------------------
constexpr int kUnitTile = 4096;
void launch_units_block(const unsigned long long* keys, uint64_t n, int rle, BlockKeyParams kp, UnitOutputs out,
                        LookBackState lb, uint32_t* tile_counter, uint32_t* err, cudaStream_t st);
void launch_units_direct(const unsigned long long* keys, uint64_t n, int rle, DirectKeyParams kp, UnitOutputs out,
                         LookBackState lb, uint32_t* tile_counter, uint32_t* err, cudaStream_t st);
// unit_pos null: counts[] is the input (cell tables), else counts[] receives the run lengths.
void launch_count_stats(const uint32_t* unit_pos, uint64_t units, uint64_t n, int32_t* counts, CountStats cs,
                        cudaStream_t st);
// Block deltas (blk ids and block unit counts) and their maxima.
void launch_block_deltas(const unsigned long long* blk_id, const uint32_t* blk_unit, uint64_t nblocks, uint64_t units,
                         unsigned long long* d_blk, unsigned long long* d_cnt, unsigned long long* max2,
                         cudaStream_t st);
void launch_bitpack(const unsigned long long* vals, uint64_t n, int width, uint32_t* words, cudaStream_t st);

constexpr int kEncTile = 4096;
// Encoders write at most cap_bits bits (the output buffer's size) and flag an overflow beyond.
void launch_gr_encode(const unsigned long long* vals, uint64_t n, int k, uint32_t* words, uint64_t cap_bits,
                      LookBackState lb, uint32_t* tile_counter, unsigned long long* total_bits, uint32_t* err,
                      cudaStream_t st);
// A code whose codewords all have one length len (1..24): symbol i at stream bits [i len, (i + 1) len)
// (code_bits indexed by the symbol; for counts the dense table); *total_bits = n * len.
void launch_fixed_encode_u8(const uint8_t* sym, uint64_t n, const uint32_t* code_bits, int len, uint32_t* words,
                            unsigned long long* total_bits, cudaStream_t st);
void launch_fixed_encode_i32(const int32_t* sym, uint64_t n, const uint32_t* code_bits, int len, uint32_t* words,
                             unsigned long long* total_bits, cudaStream_t st);
void launch_huff_encode_u8(const uint8_t* sym, uint64_t n, const ByteCodes* codes, uint32_t* words,
                           uint64_t cap_bits, LookBackState lb, uint32_t* tile_counter, unsigned long long* total_bits,
                           uint32_t* err, cudaStream_t st);
// counts: Huffman (eg_k < 0) with a dense table [kCountDense] and sorted sparse values, or
// exp-Golomb with parameter eg_k >= 0.
void launch_count_encode(const int32_t* counts, uint64_t n, int eg_k, const uint32_t* dense_bits,
                         const uint8_t* dense_len, const uint32_t* sparse_val, const uint32_t* sparse_bits,
                         const uint8_t* sparse_len, uint32_t sparse_n, uint32_t* words, uint64_t cap_bits,
                         LookBackState lb, uint32_t* tile_counter, unsigned long long* total_bits, uint32_t* err,
                         cudaStream_t st);

// --- decompress -------------------------------------------------------------------------
constexpr int kScanTile = 4096;  // elements per tile of the decompress-side chained scans

// Parallel decoding of one unindexed prefix-code stream (Huffman, Golomb-Rice, exp-Golomb),
// implemented in k_stream_decode.cu.
enum CodeKind { kCodeHuffman = 0, kCodeGolombRice = 1, kCodeExpGolomb = 2 };
struct DecodeTable {
    // Huffman: primary table of 2^root_bits entries (1 <= root_bits <= 11): (len << 24) |
    // payload for codes of at most root_bits bits, 0 for a prefix that is no code,
    // (1u << 31) | node for longer codes; tree nodes hold two children each (leaf =
    // (1u << 31) | payload, internal = node index, missing = 0xffffffff).  The payload is
    // the symbol value when symvals is null, else an index into symvals.
    const uint32_t* root;
    const uint32_t* tree;
    const unsigned long long* symvals;
    int root_bits;
    int param;   // Golomb-Rice / exp-Golomb k
    int zigzag;  // exp-Golomb of a signed symbol type
};
constexpr int kDecodeMaxL = 64;       // longest entry offset tracked per subsequence
constexpr int kDecodeSubBits = 512;   // bits per subsequence (thread): Huffman, exp-Golomb
constexpr int kDecodeSubBitsGR = 1024;  // Golomb-Rice (longer subsequences amortise its entry tables)
constexpr int kDecodeBlockSubs = 128; // subsequences per thread block
// flag: [tiles]; agg: [tiles * kDecodeMaxL]; inc: [tiles * 2];
// tiles = ceil(ceil(bits / sub bits) / kDecodeBlockSubs) (kDecodeSubBits, the smaller, bounds
// the tiles of every kind).
// The stream starts `base_bits` (< 32) into `words`.  L = entry offsets tracked (the longest
// codeword; Golomb-Rice derives k + 2 from its parameter, L_run is unused).
void launch_decode_stream(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits, DecodeTable t,
                          int L, const uint32_t* L_run, uint64_t nsym, int out_width, void* out, uint32_t* flag,
                          unsigned long long* agg, unsigned long long* inc, uint32_t* tile_counter, uint32_t* err,
                          uint32_t* need_fallback, unsigned long long* total_codewords, cudaStream_t st);
// One-thread decoder the host runs when a bounded wait of the parallel decoder expired.
// A Huffman stream whose codewords all have length len (== t.root_bits <= 11): every symbol
// from its own len bits (out_width 1: u8, 4: u32 values; with out_width 4 and sum_out, *sum_out
// += the sum of max(value, 0) over the values, as int32).
void launch_decode_fixed(const uint32_t* words, uint64_t base_bits, uint64_t total_bits, DecodeTable t, int len,
                         uint64_t nsym, int out_width, void* out, uint32_t* err, cudaStream_t st,
                         unsigned long long* sum_out = nullptr);
void launch_decode_sequential(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits,
                              DecodeTable t, uint64_t nsym, int out_width, void* out,
                              unsigned long long* total_codewords, uint32_t* err, cudaStream_t st);
void launch_count_total(const int32_t* counts, uint64_t n, unsigned long long* total, cudaStream_t st);
void launch_fill_u8(uint8_t* p, uint64_t n, uint8_t v, cudaStream_t st);
void launch_fill_u32(uint32_t* p, uint64_t n, uint32_t v, cudaStream_t st);

// Division of any 64-bit value by an invariant divisor d >= 1 through one high multiply
// (T. Granlund and P. Montgomery, "Division by invariant integers using multiplication",
// PLDI 1994, section 4, figure 4.1): with l = ceil(log2 d) and m = floor(2^64 (2^l - d) / d)
// + 1, x / d = (t + ((x - t) >> min(l, 1))) >> max(l - 1, 0) where t = mulhi(m, x).
struct U64Div {
    unsigned long long m;
    unsigned int sh1, sh2;
};
inline U64Div make_u64div(unsigned long long d) {
    unsigned int l = 0;
    while (l < 64 && (static_cast<unsigned __int128>(1) << l) < d) ++l;
    const unsigned __int128 num = (static_cast<unsigned __int128>(1) << 64) *
                                  ((static_cast<unsigned __int128>(1) << l) - d);
    U64Div r;
    r.m = static_cast<unsigned long long>(num / d + 1);
    r.sh1 = l < 1 ? l : 1;
    r.sh2 = l > 1 ? l - 1 : 0;
    return r;
}

// LCP recovery (block mode) or SFC prefix sum (direct mode) fused with the PFor decode,
// -rle expansion, recover and unshift.
struct RecoverParams {
    QuantParams q;
    float off[3];
    unsigned long long nx, ny;
    U64Div div_nx, div_ny;   // make_u64div(nx), make_u64div(ny)
    int hilbert;
    unsigned int hstart_inv;  // inverse-Hilbert state after levels 20..6 of zero digits
    int rle;
    int direct;
    int bits;   // direct mode hilbert_bits
    int cells;  // write the units' int32 lattice cells instead of points (no expansion, no recover)
};
struct RecoverInputs {
    const uint8_t* rep_sym;
    const unsigned long long* rep_patch;
    uint64_t npatch;
    const uint8_t* quad_sym;
    const uint8_t* is_start;       // block mode: 1 where a non-empty block starts
    const uint32_t* start_block;   // block mode: block index at those units
    const unsigned long long* blk_ids;
    uint64_t nblocks;
    const int32_t* counts;         // -rle
    const unsigned long long* rep_val;  // extended container: repos / sfc delta per unit (replaces rep_sym + patches)
};
// Block streams of block mode in one pass: bit-unpack (widths <= 64), inclusive prefix sums of
// the block-id and block-count deltas, block-start marks (is_start zeroed by the caller).
// lb: flag [2 * tiles], agg and inc [4 * tiles] u64; tiles = ceil(nblocks / 4096).
void launch_block_streams(const uint32_t* words_blk, uint64_t base_blk, int width_blk, const uint32_t* words_cnt,
                          uint64_t base_cnt, int width_cnt, uint64_t nblocks, uint64_t units,
                          unsigned long long* blk_ids, uint8_t* is_start, uint32_t* start_block, LookBackState lb,
                          uint32_t* tile_counter, unsigned long long* count_total, uint32_t* err, cudaStream_t st);
// flag: [5 * tiles]; agg, inc: [10 * tiles]; tiles = ceil(units / 4096)
void launch_recover_units(const RecoverInputs& in, uint64_t units, uint64_t nout, RecoverParams rp,
                          const uint8_t* hilbert_inv_tab, uint32_t* flag, unsigned long long* agg,
                          unsigned long long* inc, uint32_t* tile_counter, float* out, uint32_t* err,
                          cudaStream_t st);


// --- block-parameter coding (extended container) and its predictor ------------------------
constexpr int kParamBlock = 1024;     // values per block
constexpr int kParamFeatures = 34;    // features per block (row stride of the feature array)
constexpr int kParamInputs = 34;
constexpr int kParamOutputsK = 32;    // Golomb-Rice k in 0..31
constexpr int kParamOutputsW = 33;    // PFor width w in 0..32
constexpr int kParamCount = 64 * 48 + 64 + 64 * 64 + 64 + 72 * 64 + 72;  // FP32 parameters of the MLP
void launch_block_features(const unsigned long long* v, uint64_t n, float* feats, cudaStream_t st);
// Exhaustive (w, k) search per block; `only` (may be null) restricts it to flagged blocks.
void launch_block_search(const unsigned long long* v, uint64_t n, const uint8_t* only, uint8_t* w, uint8_t* k,
                         uint32_t* cost, cudaStream_t st);
void launch_block_cost(const unsigned long long* v, uint64_t n, const uint8_t* w, const uint8_t* k, uint32_t* cost,
                       cudaStream_t st);
void launch_block_offsets(const uint32_t* cost, uint64_t nblk, unsigned long long* offs, unsigned long long* total,
                          cudaStream_t st);
void launch_block_encode(const unsigned long long* v, uint64_t n, const uint8_t* w, const uint8_t* k,
                         const unsigned long long* offs, uint32_t* payload, cudaStream_t st);
void launch_block_decode(const uint32_t* payload, uint64_t payload_bits, uint64_t n, const uint8_t* w,
                         const uint8_t* k, const unsigned long long* offs, unsigned long long* out, uint32_t* err,
                         cudaStream_t st);
void launch_block_fallback(const float* conf, uint64_t nblk, float thr, uint8_t* flags, unsigned long long* count,
                           cudaStream_t st);
// One (w = 0, k = floor(log2(mean))) pair for every block; sum: device double, zeroed.
void launch_block_global(const unsigned long long* v, uint64_t n, double* sum, uint8_t* w, uint8_t* k,
                         cudaStream_t st);
void launch_mlp_forward(const float* prm, const float* feats, uint64_t count, uint8_t* w, uint8_t* k, float* conf,
                        float* logits, cudaStream_t st);
size_t mlp_gather_floats(uint64_t count);
void launch_mlp_train(const float* prm, const float* feats, const uint8_t* wlab, const uint8_t* klab,
                      const uint32_t* idx, uint64_t first, uint64_t count, float scale, float* grad, float* loss,
                      float* gather, cudaStream_t st);
void launch_mlp_adam(float* prm, float* grad, float* m, float* v, float lr, int step, cudaStream_t st);

// zstd frames on the GPU (k_zstd.cu): frame i of src_len[i] bytes at src[i] into dst[i]
// (capacity cap[i]); out_len[i] = content size or < 0 (zstd_dec.cuh error codes).  The
// pointer and size arrays are in device memory; `workspace` holds count * zstd_workspace_bytes().
size_t zstd_workspace_bytes();
void launch_zstd_frames(const uint8_t* const* src, const uint64_t* src_len, uint8_t* const* dst, const uint64_t* cap,
                        long long* out_len, void* workspace, uint64_t count, cudaStream_t st);

}  // namespace dev
}  // namespace xnyz
