/*
 * xnyz.h - C ABI of the B200-native XnYZip compress/decompress path.
 *
 * Every compute stage runs as a hand-written sm_100a CUDA kernel; host code only builds
 * Huffman codebooks (they depend on libstdc++ container order, see below), writes the
 * container header and calls libzstd.  Signatures use plain pointers and sizes only.
 *
 * Reference interfaces replaced (paths relative to the reference's source/ directory):
 *   xnyz_compress    <- XnYZip::BlockCompressor<float>::compress        composer/block_compressor.hpp:35,39
 *                       XnYZip::BlockCompressorRLE<float>::compress     composer/block_compressor_rle.hpp:34,38
 *   xnyz_decompress  <- XnYZip::BlockDecompressor<float>::decompress    composer/block_decompressor.hpp:27,31
 *                       XnYZip::BlockDecompressorRLE<float>::decompress composer/block_decompressor_rle.hpp:28,32
 *   quantizer codes  <- XnYZip::QUANTIZER_TYPE {CUBE, TRUNCATED_OCTAHEDRON, ADAPTIVE} composer/utils.hpp:55-59
 *                       (ADAPTIVE: AdaptiveQuantizer quantizer/adaptive_quantizer.hpp:16-97, its three
 *                       steps in the container's params; the stage entry points and the cell tables
 *                       take cube and truncated octahedron only)
 *   stage entry points (xnyz_stage_*) <- shift_points preprocessor/shifting.hpp:11,
 *       TruncatedOctahedronQuantizer/CubeQuantizer::quantize/recover quantizer/truncated_octahedron_quantizer.hpp, cube_quantizer.hpp,
 *       mve::mortonToHilbert3/hilbertToMorton3 quantizer/hilbert-curves-cpp/hilbert.hpp:8-9,
 *       radix_sort quantizer/block_quantizer.hpp:33.
 *
 * Errors are status codes; nothing throws across this boundary.  Calls on one context are
 * serialised on that context's CUDA stream; contexts are independent.
 */
#ifndef XNYZ_H
#define XNYZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum xnyz_status {
    XNYZ_OK = 0,
    XNYZ_ERR_INVALID_ARG = 1,  /* bad argument (null pointer, n == 0, unknown quantizer, ...) */
    XNYZ_ERR_BAD_STREAM = 2,   /* malformed or truncated container / bit stream */
    XNYZ_ERR_CUDA = 3,         /* a CUDA runtime call failed; see xnyz_last_error() */
    XNYZ_ERR_OOM = 4,          /* device or host allocation failed */
    XNYZ_ERR_TIMEOUT = 5,      /* a bounded device-side wait expired (kernel returned early) */
    XNYZ_ERR_UNSUPPORTED = 6,  /* input outside the supported envelope (e.g. > 64 key bits) */
    XNYZ_ERR_ZSTD = 7,         /* libzstd 1.5.7 missing, wrong version, or it reported an error */
    XNYZ_ERR_NO_DEVICE = 8     /* no CUDA device / the library was not built for this device */
} xnyz_status;

/* Quantizer codes (values follow XnYZip::QUANTIZER_TYPE). */
enum { XNYZ_QUANT_CUBE = 0, XNYZ_QUANT_TO = 1, XNYZ_QUANT_ADAPTIVE = 2 };

typedef struct xnyz_ctx xnyz_ctx;

/* Per-call configuration, mirroring the reference constructors and CLI flags. */
typedef struct xnyz_params {
    int quantizer;        /* XNYZ_QUANT_CUBE, XNYZ_QUANT_TO ("cube" / "to") or XNYZ_QUANT_ADAPTIVE */
    float l2_bound;       /* the L2 bound (CLI argv[3]) */
    int hilbert;          /* 1 = Hilbert curve ("-h"), 0 = Morton / z-order ("-z") */
    int rle;              /* 1 = "-rle" container, 0 = "-normal" */
    int direct_threshold; /* direct SFC mode when max range < threshold (CLI default 1024; 0 forces block) */
} xnyz_params;

/* Statistics of the last compress call (what the reference prints on stdout). */
typedef struct xnyz_compress_info {
    uint64_t num_points;      /* input points */
    uint64_t num_units;       /* unique cells (-rle) or points (-normal) */
    uint64_t num_blocks;      /* 128^3 super-block runs (block mode) */
    uint64_t num_patches;     /* PFor patches of the repos / SFC-delta stream */
    uint64_t container_bytes; /* pre-zstd container size */
    uint64_t output_bytes;    /* bytes returned (zstd frame, or container when zstd is off) */
    int32_t range[3];         /* max lattice index per axis (container fields) */
    int is_direct;            /* 1 = direct SFC mode, 0 = block mode */
    int counts_exp_golomb;    /* 1 if the -rle count stream switched to exp-Golomb */
    double max_l2_error;      /* max |p - recover(quantize(p))| (block_compressor_rle.hpp:53-67) */
    double mse;               /* mean squared error of the same */
    double gpu_ms;            /* device time of the call (CUDA events) */
} xnyz_compress_info;

/* ---- context ------------------------------------------------------------------------ */

/* Creates a context on `device`.  `stream` (a cudaStream_t, may be NULL) is the stream all
 * work of this context is issued on; NULL creates a private non-blocking stream. */
xnyz_status xnyz_create(xnyz_ctx** ctx, int device, void* stream);
xnyz_status xnyz_destroy(xnyz_ctx* ctx);
/* Message of the last error on this thread (static storage, never NULL). */
const char* xnyz_last_error(void);
/* Library version string. */
const char* xnyz_version(void);

/* Path of libzstd 1.5.7 (loaded on first use; the environment variable XNYZ_ZSTD_LIBRARY
 * overrides).  Returns XNYZ_ERR_ZSTD if it cannot be loaded or is not version 1.5.7. */
xnyz_status xnyz_set_zstd_library(const char* path);

/* Pinned host buffers (cudaHostAlloc) for fast host<->device copies. */
xnyz_status xnyz_host_alloc(void** ptr, size_t bytes);
xnyz_status xnyz_host_free(void* ptr);

/* Releases the context's cached device workspace. */
xnyz_status xnyz_trim(xnyz_ctx* ctx);

/* ---- whole path ------------------------------------------------------------------------ */

/* Compress n float32 xyz points (AoS, 12 bytes each).
 *   xyz_is_device : 1 if `xyz` is a device pointer, 0 if host memory (copied in).
 *   use_zstd      : 1 -> output is the zstd level-3 frame the reference returns
 *                   (composer/utils.hpp:35-53); 0 -> the raw pre-zstd container.
 *   out/out_len   : malloc'd host buffer with the result; release with xnyz_free().
 *   sort_order    : optional host array of n uint64 receiving, for each position of the
 *                   container's point order, the index of the input point (what
 *                   compress() does to its argument, block_compressor.hpp:141-144); NULL to skip.
 *   info          : optional statistics. */
xnyz_status xnyz_compress(xnyz_ctx* ctx, const float* xyz, uint64_t n, int xyz_is_device, const xnyz_params* params,
                          int use_zstd, uint8_t** out, uint64_t* out_len, uint64_t* sort_order,
                          xnyz_compress_info* info);

/* Compress into a device-resident container.  `xyz` is a device pointer; the container
 * stays in the context's workspace and is described by (*dev_container, *container_len)
 * until the next call on the context. */
xnyz_status xnyz_compress_device(xnyz_ctx* ctx, const float* xyz, uint64_t n, const xnyz_params* params,
                                 const uint8_t** dev_container, uint64_t* container_len, xnyz_compress_info* info);

/* No counterpart in the reference, which decodes its zstd frames with libzstd on the CPU
 * (composer/utils.hpp:11-33).  Decodes `count` zstd frames on the GPU, one frame per warp:
 * dev_frames[i] (device memory, frame_len[i] bytes) into dev_out[i] (device memory, out_cap[i]
 * bytes); out_len[i] receives the content size, or a negative code for a frame that did not
 * decode (then the call returns XNYZ_ERR_BAD_STREAM).  The pointer and size arrays are host
 * memory.  Workspace: about 137 KB per frame in the context's workspace.  Frames without a
 * dictionary only (the container frames have none). */
xnyz_status xnyz_zstd_decompress_device(xnyz_ctx* ctx, uint64_t count, const uint8_t* const* dev_frames,
                                        const uint64_t* frame_len, uint8_t* const* dev_out, const uint64_t* out_cap,
                                        int64_t* out_len);

/* Shared codebooks <- BlockCompressor<float>::fit_profile / compress_with_profile
 * (composer/block_compressor.hpp:241-431) and the profile blob of serialize_profile /
 * deserialize_profile (composer/block_encoding_profile.hpp:17-72): [u32 LE length][repos
 * Huffman meta][u32 LE length][quad Huffman meta].  Both write the -normal container in block
 * mode whatever the ranges (params->rle must be 0, direct_threshold is ignored) and reject
 * the extended container.  xnyz_fit_profile builds Huffman codes that cover every symbol
 * 0..255 (build_complete) and returns the container plus a malloc'd profile (free with
 * xnyz_free); xnyz_compress_with_profile codes with the profile's codebooks (load_meta) and
 * returns XNYZ_ERR_INVALID_ARG for an empty or malformed profile.  Frames decode with
 * xnyz_decompress as usual.  sort_order as in xnyz_compress. */
xnyz_status xnyz_fit_profile(xnyz_ctx* ctx, const float* xyz, uint64_t n, int xyz_is_device, const xnyz_params* params,
                             int use_zstd, uint8_t** out, uint64_t* out_len, uint64_t* sort_order, uint8_t** profile,
                             uint64_t* profile_len);
xnyz_status xnyz_compress_with_profile(xnyz_ctx* ctx, const float* xyz, uint64_t n, int xyz_is_device,
                                       const xnyz_params* params, const uint8_t* profile, uint64_t profile_len,
                                       int use_zstd, uint8_t** out, uint64_t* out_len, uint64_t* sort_order);

/* Decompress.  `in` is host memory holding a zstd frame (is_zstd = 1) or a raw container.
 * quantizer / l2_bound / rle must be the values used to compress (the container does not
 * record them, exactly as in the reference).  The result is written to a malloc'd host
 * array of 3*n floats (*xyz, release with xnyz_free) in the container's point order. */
xnyz_status xnyz_decompress(xnyz_ctx* ctx, const uint8_t* in, uint64_t in_len, int is_zstd, int quantizer,
                            float l2_bound, int rle, float** xyz, uint64_t* n);

/* As xnyz_decompress, into a caller-provided host array of `capacity` points (3 floats each;
 * pinned memory from xnyz_host_alloc gives the fastest copy).  *n receives the point count;
 * if it exceeds `capacity` nothing is copied and XNYZ_ERR_INVALID_ARG is returned. */
xnyz_status xnyz_decompress_into(xnyz_ctx* ctx, const uint8_t* in, uint64_t in_len, int is_zstd, int quantizer,
                                 float l2_bound, int rle, float* xyz, uint64_t capacity, uint64_t* n);

/* Decompress a device-resident raw container into a device array owned by the context
 * (valid until the next call).  Host code reads the few header fields it needs. */
xnyz_status xnyz_decompress_device(xnyz_ctx* ctx, const uint8_t* dev_container, uint64_t len, int quantizer,
                                   float l2_bound, int rle, const float** dev_xyz, uint64_t* n);

void xnyz_free(void* p);

/* ---- stage entry points (device pointers; used by the parity tests) ------------------ */

/* shift_points + quantize: offset3 (host, 3 floats) and cells (device, 3*n int32). */
xnyz_status xnyz_stage_quantize(xnyz_ctx* ctx, const float* dev_xyz, uint64_t n, int quantizer, float l2_bound,
                                float* offset3, int32_t* dev_cells);
/* quantizer->recover + unshift_points on device cells. */
xnyz_status xnyz_stage_recover(xnyz_ctx* ctx, const int32_t* dev_cells, uint64_t n, int quantizer, float l2_bound,
                               const float* offset3, float* dev_xyz);
/* mortonToHilbert3 (inverse = 0) or hilbertToMorton3 (inverse = 1) on n device codes. */
xnyz_status xnyz_stage_hilbert(xnyz_ctx* ctx, const uint64_t* dev_in, uint64_t n, unsigned iteration, int inverse,
                               uint64_t* dev_out);
/* Stable LSD radix sort of n uint64 keys over bits [0, key_bits) with an optional uint32
 * payload; results replace the inputs. */
xnyz_status xnyz_stage_sort(xnyz_ctx* ctx, uint64_t* dev_keys, uint32_t* dev_payload, uint64_t n, int key_bits);

/* ---- batches of independent clouds ----------------------------------------------------------- */

/* The reference compresses one cloud per call, and a file in chunks (main.cpp:15-71
 * --offset/--count, one container per chunk; the MPI driver runs chunks in parallel,
 * mpi_driver.cpp:809-941).  A batch runs many such calls at once: a pool of `workers` host
 * threads (<= 0: one per hardware thread, at most 32), each with its own context and CUDA
 * stream on `device`, takes clouds largest first, so the single-threaded libzstd frame of one
 * cloud overlaps the GPU work and the zstd frames of the others.  Every output is identical
 * to xnyz_compress / xnyz_decompress_into of that cloud alone. */
typedef struct xnyz_batch xnyz_batch;
xnyz_status xnyz_batch_create(xnyz_batch** batch, int device, int workers);
xnyz_status xnyz_batch_destroy(xnyz_batch* batch);
int xnyz_batch_workers(const xnyz_batch* batch);

/* Cloud i: xyz[i] (host, or device if xyz_is_device) with n[i] points and params[i].  out[i]
 * receives a malloc'd frame (release with xnyz_free) of out_len[i] bytes.  item_status (may
 * be NULL) receives each cloud's status; the return value is the status of the first failing
 * cloud by index (its message in xnyz_last_error), or XNYZ_OK. */
xnyz_status xnyz_batch_compress(xnyz_batch* batch, uint64_t count, const float* const* xyz, const uint64_t* n,
                                int xyz_is_device, const xnyz_params* params, int use_zstd, uint8_t** out,
                                uint64_t* out_len, xnyz_status* item_status);

/* Frame i: in[i] of in_len[i] bytes, decoded with quantizer[i], l2_bound[i], rle[i] into the
 * caller's host array xyz[i] of capacity[i] points; n[i] receives the point count. */
xnyz_status xnyz_batch_decompress(xnyz_batch* batch, uint64_t count, const uint8_t* const* in, const uint64_t* in_len,
                                  int is_zstd, const int* quantizer, const float* l2_bound, const int* rle,
                                  float* const* xyz, const uint64_t* capacity, uint64_t* n, xnyz_status* item_status);

/* No counterpart in the reference.  Host-buffer round trip of every cloud: the zstd frame
 * (malloc'd in frame[i], free with xnyz_free; byte-identical to xnyz_compress) and its
 * decompression into out[i] (n[i] points, in container order as xnyz_decompress returns
 * them), both on the same worker, so that one cloud's host zstd work overlaps another's GPU
 * work.  The reference's per-chunk threads do the same pair per chunk. */
xnyz_status xnyz_batch_roundtrip(xnyz_batch* batch, uint64_t count, const float* const* xyz, const uint64_t* n,
                                 const xnyz_params* params, uint8_t** frame, uint64_t* frame_len, float* const* out,
                                 xnyz_status* item_status);

/* ---- distributed-RLE cell tables ------------------------------------------------------------ */

/* XnYZip::BlockCompressorRLE<float>::encode_cells_with_counts (composer/block_compressor_rle.hpp:341-470):
 * n unique lattice cells (int32 xyz triples) with their counts, the GLOBAL ranges and offset,
 * Hilbert (1) or Morton (0) curve -> a -rle container in block mode (zstd frame when use_zstd).
 * Cells must lie in [0, range] (z may be -1, the truncated-octahedron edge cell); counts
 * travel in the container's cell order.  Inputs in device memory when cells_is_device. */
xnyz_status xnyz_encode_cells(xnyz_ctx* ctx, const int32_t* cells, const int32_t* counts, uint64_t n,
                              int cells_is_device, const int32_t* ranges, const float* offset, int hilbert,
                              int use_zstd, uint8_t** out, uint64_t* out_len);
/* XnYZip::BlockDecompressorRLE<float>::decompress_to_cells (composer/block_decompressor_rle.hpp:230-335):
 * a -rle block-mode container (zstd frame when is_zstd) -> its cells and counts in container
 * order (malloc'd, release with xnyz_free), the offset, ranges and curve flag.  A direct-mode
 * container is rejected with XNYZ_ERR_BAD_STREAM, as the reference throws. */
xnyz_status xnyz_decompress_to_cells(xnyz_ctx* ctx, const uint8_t* in, uint64_t in_len, int is_zstd,
                                     int32_t** cells, int32_t** counts, uint64_t* n, float* offset,
                                     int32_t* ranges, int* hilbert);
/* XnYZip::BlockDecompressorRLE<float>::expand_cells_to_points (composer/block_decompressor_rle.hpp:339-358):
 * every cell repeated counts[i] times, recovered by the quantizer and unshifted by offset
 * (host arrays in, a malloc'd array of 3 * n_points floats out). */
xnyz_status xnyz_expand_cells(xnyz_ctx* ctx, const int32_t* cells, const int32_t* counts, uint64_t n, int quantizer,
                              float l2_bound, const float* offset, float** xyz, uint64_t* n_points);

/* ---- extended container: block parameters of the repos / SFC-delta stream ------------------ *
 * No counterpart in the reference (it codes this stream with one Golomb-Rice k for the
 * patches and a Huffman code for the PFor symbols, block_compressor.hpp:122-136,174-190).
 * With a block mode other than XNYZ_BLOCKS_OFF, compress calls on the context write an
 * extended container: the first 8 bytes are "XNYZBX01", the rest is the reference layout
 * except that the stream's two entries (Golomb-Rice patches, Huffman symbols) become one
 * block-coded entry and an empty one.  Each block of 1024 values has its own PFor slot width
 * w in 0..32 and Golomb-Rice k in 0..31 (escapes, v >= 2^w - 1, hold v - (2^w - 1) as a
 * Golomb-Rice codeword capped at 96 bits) and its own bit offset, so blocks encode and decode
 * independently and the decoder never needs the predictor.  Every decompress entry point
 * recognises the prefix.
 *   XNYZ_BLOCKS_EXHAUSTIVE  (w, k) minimising each block's size over all 33 x 32 pairs
 *   XNYZ_BLOCKS_LEARNED     (w, k) predicted by a 34-64-64-(32+33) MLP (BF16 tensor-core
 *                           layers, FP32 accumulation) from block statistics; blocks whose
 *                           weaker head has softmax confidence at or below the fallback
 *                           threshold get the exhaustive search
 *   XNYZ_BLOCKS_GLOBAL      one pair for all blocks: w = 0, k = floor(log2(mean)) (the plain
 *                           method's parameter rule, golomb_rice_encoder.hpp:96-104) */
enum { XNYZ_BLOCKS_OFF = 0, XNYZ_BLOCKS_EXHAUSTIVE = 1, XNYZ_BLOCKS_LEARNED = 2, XNYZ_BLOCKS_GLOBAL = 3 };

typedef struct xnyz_block_info {
    uint64_t values;           /* values of the block-coded stream (units) */
    uint64_t blocks;           /* blocks of 1024 values */
    uint64_t payload_bits;     /* payload size (without the per-block w, k and offsets) */
    uint64_t fallback_blocks;  /* learned mode: blocks that got the exhaustive search */
    int mode;                  /* the block mode of the call (0: reference container) */
} xnyz_block_info;

xnyz_status xnyz_set_block_mode(xnyz_ctx* ctx, int mode);
/* Predictor parameters (host FP32 array of xnyz_model_param_count() values, the layout the
 * training entry points use) and the fallback confidence threshold (0: no block falls back,
 * 1: every block does).
 * Without a call, learned mode loads model/blockparams.f32 next to the library (or the file
 * named by XNYZ_MODEL) on first use. */
xnyz_status xnyz_set_model(xnyz_ctx* ctx, const float* params, uint64_t count, float fallback_confidence);
uint64_t xnyz_model_param_count(void);
/* Block statistics of the last compress call on the context. */
xnyz_status xnyz_last_block_info(xnyz_ctx* ctx, xnyz_block_info* info);
/* Sets the block mode of every context of a batch. */
xnyz_status xnyz_batch_set_block_mode(xnyz_batch* batch, int mode);

/* Stage entry points of the block coder and its predictor, for training and tests (device
 * pointers; `stream` is a cudaStream_t, NULL = default stream; all asynchronous).
 *   xnyz_stage_repos      the repos / SFC-delta value of every unit in container order (the
 *                         input of the block coder): runs the compress path on the context and
 *                         copies min(*count, cap) values to dev_out, *count = number of units
 *   xnyz_block_features   34 FP32 features per block: fraction of values per
 *                         min(31, bitlen(v)), mean and max of log2(v + 1) / 64
 *   xnyz_block_search     exhaustive (w, k) per block and its size in bits (dev_cost may be NULL)
 *   xnyz_block_cost       size in bits of each block under the given (w, k)
 *   xnyz_mlp_forward      predictor: argmax w and k per block, the two heads' softmax
 *                         confidences (dev_conf, 2 per block, may be NULL) and the 65 logits
 *                         (k logits 0..31, then w logits, may be NULL)
 *   xnyz_mlp_train_batch  forward + softmax cross-entropy of both heads + backward for samples
 *                         idx[first .. first + count) (idx NULL: first + i); adds scale * the
 *                         gradient to dev_grad and scale * the summed loss to dev_loss;
 *                         dev_gather is scratch of xnyz_mlp_gather_floats(count) floats
 *   xnyz_mlp_adam         Adam step (beta 0.9 / 0.999, eps 1e-8, step counted from 1) that also
 *                         clears dev_grad */
xnyz_status xnyz_stage_repos(xnyz_ctx* ctx, const float* dev_xyz, uint64_t n, const xnyz_params* params,
                             uint64_t* dev_out, uint64_t cap, uint64_t* count);
xnyz_status xnyz_block_features(const uint64_t* dev_vals, uint64_t n, float* dev_feats, void* stream);
xnyz_status xnyz_block_search(const uint64_t* dev_vals, uint64_t n, uint8_t* dev_w, uint8_t* dev_k,
                              uint32_t* dev_cost, void* stream);
xnyz_status xnyz_block_cost(const uint64_t* dev_vals, uint64_t n, const uint8_t* dev_w, const uint8_t* dev_k,
                            uint32_t* dev_cost, void* stream);
xnyz_status xnyz_mlp_forward(const float* dev_params, const float* dev_feats, uint64_t count, uint8_t* dev_w,
                             uint8_t* dev_k, float* dev_conf, float* dev_logits, void* stream);
uint64_t xnyz_mlp_gather_floats(uint64_t count);
xnyz_status xnyz_mlp_train_batch(const float* dev_params, const float* dev_feats, const uint8_t* dev_w,
                                 const uint8_t* dev_k, const uint32_t* dev_idx, uint64_t first, uint64_t count,
                                 float scale, float* dev_grad, float* dev_loss, float* dev_gather, void* stream);
xnyz_status xnyz_mlp_adam(float* dev_params, float* dev_grad, float* dev_m, float* dev_v, float lr, int step,
                          void* stream);

/* Device-resident round trip of a batch: each cloud (device points) is compressed into a
 * device container and decompressed again on a worker; the containers never leave HBM.
 * out_len[i] receives the container size, out_n[i] the decoded point count.  Clouds are
 * run by size class (point counts in powers of four from 16K), largest first, each class on
 * the number of concurrent workers xnyz_batch_autotune chose (all workers by default).  No
 * counterpart in the reference: it is the batch form of xnyz_compress_device +
 * xnyz_decompress_device, used to measure and verify whole batches. */
xnyz_status xnyz_batch_roundtrip_device(xnyz_batch* batch, uint64_t count, const float* const* dev_xyz,
                                        const uint64_t* n, const xnyz_params* params, uint64_t* out_len,
                                        uint64_t* out_n, xnyz_status* item_status);
/* Times the round trip on a sample of each size class with 1, 2, 4, ... workers and keeps the
 * fastest per class (class_workers, may be NULL, receives the 6 choices). */
xnyz_status xnyz_batch_autotune(xnyz_batch* batch, uint64_t count, const float* const* dev_xyz, const uint64_t* n,
                                const xnyz_params* params, int* class_workers);

/* ---- allocation-free entry point ---------------------------------------------------------- */

/* No counterpart in the reference.  The stable LSD radix sort of xnyz_stage_sort for callers
 * that cannot allocate device memory while they run (a real-time loop that must not block on
 * the CUDA allocator, a plugin whose host application owns all device memory): no context,
 * no cudaMalloc / cudaFree; all scratch lives in one fixed device array of about 12.6 MB
 * that every GPU loading the library holds until exit.  Sorts n <= 2^20 uint64 keys (and an
 * optional uint32 payload) in place over bits [0, key_bits) on `stream` (a cudaStream_t, NULL
 * = default stream) on the current device, and waits for the result.  n > 2^20 returns
 * XNYZ_ERR_UNSUPPORTED.  The first call on a device looks up the array's device address; make
 * it before any stream capture.  That address is cached per device for the primary context:
 * after cudaDeviceReset it is stale.  Calls share the array: calls that overlap on the GPU
 * (two streams, two host threads) race, so serialise them. */
xnyz_status xnyz_sort_noalloc(uint64_t* dev_keys, uint32_t* dev_payload, uint64_t n, int key_bits, void* stream);

/* ---- profiling ---------------------------------------------------------------------------- */

/* Enables (1) or disables (0) per-stage CUDA-event timing on the context's stream and clears
 * what was recorded. */
xnyz_status xnyz_profile(xnyz_ctx* ctx, int enable);
/* Synchronises the stream and writes a JSON object {stage: {"ms", "launches", "calls",
 * "bytes"}} of everything recorded since the last read (bytes = algorithmic traffic); *len
 * receives the full length.  Clears the record. */
xnyz_status xnyz_profile_read(xnyz_ctx* ctx, char* json, uint64_t cap, uint64_t* len);

/* ---- host-side helpers (no GPU needed) ----------------------------------------------- */

/* The table-driven Hilbert transform the kernels use, evaluated on the host
 * (mortonToHilbert3 / hilbertToMorton3, quantizer/hilbert-curves-cpp/hilbert.cpp:412-464). */
xnyz_status xnyz_host_hilbert(const uint64_t* in, uint64_t n, unsigned iteration, int inverse, uint64_t* out);

/* Huffman / exp-Golomb codebook of one stream from per-symbol statistics, exactly as
 * HuffmanEncoder<T>::build + get_meta produce it (encoder/huffman_encoder.hpp:33-147).
 *   symtype      : 0 uint64_t, 1 uint8_t, 2 int
 *   count_stream : 1 = the -rle count stream's build / measure / rebuild sequence
 *                  (composer/block_compressor_rle.hpp:290-303)
 *   symbols, counts, first_index : nsyms distinct symbols, their frequencies and the index
 *                  of their first occurrence; total = number of symbols in the data
 *   meta         : receives up to *meta_len bytes; *meta_len is set to the meta size */
xnyz_status xnyz_host_codebook(int symtype, int count_stream, const uint64_t* symbols, const uint64_t* counts,
                               const uint64_t* first_index, uint64_t nsyms, uint64_t total, uint8_t* meta,
                               uint64_t* meta_len, uint64_t* encoded_bits, int* exp_golomb);

#ifdef __cplusplus
}
#endif

#endif /* XNYZ_H */
