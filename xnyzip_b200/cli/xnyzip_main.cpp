// XnYZip command line on the B200 path: same arguments, output files and stdout lines as
// the reference CLI (source/main.cpp:15-203), with compress/decompress through the C ABI.
//
//   XnYZip <input_file> <cube|to> <L2 bound> <-z|-h> <-rle|-normal> <decompression_file>
//          [direct_threshold (default 1024, 0 = force block)] [--offset=BYTES] [--count=BYTES]
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#include "xnyz.h"

namespace {

struct Chunk {
    bool active = false;
    uint64_t offset = 0, count = 0;
};

bool read_points(const char* path, const Chunk& ch, std::vector<float>& xyz, uint64_t& file_size) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) {
        std::fprintf(stderr, "Failed to open file: %s\n", path);
        return false;
    }
    file_size = static_cast<uint64_t>(f.tellg());
    uint64_t off = 0, bytes = file_size - file_size % 12;
    if (ch.active) {  // read_file_chunk (io/fileUtils.hpp:44-97)
        if (ch.offset % 12 || ch.count % 12) {
            std::fprintf(stderr, "offset/count must be multiples of 12\n");
            return false;
        }
        off = ch.offset;
        if (off >= file_size) {
            bytes = 0;
        } else {
            const uint64_t rem = file_size - off;
            bytes = (ch.count == 0 || ch.count > rem) ? rem - rem % 12 : ch.count;
        }
    }
    xyz.resize(bytes / 4);
    f.seekg(static_cast<std::streamoff>(off));
    if (bytes && !f.read(reinterpret_cast<char*>(xyz.data()), static_cast<std::streamsize>(bytes))) {
        std::fprintf(stderr, "short read\n");
        return false;
    }
    return true;
}

double seconds_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

int die(xnyz_status s) {
    std::fprintf(stderr, "xnyz error %d: %s\n", static_cast<int>(s), xnyz_last_error());
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    Chunk ch;
    std::vector<char*> pos;
    for (int i = 0; i < argc; ++i) {
        std::string a = argv[i];
        if (a.rfind("--offset=", 0) == 0) {
            ch.offset = std::stoull(a.substr(9));
            ch.active = true;
        } else if (a.rfind("--count=", 0) == 0) {
            ch.count = std::stoull(a.substr(8));
            ch.active = true;
        } else {
            pos.push_back(argv[i]);
        }
    }
    if (pos.size() < 7 || pos.size() > 8) {
        std::printf("Usage: %s <input_file> <quantizer_type (cube/to)> <L2 bound> <curve_type (-z/-h)> "
                    "<-rle/-normal> <decompression_file_name> [direct_threshold (default 1024, 0=force block)] "
                    "[--offset=BYTES] [--count=BYTES]\n",
                    argv[0]);
        return 1;
    }
    std::vector<float> xyz;
    uint64_t file_size = 0;
    if (!read_points(pos[1], ch, xyz, file_size)) return 1;
    const uint64_t n = xyz.size() / 3;
    if (ch.active)
        std::printf("Chunk mode: file_size=%lu offset=%lu count=%lu points=%lu\n", (unsigned long)file_size,
                    (unsigned long)ch.offset, (unsigned long)ch.count, (unsigned long)n);
    const std::string qname = pos[2];
    const bool hilbert = std::string(pos[4]) == "-h";
    const bool rle = std::string(pos[5]) == "-rle";
    const int threshold = pos.size() >= 8 ? std::stoi(pos[7]) : 1024;
    std::printf("SFC type: %s\nUse RLE: %s\nDirect threshold: %d\n", hilbert ? "Hilbert" : "Z-order", rle ? "Yes" : "No",
                threshold);
    const uint64_t input_bytes = n * 3 * sizeof(float);
    uint64_t compressed_bytes = 0;
    std::vector<float> recovered;
    std::vector<uint64_t> order;
    if (qname == "cube" || qname == "to") {
        const float l2 = std::stof(pos[3]);
        const int quant = qname == "to" ? XNYZ_QUANT_TO : XNYZ_QUANT_CUBE;
        xnyz_ctx* ctx = nullptr;
        xnyz_status s = xnyz_create(&ctx, 0, nullptr);
        if (s) return die(s);
        xnyz_params p{quant, l2, hilbert ? 1 : 0, rle ? 1 : 0, threshold};
        uint8_t* frame = nullptr;
        uint64_t flen = 0;
        xnyz_compress_info info{};
        if (!rle) order.resize(n);
        auto t0 = std::chrono::steady_clock::now();
        s = xnyz_compress(ctx, xyz.data(), n, 0, &p, 1, &frame, &flen, rle ? nullptr : order.data(), &info);
        const double tc = seconds_since(t0);
        if (s) return die(s);
        if (rle) {
            // BlockCompressorRLE::compress prints its quantization error statistics
            // (block_compressor_rle.hpp:53-87) and the dedup counts (:122-123).
            float mn[3] = {1e9f, 1e9f, 1e9f}, mx[3] = {-1e9f, -1e9f, -1e9f};
            for (uint64_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) {
                    mn[k] = std::min(mn[k], xyz[3 * i + k]);
                    mx[k] = std::max(mx[k], xyz[3 * i + k]);
                }
            const double range = (mx[0] - mn[0]) * (mx[0] - mn[0]) + (mx[1] - mn[1]) * (mx[1] - mn[1]) +
                                 (mx[2] - mn[2]) * (mx[2] - mn[2]);
            std::printf("Max L2 error: %lf\n", info.max_l2_error);
            std::printf("p2p psnr: %lf\n", 10.0 * std::log10(range / info.mse));
            std::printf("MSE: %f, range: %f\n", info.mse, range);
            std::printf("Max diff: %f, %f, %f\n", mx[0], mx[1], mx[2]);
            std::printf("Unique points: %lu\n", (unsigned long)info.num_units);
            std::printf("Duplicate ratio: %.3f\n", 1.0 - (double)info.num_units / (double)n);
        }
        std::printf("Encoding mode: %s\n", info.is_direct ? "direct" : "block");
        std::printf("compressed size of coords (after zstd): %lu\n", (unsigned long)flen);
        std::printf("compression ratio of coords (after zstd): %g\n", (double)n * 3 * sizeof(float) / flen);
        std::printf("XnYZip compression time = %gs\n", tc);
        compressed_bytes = flen;
        std::printf("compression ratio: %f\n", (float)n * 3 * sizeof(float) / flen * sizeof(uint8_t));
        float* out = nullptr;
        uint64_t nout = 0;
        t0 = std::chrono::steady_clock::now();
        s = xnyz_decompress(ctx, frame, flen, 1, quant, l2, rle ? 1 : 0, &out, &nout);
        const double td = seconds_since(t0);
        xnyz_free(frame);
        if (s) return die(s);
        std::printf("XnYZip decompression time = %gs\n", td);
        if (qname == "to") std::printf("decompressed finished, size: %lu\n", (unsigned long)nout);
        recovered.assign(out, out + 3 * nout);
        xnyz_free(out);
        xnyz_destroy(ctx);
    }
    std::printf("chunk input bytes: %lu\n", (unsigned long)input_bytes);
    std::printf("chunk compressed bytes: %lu\n", (unsigned long)compressed_bytes);
    {
        std::ofstream o(pos[6], std::ios::binary);
        o.write(reinterpret_cast<const char*>(recovered.data()),
                static_cast<std::streamsize>(recovered.size() * sizeof(float)));
    }
    if (!rle && (qname == "cube" || qname == "to")) {
        // main.cpp:161-201: compare the reordered input with the decoded points.
        const float bound = std::stof(pos[3]);
        double acc = 0;
        float maxerr = 0;
        int overflow = 0;
        std::vector<float> errors;
        errors.reserve(n);
        for (uint64_t i = 0; i < n && 3 * i + 2 < recovered.size(); ++i) {
            const float* a = &xyz[3 * order[i]];
            const float* b = &recovered[3 * i];
            float d[3];
            for (int k = 0; k < 3; ++k) {
                d[k] = a[k] - b[k];
                acc += d[k] * d[k];
            }
            const float e = std::sqrt(d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]));
            errors.push_back(e);
            if (e > bound) ++overflow;
            maxerr = std::max(maxerr, e);
        }
        {
            std::ofstream o("errors-" + qname + ".bin", std::ios::binary);
            o.write(reinterpret_cast<const char*>(errors.data()), static_cast<std::streamsize>(errors.size() * 4));
        }
        std::printf("overflow count: %d\n", overflow);
        std::printf("Max L2 error: %f\n", maxerr);
        acc /= n;
        float mn[3] = {1e9f, 1e9f, 1e9f}, mx[3] = {-1e9f, -1e9f, -1e9f};
        for (uint64_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                mn[k] = std::min(mn[k], xyz[3 * i + k]);
                mx[k] = std::max(mx[k], xyz[3 * i + k]);
            }
        const double range = (mx[0] - mn[0]) * (mx[0] - mn[0]) + (mx[1] - mn[1]) * (mx[1] - mn[1]) +
                             (mx[2] - mn[2]) * (mx[2] - mn[2]);
        std::printf("p2p psnr: %lf\n", 10.0 * std::log10(range / acc));
        std::printf("MSE: %f, range: %f\n", acc, range);
        std::printf("Max diff: %f, %f, %f\n", mx[0], mx[1], mx[2]);
    }
    return 0;
}
