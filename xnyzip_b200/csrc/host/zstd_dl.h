// Run-time binding of libzstd 1.5.7, the version the reference pins (conanfile.py:14).
// The container's final stage is one ZSTD_compress(level 3) frame (composer/utils.hpp:35-53);
// a byte-identical frame needs exactly this library version, so others are refused.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace xnyz {

// Loads the library (path, else $XNYZ_ZSTD_LIBRARY, else the build-time default).
bool zstd_load(const char* path, std::string& err);
bool zstd_available(std::string& err);

// ZSTD_compress(level) into `out` (resized).  Returns false with a message on error.
bool zstd_compress(const uint8_t* src, size_t n, int level, std::vector<uint8_t>& out, std::string& err);
bool zstd_compress_into(const uint8_t* src, size_t n, int level, uint8_t* dst, size_t cap, size_t& written,
                        std::string& err);
size_t zstd_bound(size_t n);
// Frame content size (decompress_buffer, composer/utils.hpp:11-32); false if not a frame
// or the size is unknown.
bool zstd_content_size(const uint8_t* src, size_t n, uint64_t& size, std::string& err);
bool zstd_decompress(const uint8_t* src, size_t n, uint8_t* dst, uint64_t dst_size, std::string& err);

}  // namespace xnyz
