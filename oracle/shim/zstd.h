/* Declarations of the libzstd 1.5.x entry points that the XnYZip reference calls.
 * Test infrastructure only: lets the unmodified reference sources compile against the
 * libzstd 1.5.7 runtime library on this image, whose development header is absent.
 * Names, signatures and the two content-size constants follow zstd's public API. */
#ifndef XNYZ_ORACLE_ZSTD_SHIM_H
#define XNYZ_ORACLE_ZSTD_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define ZSTD_CONTENTSIZE_UNKNOWN (0ULL - 1)
#define ZSTD_CONTENTSIZE_ERROR (0ULL - 2)
unsigned ZSTD_versionNumber(void);
size_t ZSTD_compressBound(size_t srcSize);
size_t ZSTD_compress(void* dst, size_t dstCapacity, const void* src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompress(void* dst, size_t dstCapacity, const void* src, size_t compressedSize);
unsigned long long ZSTD_getFrameContentSize(const void* src, size_t srcSize);
unsigned ZSTD_isError(size_t code);
const char* ZSTD_getErrorName(size_t code);
#ifdef __cplusplus
}
#endif
#endif
