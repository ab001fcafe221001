/* Minimal declarations of the public libzstd API used by the reference CPU
 * Chain modules.  No zstd development headers are installed in this image;
 * the shared library itself (libzstd.so.1) is, so the oracle build links
 * against it directly.  Only names and signatures of the documented public
 * functions are declared here. */
#ifndef CHAIN_ORACLE_ZSTD_SHIM_H
#define CHAIN_ORACLE_ZSTD_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define ZSTD_CONTENTSIZE_UNKNOWN (0ULL - 1)
#define ZSTD_CONTENTSIZE_ERROR   (0ULL - 2)
size_t ZSTD_compressBound(size_t srcSize);
size_t ZSTD_compress(void* dst, size_t dstCapacity, const void* src, size_t srcSize,
                     int compressionLevel);
size_t ZSTD_decompress(void* dst, size_t dstCapacity, const void* src, size_t compressedSize);
unsigned ZSTD_isError(size_t code);
const char* ZSTD_getErrorName(size_t code);
unsigned long long ZSTD_getFrameContentSize(const void* src, size_t srcSize);
#ifdef __cplusplus
}
#endif
#endif
