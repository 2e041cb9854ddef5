/* Prototype-only stand-in for <zstd.h> so the reference's sz_lossless.cpp
 * compiles against the system libzstd.so.1 (the image ships the shared
 * library but not its development header).  Only the three entry points and
 * the one constant that the reference calls are declared; signatures follow
 * the public zstd API. */
#ifndef CPSZ_ORACLE_ZSTD_PROTO_H
#define CPSZ_ORACLE_ZSTD_PROTO_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define ZSTD_CONTENTSIZE_ERROR (0ULL - 2)
size_t ZSTD_compress(void* dst, size_t dstCapacity, const void* src, size_t srcSize, int compressionLevel);
size_t ZSTD_decompress(void* dst, size_t dstCapacity, const void* src, size_t compressedSize);
unsigned long long ZSTD_getFrameContentSize(const void* src, size_t srcSize);
#ifdef __cplusplus
}
#endif
#endif
