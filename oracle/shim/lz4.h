/* Clean-room declaration shim for the LZ4 block API (test infrastructure only).
 *
 * The reference vendors LZ4 as the git submodule external/lz4 (unpinned
 * commit), which is empty in this checkout.  The reference only calls four
 * names of the public LZ4 block API (phase1_bucket_write/bucket_io.hpp:255-263,
 * :695; phase3_stitch/stitch_extmem.hpp:520,583-585).  This header declares
 * exactly those, with the signatures of the public lz4.h documentation, and
 * the build links the system runtime library liblz4.so.1 (1.9.4) that
 * implements them.  Compressed bytes never affect decoded content. */
#ifndef CDBG_SHIM_LZ4_H
#define CDBG_SHIM_LZ4_H

#ifdef __cplusplus
extern "C" {
#endif

#define LZ4_MAX_INPUT_SIZE 0x7E000000 /* 2 113 929 216 bytes, per the LZ4 format doc */

int LZ4_compressBound(int inputSize);
int LZ4_compress_default(const char* src, char* dst, int srcSize, int dstCapacity);
int LZ4_decompress_safe(const char* src, char* dst, int compressedSize, int dstCapacity);

#ifdef __cplusplus
}
#endif

#endif
