/*
 * crc32.h -- bzip2 block CRC of a host buffer, computed on the GPU.
 * Replaces the reference's src/compression/crc32.h:7-8 (crc32.cpp:3-29).
 */
#ifndef BZ2GPU_B200_CRC32_H
#define BZ2GPU_B200_CRC32_H

#include <stddef.h>
#include <stdint.h>

/* Kept for source compatibility; the GPU path needs no table set-up. */
void crc32_init();
/* CRC of `length` HOST bytes (copied to the current device). */
uint32_t bzip2_crc32(const uint8_t *data, size_t length);

#endif
