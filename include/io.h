/*
 * io.h -- chunked input stream feeding bzip2_gpu_compress.
 *
 * Replaces the reference's BZFileInputStream (include/io.h:17-66,
 * src/utils/io.cpp:2-55): a reader thread fills up to n_buffers pinned
 * chunks of buffer_size bytes ahead from a file or stdin; fetch hands them
 * out in order.  Differences: a file that cannot be opened ends the stream at
 * once (the reference waits forever), no zero-length chunk is produced at end
 * of input, and the reader thread is joined by the destructor.
 *
 * Beyond the reference: fetch_pooled / release hand out chunks from a pool of
 * pinned buffers that are reused (no allocation per chunk), for consumers
 * that give every chunk back once it is compressed.
 */
#ifndef BZ2GPU_B200_IO_H
#define BZ2GPU_B200_IO_H

#include <stdint.h>

#include <string>

struct BZFileInputStream {
  /* read stdin */
  BZFileInputStream(int n_buffers, int buffer_size);
  /* read a file */
  BZFileInputStream(int n_buffers, int buffer_size, std::string filename);
  ~BZFileInputStream();
  BZFileInputStream(const BZFileInputStream &) = delete;
  BZFileInputStream &operator=(const BZFileInputStream &) = delete;

  /* Next chunk: result = cudaMallocHost'ed bytes (release with
   * cudaFreeHost), chunk_idx = its index.  Returns its length, or -1 at the
   * end of the input. */
  int fetch(uint8_t *&result, int &chunk_idx);
  /* Same, but the chunk stays owned by the stream's pool: give it back with
   * release() (and do not free it). */
  int fetch_pooled(uint8_t *&result, int &chunk_idx);
  void release(uint8_t *chunk);
  /* true if the input could not be opened or a read failed */
  bool failed() const;
  int buffer_size() const;

  struct Impl;

 private:
  Impl *impl_;
};

#endif
