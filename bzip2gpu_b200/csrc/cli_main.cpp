// bzip2gpu command line tool (reference: src/main.cpp:20-60).  Blocks are
// 900,000 raw bytes for every level, as in the reference (its input stream
// always uses 900000-byte buffers); the level only sets the header digit.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "cli.h"
#include "compression.h"
#include "io.h"

static bool write_file(const std::string &name, const std::vector<uint8_t> &data) {
  std::ofstream f(name, std::ios::out | std::ios::binary);
  if (!f) {
    std::cerr << "Failed to open file for writing: " << name << std::endl;
    return false;
  }
  f.write(reinterpret_cast<const char *>(data.data()), (std::streamsize)data.size());
  return f.good();
}

int main(int argc, char **argv) {
  CliOptions opt = parse_args(argc, argv);
  const bool timing = std::getenv("BZ2G_TIMING") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  int rc = 0;
  if (opt.input_files.empty()) {
    BZFileInputStream in(10, 900000);
    std::vector<uint8_t> out;
    bzip2_gpu_compress(in, opt.block_size, out);
    std::cout.write(reinterpret_cast<const char *>(out.data()), (std::streamsize)out.size());
    if (in.failed()) rc = 1;
  } else {
    for (const auto &file : opt.input_files) {
      BZFileInputStream in(10, 900000, file);
      if (in.failed()) {
        rc = 1;
        continue;
      }
      std::vector<uint8_t> out;
      bzip2_gpu_compress(in, opt.block_size, out);
      if (in.failed()) {
        rc = 1;
        continue;
      }
      if (opt.stdout_output)
        std::cout.write(reinterpret_cast<const char *>(out.data()), (std::streamsize)out.size());
      else if (!write_file(file + ".bz2", out))
        rc = 1;
    }
  }
  std::cout.flush();
  if (timing) {
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                    .count();
    std::cerr << "All: " << ms << "\n";
  }
  return rc;
}
