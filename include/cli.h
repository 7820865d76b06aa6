/*
 * cli.h -- command line options of the bzip2gpu tool.
 * Replaces the reference's include/cli.h:7-14 and src/utils/argsparce.cpp:
 * -h/--help, -z/--compress, -c/--stdout, -1..-9, --fast (-1), --best (-9),
 * then input files.
 */
#ifndef BZ2GPU_B200_CLI_H
#define BZ2GPU_B200_CLI_H

#include <string>
#include <vector>

struct CliOptions {
  bool compress = true;
  bool stdout_output = false;
  int block_size = 9;
  std::vector<std::string> input_files;
};

CliOptions parse_args(int argc, char **argv);

#endif
