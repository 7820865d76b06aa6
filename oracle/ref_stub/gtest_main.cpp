/* Runner for the reference's test sources compiled with ORC_GTEST_RUNNER
 * (oracle/ref_stub/gtest/gtest.h).  TEST INFRASTRUCTURE ONLY.
 * Runs every registered test in registration order, prints one line per test
 * and a summary, and exits 1 if any test failed.  An optional argument keeps
 * only the tests whose "suite.name" contains it. */
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gtest/gtest.h"

namespace orc_gtest {
namespace {
struct Entry {
  std::string name;
  TestFn fn;
};
std::vector<Entry> &registry() {
  static std::vector<Entry> r;
  return r;
}
bool g_failed = false;
}  // namespace

int add_test(const char *suite, const char *name, TestFn fn) {
  registry().push_back({std::string(suite) + "." + name, fn});
  return (int)registry().size() - 1;
}

void fail() { g_failed = true; }

}  // namespace orc_gtest

int main(int argc, char **argv) {
  using namespace orc_gtest;
  const char *filter = argc > 1 ? argv[1] : nullptr;
  int passed = 0, failed = 0;
  for (const Entry &e : registry()) {
    if (filter && !std::strstr(e.name.c_str(), filter)) continue;
    std::printf("[ RUN      ] %s\n", e.name.c_str());
    std::fflush(stdout);
    g_failed = false;
    e.fn();
    if (g_failed) {
      failed++;
      std::printf("[  FAILED  ] %s\n", e.name.c_str());
    } else {
      passed++;
      std::printf("[       OK ] %s\n", e.name.c_str());
    }
    std::fflush(stdout);
  }
  std::printf("%d passed, %d failed\n", passed, failed);
  return failed ? 1 : 0;
}
