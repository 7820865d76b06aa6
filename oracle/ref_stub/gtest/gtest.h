/* Minimal stand-in for <gtest/gtest.h>, written for this project so the
 * reference's test sources compile without GoogleTest (absent here).
 * TEST INFRASTRUCTURE ONLY.
 *
 * Two modes:
 *  - default: TEST bodies become unused static functions; only the CPU
 *    oracle functions defined beside them in those files are used (the
 *    reference's test oracles, oracle/ref_testoracles.cpp).
 *  - ORC_GTEST_RUNNER defined: a small test runner.  Every TEST registers
 *    itself; ASSERT_* on failure prints the file, line and both values and
 *    leaves the test; EXPECT_* prints and marks the test failed but goes on.
 *    oracle/ref_stub/gtest_main.cpp runs every registered test and exits
 *    non-zero if any failed.
 */
#pragma once

#ifndef ORC_GTEST_RUNNER

#define TEST(suite, name) [[maybe_unused]] static void suite##_##name##_unused_body()
#define ORC_STUB_CHECK(c) do { if (!(c)) return; } while (0)
#define ASSERT_EQ(a, b) ORC_STUB_CHECK((a) == (b))
#define ASSERT_NE(a, b) ORC_STUB_CHECK((a) != (b))
#define ASSERT_GE(a, b) ORC_STUB_CHECK((a) >= (b))
#define ASSERT_LE(a, b) ORC_STUB_CHECK((a) <= (b))
#define ASSERT_GT(a, b) ORC_STUB_CHECK((a) > (b))
#define ASSERT_LT(a, b) ORC_STUB_CHECK((a) < (b))
#define EXPECT_EQ(a, b) (void)((a) == (b))

#else

#include <cstddef>
#include <cstdio>
#include <sstream>
#include <string>
#include <type_traits>

namespace orc_gtest {

using TestFn = void (*)();
// Registers a test; returns its index.
int add_test(const char *suite, const char *name, TestFn fn);
// Marks the running test failed.
void fail();

template <typename T>
std::string show(const T &v) {
  std::ostringstream os;
  if constexpr (std::is_same<T, std::nullptr_t>::value)
    os << "nullptr";
  else if constexpr (std::is_pointer<T>::value)
    os << (const void *)v;  // an address, never the bytes it points to
  else if constexpr (sizeof(T) == 1 && std::is_integral<T>::value)
    os << (int)v;
  else
    os << v;
  return os.str();
}

template <typename A, typename B>
bool report(bool ok, const char *expr, const A &a, const B &b, const char *file, int line) {
  if (!ok) {
    std::fprintf(stderr, "%s:%d: failure: %s (values %s, %s)\n", file, line, expr,
                 show(a).c_str(), show(b).c_str());
    fail();
  }
  return ok;
}

}  // namespace orc_gtest

#define TEST(suite, name)                                                              \
  static void suite##_##name##_body();                                                 \
  [[maybe_unused]] static const int suite##_##name##_reg =                             \
      orc_gtest::add_test(#suite, #name, &suite##_##name##_body);                     \
  static void suite##_##name##_body()

#define ORC_CMP(op, a, b, on_fail)                                                     \
  do {                                                                                 \
    const auto &orc_a_ = (a);                                                          \
    const auto &orc_b_ = (b);                                                          \
    if (!orc_gtest::report(orc_a_ op orc_b_, #a " " #op " " #b, orc_a_, orc_b_,       \
                           __FILE__, __LINE__)) {                                      \
      on_fail;                                                                         \
    }                                                                                  \
  } while (0)

#define ASSERT_EQ(a, b) ORC_CMP(==, a, b, return)
#define ASSERT_NE(a, b) ORC_CMP(!=, a, b, return)
#define ASSERT_GE(a, b) ORC_CMP(>=, a, b, return)
#define ASSERT_LE(a, b) ORC_CMP(<=, a, b, return)
#define ASSERT_GT(a, b) ORC_CMP(>, a, b, return)
#define ASSERT_LT(a, b) ORC_CMP(<, a, b, return)
#define EXPECT_EQ(a, b) ORC_CMP(==, a, b, (void)0)

#endif
