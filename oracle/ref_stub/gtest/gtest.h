/* Minimal stand-in for <gtest/gtest.h>, written for this project so the
 * reference's test sources compile without GoogleTest.  TEST bodies become
 * unused static functions; only the CPU oracle functions defined beside them
 * in those files are called (from oracle/ref_testoracles.cpp).
 * TEST INFRASTRUCTURE ONLY. */
#pragma once
#define TEST(suite, name) [[maybe_unused]] static void suite##_##name##_unused_body()
#define ORC_STUB_CHECK(c) do { if (!(c)) return; } while (0)
#define ASSERT_EQ(a, b) ORC_STUB_CHECK((a) == (b))
#define ASSERT_NE(a, b) ORC_STUB_CHECK((a) != (b))
#define ASSERT_GE(a, b) ORC_STUB_CHECK((a) >= (b))
#define ASSERT_LE(a, b) ORC_STUB_CHECK((a) <= (b))
#define ASSERT_GT(a, b) ORC_STUB_CHECK((a) > (b))
#define ASSERT_LT(a, b) ORC_STUB_CHECK((a) < (b))
#define EXPECT_EQ(a, b) (void)((a) == (b))
